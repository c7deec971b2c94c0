"""B200-native H|psi> and block iterative eigensolver for cpw2000.

Drop-in for cpw2000's ``hk_psi_c16`` (Src/hk_psi/reference/hk_psi_c16.f90) and
``ditsp_c16`` (Src/ditsp/ditsp_c16.f90): the compute runs in hand-written
sm_100a CUDA behind a C ABI (include/cpw_b200.h); this package holds the
host-side set-up and a thin Python mirror of the reference interface.
"""
from . import crystal, pseudo, configs  # noqa: F401

__all__ = ["crystal", "pseudo", "configs"]
