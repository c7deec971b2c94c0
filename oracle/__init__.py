"""CPU oracle for the H|psi> / block-eigensolver path -- TEST INFRASTRUCTURE ONLY.

This package restates, in plain numpy / scipy FP64, the reference's algorithm
for the path (each function cites the Fortran file:line it follows). It is
the checker: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
legs of ``bench.py`` may import it. The product (``cpw2000_b200``) never calls
it and has no CPU fallback.

Parity status: UNPINNED against reference-produced vectors. The reference is
Fortran, no Fortran compiler exists in the build container, and its own tests
(Validation/verify) only pin whole SCF runs with real pseudopotentials; no
function-level golden vectors exist for hk_psi_c16 / ditsp_c16. The oracle is
instead pinned by self-contained known-answer tests (analytic single plane
waves, explicit dense matrix elements, Hermiticity, dense diagonalisation
ground truth), committed as fixtures under tests/golden/.

Modules
-------
fft      -- Src/fft/_cfft/cfft_wf_c16.f pruned 3D FFT (conventions and pruning)
hk_psi   -- Src/hk_psi/reference/hk_psi_c16.f90, hk_psi_spin_c16.f90 (spinors),
            Src/cpw_lib/hk_psi_nl_c16.f90
ditsp    -- Src/ditsp/*.f90, Src/omp/diag_rq_jac_c16.f90, Src/numeric/ran2.f90
forces   -- Src/ALFA/for_str_nl_kb.f90, Src/ALFA/for_str_local_force.f90, and the density
            Src/omp/charge_by_fft.f90
stress   -- Src/ALFA/for_str_kinetic_stress.f90, for_str_local_stress.f90, for_str_nl_kb.f90 (stress)
c/       -- C + OpenMP restatement of hk_psi_c16 (CPU baseline timing)
"""
