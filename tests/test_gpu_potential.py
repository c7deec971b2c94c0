"""GPU screened-potential producer (cpw_b200_pot_local) against the host potential.

The host builds vscr by placing V(G) on the box and taking numpy's unscaled backward FFT
(pseudo.local_potential_box, the route of Src/cpw_lib/pot_local.f90); the device gets the same
V(G) through pot_local's star arguments and must give the same vscr within 1e-12 of max|vscr|,
the same mesh (kmscr(4:7)) and extrema. Star structures with partners (G, -G) taking the
conjugate, and with non-trivial phases, exercise both branches of the unfolding; a non-real
potential is rejected like the reference's stop; the installed potential drives H|psi> exactly
as the uploaded vscr does.
"""
import numpy as np
import pytest

from cpw2000_b200 import configs, pseudo
from cpw2000_b200 import hk_psi as H
from cpw2000_b200._lib import CpwB200Error

pytestmark = pytest.mark.gpu

TOL = 1e-12


def relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def workload(name):
    return configs.WORKLOADS[name]()


@pytest.mark.parametrize("name,idpad", [("si2", 0), ("si2", 3), ("si64", 0), ("zb64", 1)])
def test_one_star_per_g_matches_host(cuda, name, idpad):
    w = workload(name)
    want, _ = pseudo.local_potential_box(w.species, w.adot, w.box, idpad)
    kgv, vg = pseudo.local_potential_coefficients(w.species, w.adot, w.box)
    km = [(n - 1) // 2 for n in w.box]
    r = H.Context(0).pot_local(vg, kgv, np.arange(1, vg.size + 1), kmscr=km, idshift=idpad, install=False)
    assert tuple(r["kmscr"][3:6]) == tuple(w.box) and r["kmscr"][6] == w.box[0] + idpad
    assert relerr(r["vscr"], want) < TOL
    n1 = w.box[0]
    body = want.reshape(w.box[2], w.box[1], n1 + idpad)[:, :, :n1]
    assert abs(r["vmax"] - body.max()) < 1e-10 and abs(r["vmin"] - body.min()) < 1e-10
    assert r["cmax"] < 1e-9


def test_stars_with_conjugate_partners_and_phases(cuda):
    w = workload("si2")
    want, _ = pseudo.local_potential_box(w.species, w.adot, w.box)
    kgv, vg = pseudo.local_potential_coefficients(w.species, w.adot, w.box)
    key = {tuple(g): i for i, g in enumerate(kgv.T)}
    rng = np.random.default_rng(5)
    veff, inds, phase, conj = [], np.zeros(vg.size, np.int32), np.ones(vg.size, np.complex128), np.ones(vg.size)
    for i, g in enumerate(kgv.T):
        if inds[i]:
            continue
        j = key.get(tuple(-g))
        ph = np.exp(2j * np.pi * rng.random())
        veff.append(vg[i] * ph)          # unfolded as veff * conj(phase) = V(G)
        inds[i] = len(veff)
        phase[i] = ph
        if j is not None and j != i:     # -G: conj(veff) * phase' = V(-G) = conj(V(G)) with phase' = ph
            inds[j] = len(veff)
            phase[j] = ph
            conj[j] = -1.0
    assert len(veff) < vg.size           # the partners really share stars
    km = [(n - 1) // 2 for n in w.box]
    r = H.Context(0).pot_local(np.array(veff), kgv, inds, phase=phase, conj=conj, kmscr=km, install=False)
    assert relerr(r["vscr"], want) < TOL


def test_complex_potential_is_rejected(cuda):
    w = workload("si2")
    kgv, vg = pseudo.local_potential_coefficients(w.species, w.adot, w.box)
    vg = vg.copy()
    vg[1] += 0.5j                        # breaks V(-G) = conj(V(G))
    km = [(n - 1) // 2 for n in w.box]
    with pytest.raises(CpwB200Error, match="complex potential"):
        H.Context(0).pot_local(vg, kgv, np.arange(1, vg.size + 1), kmscr=km, install=False)


@pytest.mark.parametrize("prec", [H.FP64, H.MIXED])
def test_installed_potential_drives_hpsi(cuda, prec):
    import torch
    w = workload("si64")
    d = configs.kpoint_inputs(w, 0)
    nb = 12
    psi = configs.random_psi(d["mtxd"], nb, 3)
    x = torch.from_numpy(np.ascontiguousarray(psi.T)).to(cuda).t()
    ref = H.Context(0, precision=prec).setup(d)
    y_ref = torch.zeros((nb, d["mtxd"]), dtype=torch.complex128, device=cuda).t()
    ref.hk_psi(x, y_ref)
    ctx = H.Context(0, precision=prec)
    ctx.set_kpoint(d["mtxd"], d["isort"], d["kgv"], d["ekpg"], d["kmscr"])
    kgv, vg = pseudo.local_potential_coefficients(w.species, w.adot, w.box)
    ctx.pot_local(vg, kgv, np.arange(1, vg.size + 1), kmscr=d["kmscr"][:3], install=True, want_vscr=False)
    ctx.set_projectors(d["anlga"], d["xnlkb"])
    y = torch.zeros_like(y_ref)
    ctx.hk_psi(x, y)
    torch.cuda.synchronize()
    assert relerr(y.cpu().numpy(), y_ref.cpu().numpy()) < (1e-12 if prec == H.FP64 else 1e-6)


def test_empty_star_list_gives_zero_potential(cuda):
    w = workload("si2")
    km = [(n - 1) // 2 for n in w.box]
    r = H.Context(0).pot_local(np.zeros(1, complex), np.zeros((3, 0), np.int32), np.zeros(0, np.int32), kmscr=km,
                               install=False)
    assert np.all(r["vscr"] == 0.0) and r["cmax"] == 0.0 and r["vmax"] == 0.0 and r["vmin"] == 0.0
