"""GPU KB projector set-up (cpw_b200_proj_nl_kb_device) against the host restatement of
Src/omp/proj_nl_kb_c16.f90 (pseudo.proj_nl_kb): the projector columns within 1e-12 of
max|anlga| (FP64 rounding: the device takes the phase from sincospi and the table in the
reference layout), xnlkb exactly, and H|psi> with device-built projectors equal to H|psi>
with uploaded ones. Covers k-points off Gamma, two atom types, l up to 3 (every solid
harmonic), the reference's nanl consistency error and every precision form.
"""
import numpy as np
import pytest

from cpw2000_b200 import configs, pseudo
from cpw2000_b200 import hk_psi as H
from cpw2000_b200._lib import CpwB200Error

pytestmark = pytest.mark.gpu

TOL = 1e-12


def device_projectors(ctx, d, w, torch, dev, vkb=None, nkb=None, species=None):
    vkb = d["vkb"] if vkb is None else vkb
    nkb = d["nkb"] if nkb is None else nkb
    species = w.species if species is None else species
    nanl = pseudo.nanl_of(species, nkb)
    out = torch.zeros((nanl, d["mtxd"]), dtype=torch.complex128, device=dev).t()
    xnl = ctx.proj_nl_kb(d["rkpt"], species, vkb, nkb, w.adot, anlga_out=out)
    torch.cuda.synchronize()
    return out.cpu().numpy(), xnl


def relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("wname,ik", [("si2", 0), ("si2", 3), ("si8_cubic_kbatch", 5), ("zb64_cubic", 0)])
def test_projectors_match_host_restatement(cuda, wname, ik):
    import torch
    w = configs.WORKLOADS[wname]() if wname in configs.WORKLOADS else getattr(configs, wname)()
    d = configs.kpoint_inputs(w, ik)
    ctx = H.Context(0)
    ctx.set_kpoint(d["mtxd"], d["isort"], d["kgv"], d["ekpg"], d["kmscr"])
    got, xnl = device_projectors(ctx, d, w, torch, cuda)
    assert got.shape == d["anlga"].shape
    assert relerr(got, d["anlga"]) < TOL
    assert np.array_equal(xnl, d["xnlkb"])


def test_projectors_up_to_l3(cuda):
    # s, p, d and f channels with both signs of E_KB: every branch of the solid harmonics
    import torch
    w = configs.WORKLOADS["si2"]()
    species = [pseudo.Species(v0=sp.v0, sigma=sp.sigma, ekb=(2.0, -1.5, 0.7, -0.3), sigma_kb=0.9, rat=sp.rat)
               for sp in w.species]
    d = configs.kpoint_inputs(w, 2)
    vkb, nkb = pseudo.kb_tables(species, 0.01, 4000, lmax=3)
    want, xwant = pseudo.proj_nl_kb(d["rkpt"], d["isort"], d["kgv"], species, vkb, nkb, w.adot)
    assert want.shape[1] == 16 * sum(sp.natom for sp in species)
    ctx = H.Context(0)
    ctx.set_kpoint(d["mtxd"], d["isort"], d["kgv"], d["ekpg"], d["kmscr"])
    got, xnl = device_projectors(ctx, d, w, torch, cuda, vkb=vkb, nkb=nkb, species=species)
    assert relerr(got, want) < TOL
    assert np.array_equal(xnl, xwant)


@pytest.mark.parametrize("prec", [H.FP64, H.MIXED, H.MIXED_TC])
def test_hpsi_with_device_projectors(cuda, prec):
    import torch
    w = configs.si64_cubic()
    d = configs.kpoint_inputs(w, 0)
    nb = 24
    psi = configs.random_psi(d["mtxd"], nb, 7)
    x = torch.from_numpy(np.ascontiguousarray(psi.T)).to(cuda).t()
    ref = H.Context(0, precision=prec).setup(d)
    y_ref = torch.zeros((nb, d["mtxd"]), dtype=torch.complex128, device=cuda).t()
    ref.hk_psi(x, y_ref)
    ctx = H.Context(0, precision=prec)
    ctx.set_kpoint(d["mtxd"], d["isort"], d["kgv"], d["ekpg"], d["kmscr"])
    ctx.set_potential(d["vscr"])
    ctx.proj_nl_kb(d["rkpt"], w.species, d["vkb"], d["nkb"], w.adot)
    y = torch.zeros_like(y_ref)
    ctx.hk_psi(x, y)
    torch.cuda.synchronize()
    a, b = y.cpu().numpy(), y_ref.cpu().numpy()
    assert relerr(a, b) < (1e-12 if prec == H.FP64 else 2e-6)


def test_inconsistent_nanl_is_rejected(cuda):
    w = configs.WORKLOADS["si2"]()
    d = configs.kpoint_inputs(w, 0)
    ctx = H.Context(0)
    ctx.set_kpoint(d["mtxd"], d["isort"], d["kgv"], d["ekpg"], d["kmscr"])
    nkb = np.array(d["nkb"])
    nkb[0, 1] = 0          # drop the p channel of the first type: the count no longer matches
    with pytest.raises(CpwB200Error, match="nanl"):
        _call_with_nanl(ctx, d, w, nkb, d["nanl"])


def _call_with_nanl(ctx, d, w, nkb, nanl):
    # the Python wrapper derives nanl from the tables; pass the stale count through the C ABI
    from cpw2000_b200._lib import check, dptr, iptr
    species = w.species
    ntype = len(species)
    natom = np.array([sp.natom for sp in species], dtype=np.int32)
    mxdatm = int(natom.max())
    rat = np.zeros((3, mxdatm, ntype), order="F")
    for t, sp in enumerate(species):
        rat[:, :sp.natom, t] = np.asarray(sp.rat).T
    nq = 4000
    vref = np.zeros((nq + 3, 4, 3, ntype), order="F")
    nref = np.zeros((4, 3, ntype), dtype=np.int32, order="F")
    for t in range(ntype):
        for l in range(4):
            vref[:, l, 1, t] = d["vkb"][t, l]
            nref[l, 1, t] = nkb[t, l]
    rk = np.ascontiguousarray(d["rkpt"], dtype=np.float64)
    ad = np.asfortranarray(w.adot, dtype=np.float64)
    check(ctx._L.cpw_b200_proj_nl_kb_device(ctx.handle, dptr(rk), ntype, iptr(natom), dptr(rat), mxdatm, dptr(ad),
                                            iptr(np.full(ntype, nq, dtype=np.int32)),
                                            dptr(np.full(ntype, 0.01)), dptr(vref), nq, iptr(nref), int(nanl), None,
                                            None, 0))


def test_no_projectors(cuda):
    # species without KB channels: nanl = 0, H|psi> then has no non-local term
    import torch
    w = configs.WORKLOADS["si2"]()
    d = configs.kpoint_inputs(w, 0)
    nkb = np.zeros_like(np.asarray(d["nkb"]))
    ctx = H.Context(0)
    ctx.set_kpoint(d["mtxd"], d["isort"], d["kgv"], d["ekpg"], d["kmscr"])
    ctx.set_potential(d["vscr"])
    xnl = ctx.proj_nl_kb(d["rkpt"], w.species, d["vkb"], nkb, w.adot)
    assert xnl.size == 0 and ctx.nanl == 0
    psi = configs.random_psi(d["mtxd"], 3, 1)
    x = torch.from_numpy(np.ascontiguousarray(psi.T)).to(cuda).t()
    y = torch.zeros((3, d["mtxd"]), dtype=torch.complex128, device=cuda).t()
    ctx.hk_psi(x, y)
    torch.cuda.synchronize()
    from oracle import hk_psi as O
    want = O.hk_psi_c16(d["mtxd"], 3, psi, d["ekpg"], d["isort"], d["vscr"], d["kmscr"], d["kgv"],
                        np.zeros((d["mtxd"], 0), complex), np.zeros(0))
    assert relerr(y.cpu().numpy(), want) < TOL


@pytest.mark.parametrize("ik,nder", [(2, 2), (0, 2), (3, 1), (1, 0)])
def test_projector_k_derivatives_match_restatement(cuda, ik, nder):
    # Src/omp/proj_nl_kb_der_c16.f90 on the device against oracle/projectors.py (itself pinned by
    # finite differences on the CPU): s, p, d and f channels, three atom types, Gamma included
    # (the |k+G| = 0 branch of the second derivative)
    from oracle import projectors as OP
    w = configs.WORKLOADS["si2"]()
    species = [pseudo.Species(v0=sp.v0, sigma=sp.sigma, ekb=(2.0, -1.5, 0.7, -0.3), sigma_kb=0.9, rat=sp.rat)
               for sp in w.species]
    species.append(pseudo.Species(v0=1.0, sigma=0.7, ekb=(0.0, 1.1), sigma_kb=0.8, rat=np.array([[0.3, 0.1, 0.2]])))
    d = configs.kpoint_inputs(w, ik)
    vkb, nkb = pseudo.kb_tables(species, 0.01, 4000, lmax=3)
    nt = len(species)
    a, x, da, d2a = OP.proj_nl_kb_der_c16(d["rkpt"], d["isort"], d["kgv"], [sp.rat for sp in species], vkb, nkb,
                                          np.full(nt, 4000), np.full(nt, 0.01), w.adot, nder)
    ctx = H.Context(0)
    ctx.set_kpoint(d["mtxd"], d["isort"], d["kgv"], d["ekpg"], d["kmscr"])
    A, DA, D2A, xnl = ctx.proj_nl_kb_der(d["rkpt"], species, vkb, nkb, w.adot, nder=nder)
    assert relerr(A.cpu().numpy(), a) < TOL
    assert np.array_equal(xnl, x)
    if nder > 0:
        assert relerr(DA.cpu().numpy(), da) < TOL
    else:
        assert DA is None
    if nder > 1:
        assert relerr(D2A.cpu().numpy(), d2a) < TOL
    ctx.close()
