"""FP64-accurate complex GEMM on the int8 tensor cores (cpw_b200_zgemm_i8, csrc/oz.cu) against
an FP64 reference product (numpy complex128 on the CPU).

Shapes of the eigensolver's basis products: tall-skinny Gram products A^H B with a long K
(split over work items), rotations A B with a tall A, accumulation with alpha = -1 (the
Gram-Schmidt update), ragged sizes (M, N, K not multiples of the tiles), and operands whose
magnitudes decay by orders of magnitude along K (plane-wave coefficients of smooth bands).
The triangular modes of the Cholesky QR products: the lower triangle of a Gram matrix (tiles
strictly above the diagonal written as zeros) and a product with an upper-triangular B (the
products with its zero part skipped). Tolerance: 1e-12 of max|C| with 7 slices (the operands carry 48 bits relative to their row
maxima; for K up to 1.8e5 the worst-case FP64 GEMM bound K u |A||B| is looser still); fewer
slices lose 7 bits each, which the slice sweep checks.
"""
import ctypes as C

import numpy as np
import pytest

from cpw2000_b200 import _lib
from cpw2000_b200 import hk_psi as H

pytestmark = pytest.mark.gpu


def _rand(rng, shape, decay=0.0):
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    if decay:
        x *= np.exp(-decay * np.linspace(0, 1, shape[0]))[:, None]
    return np.asfortranarray(x)


def _run(torch, dev, ctx, transa, a, b, m, n, k, alpha=1.0, c0=None, slices=7, tri=None):
    L = _lib.lib()
    A = torch.from_numpy(np.ascontiguousarray(a.T)).to(dev).t()
    B = torch.from_numpy(np.ascontiguousarray(b.T)).to(dev).t()
    Cm = torch.zeros((n, m), dtype=torch.complex128, device=dev).t() if c0 is None else \
        torch.from_numpy(np.ascontiguousarray(c0.T)).to(dev).t()
    # column-major storage: the leading dimension is the row count (torch may report any stride
    # for a dimension of extent 1)
    args = (ctx.handle, ord(transa), m, n, k, C.c_void_p(A.data_ptr()), a.shape[0], C.c_void_p(B.data_ptr()),
            b.shape[0], float(alpha), 0 if c0 is None else 1, C.c_void_p(Cm.data_ptr()), m, slices)
    st = L.cpw_b200_zgemm_i8(*args, None) if tri is None else L.cpw_b200_zgemm_i8_tri(*args, tri, None)
    _lib.check(st)
    ctx.synchronize()
    return Cm.cpu().numpy()


@pytest.mark.parametrize("transa,m,n,k,decay", [("C", 130, 70, 20000, 0.0), ("C", 257, 33, 178001, 8.0),
                                                 ("N", 300, 45, 1000, 0.0), ("N", 1000, 17, 333, 5.0),
                                                 ("C", 1, 1, 5, 0.0), ("N", 129, 65, 64, 0.0)])
def test_zgemm_i8_matches_fp64(cuda, transa, m, n, k, decay):
    import torch
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    ctx = H.Context(0)
    a = _rand(rng, (k, m) if transa == "C" else (m, k), decay if transa == "C" else 0.0)
    b = _rand(rng, (k, n), decay)
    got = _run(torch, cuda, ctx, transa, a, b, m, n, k)
    ref = (a.conj().T if transa == "C" else a) @ b
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 1e-12, f"relative error {err:.3e}"
    ctx.close()


def test_zgemm_i8_accumulate_and_alpha(cuda):
    import torch
    rng = np.random.default_rng(5)
    ctx = H.Context(0)
    m, n, k = 700, 40, 90
    a, b, c0 = _rand(rng, (m, k)), _rand(rng, (k, n)), _rand(rng, (m, n))
    got = _run(torch, cuda, ctx, "N", a, b, m, n, k, alpha=-1.0, c0=c0)
    ref = c0 - a @ b
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-12
    # long K (split into FP64 partials) with accumulation
    m, n, k = 96, 50, 150000
    a, b, c0 = _rand(rng, (k, m)), _rand(rng, (k, n)), _rand(rng, (m, n))
    got = _run(torch, cuda, ctx, "C", a, b, m, n, k, alpha=-1.0, c0=c0)
    ref = c0 - a.conj().T @ b
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-12
    ctx.close()


def test_zgemm_i8_error_shrinks_with_slices(cuda):
    import torch
    rng = np.random.default_rng(9)
    ctx = H.Context(0)
    m, n, k = 64, 24, 4000
    a, b = _rand(rng, (k, m)), _rand(rng, (k, n))
    ref = a.conj().T @ b
    errs = []
    for s in (2, 3, 4, 5, 6, 7):
        got = _run(torch, cuda, ctx, "C", a, b, m, n, k, slices=s)
        errs.append(np.abs(got - ref).max() / np.abs(ref).max())
    # each slice adds 7 bits: the error falls by orders of magnitude until FP64 rounding
    for s, e in zip((2, 3, 4, 5, 6), errs):
        assert e < 2.0 ** (-(6 + 7 * (s - 1)) + 8), (s, e)
    assert errs[-1] < 1e-12
    ctx.close()


@pytest.mark.parametrize("k,m", [(300, 20000), (600, 30000), (70, 5000)])
def test_zgemm_i8_gram_lower_triangle(cuda, k, m):
    # G = X^H X for the lower triangle (Cholesky QR Gram): k x k, K = m, long K split into partials
    import torch
    rng = np.random.default_rng(k + m)
    ctx = H.Context(0)
    x = _rand(rng, (m, k), 4.0)
    got = _run(torch, cuda, ctx, "C", x, x, k, k, m, tri=1)
    ref = x.conj().T @ x
    low = np.tril(np.ones((k, k), dtype=bool))
    err = np.abs(got - ref)[low].max() / np.abs(ref).max()
    assert err < 1e-12, f"lower triangle: relative error {err:.3e}"
    # tiles (128 rows x 32 columns) strictly above the diagonal are zeros; the others are complete
    r = np.arange(k)[:, None]
    c = np.arange(k)[None, :]
    skipped = 32 * (c // 32) > 128 * (r // 128) + 127
    assert np.all(got[skipped] == 0)
    full = ~skipped
    assert np.abs(got - ref)[full].max() / np.abs(ref).max() < 1e-12
    ctx.close()


@pytest.mark.parametrize("m,k,alpha,acc", [(20000, 500, 1.0, False), (5000, 333, -1.0, True), (130, 31, 1.0, False),
                                           (1000, 65, 1.0, False)])
def test_zgemm_i8_upper_triangular_b(cuda, m, k, alpha, acc):
    # X <- X U (Cholesky QR apply of R^-1): B upper triangular k x k
    import torch
    rng = np.random.default_rng(m + k)
    ctx = H.Context(0)
    x = _rand(rng, (m, k))
    u = np.asfortranarray(np.triu(_rand(rng, (k, k))))
    c0 = _rand(rng, (m, k)) if acc else None
    got = _run(torch, cuda, ctx, "N", x, u, m, k, k, alpha=alpha, c0=c0, tri=2)
    ref = alpha * (x @ u) + (c0 if acc else 0)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 1e-12, f"relative error {err:.3e}"
    ctx.close()


def test_zgemm_i8_tri_rejects_non_square(cuda):
    import torch
    ctx = H.Context(0)
    L = _lib.lib()
    a = torch.zeros((4, 8), dtype=torch.complex128, device=cuda)
    st = L.cpw_b200_zgemm_i8_tri(ctx.handle, ord("C"), 4, 3, 8, C.c_void_p(a.data_ptr()), 8, C.c_void_p(a.data_ptr()),
                                 8, 1.0, 0, C.c_void_p(a.data_ptr()), 4, 7, 1, None)
    assert st == 1 and "square" in L.cpw_b200_last_error().decode()
    st = L.cpw_b200_zgemm_i8_tri(ctx.handle, ord("N"), 4, 3, 3, C.c_void_p(a.data_ptr()), 4, C.c_void_p(a.data_ptr()),
                                 3, 1.0, 0, C.c_void_p(a.data_ptr()), 4, 7, 3, None)
    assert st == 1
    ctx.close()
