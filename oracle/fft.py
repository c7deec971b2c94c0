"""Pruned 3D complex FFT, restating Src/fft/_cfft/cfft_wf_c16.f.

Conventions (cfft_wf_c16.f:42-46): MODE = -1 is the backward transform
f(r) = sum_G c(G) e^{+i G.r}, unscaled; MODE = +1 is the forward transform
c(G) = (1/N) sum_r f(r) e^{-i G.r}. The box is CHD(NN1, N2, N3) with NN1 >= N1
(stored here as a C-ordered array of shape (N3, N2, NN1)).

Goedecker pruning (:110-113) is used when N_j > 2 KD_j + 5 in all three
directions: backward transforms dim 1 on the (2KD2+1)(2KD3+1) pencils that can
be non-zero, dim 2 on the 2KD3+1 planes, dim 3 everywhere (:246-410);
forward runs the same passes in reverse order and scales by 1/N only the
pencils it keeps (:123-242). Entries outside the kept region are left with
whatever the pass produced, exactly as the reference leaves them.
"""
from __future__ import annotations

import numpy as np


def _kept(n: int, kd: int) -> np.ndarray:
    """Indices 0..kd and n-kd..n-1 (1-based 1..KD+1, N-KD+1..N)."""
    return np.concatenate([np.arange(0, kd + 1), np.arange(n - kd, n)])


def cfft_wf_c16(chd: np.ndarray, nn1: int, n1: int, n2: int, n3: int,
                kd1: int, kd2: int, kd3: int, mode: int) -> np.ndarray:
    """In-place pruned 3D FFT of chd (complex128, flat size nn1*n2*n3)."""
    if mode not in (1, -1):
        raise ValueError("cfft_wf_c16: MODE should be 1 or -1")
    if min(n1, n2, n3) < 2:
        raise ValueError("cfft_wf_c16: dimension less than 2")
    box = chd.reshape(n3, n2, nn1)
    prune = n1 > 2 * kd1 + 5 and n2 > 2 * kd2 + 5 and n3 > 2 * kd3 + 5
    if not prune:
        return cfft_c16(chd, nn1, n1, n2, n3, mode)
    z = _kept(n3, kd3)
    y = _kept(n2, kd2)
    x = _kept(n1, kd1)
    if mode == -1:
        # dim 1 on kept (y, z) pencils, zeroing untrusted entries first (:260)
        sub = box[np.ix_(z, y, np.arange(n1))]
        mask = np.zeros(n1, dtype=bool)
        mask[x] = True
        sub[:, :, ~mask] = 0
        sub = np.fft.ifft(sub, axis=2) * n1
        box[np.ix_(z, y, np.arange(n1))] = sub
        # dim 2 on kept z planes (:349 zeroes the untrusted y rows)
        pl = box[z, :, :n1]
        ymask = np.zeros(n2, dtype=bool)
        ymask[y] = True
        pl[:, ~ymask, :] = 0
        box[z, :, :n1] = np.fft.ifft(pl, axis=1) * n2
        # dim 3 everywhere, zeroing untrusted planes
        zmask = np.zeros(n3, dtype=bool)
        zmask[z] = True
        col = box[:, :, :n1]
        col[~zmask] = 0
        box[:, :, :n1] = np.fft.ifft(col, axis=0) * n3
    else:
        fac = 1.0 / (n1 * n2 * n3)
        box[:, :, :n1] = np.fft.fft(box[:, :, :n1], axis=0)
        box[z, :, :n1] = np.fft.fft(box[z, :, :n1], axis=1)
        sub = box[np.ix_(z, y, np.arange(n1))]
        box[np.ix_(z, y, np.arange(n1))] = np.fft.fft(sub, axis=2) * fac
    return chd


def cfft_c16(chd: np.ndarray, nn1: int, n1: int, n2: int, n3: int, mode: int) -> np.ndarray:
    """Full 3D FFT (Src/fft/_cfft/cfft_c16.f:106-165), same conventions."""
    box = chd.reshape(n3, n2, nn1)
    if mode == -1:
        box[:, :, :n1] = np.fft.ifftn(box[:, :, :n1]) * (n1 * n2 * n3)
    else:
        box[:, :, :n1] = np.fft.fftn(box[:, :, :n1]) / (n1 * n2 * n3)
    return chd
