"""Block iterative eigensolver restated from Src/ditsp (CPU, FP64) -- test infrastructure only.

ditsp_c16        -- Src/ditsp/ditsp_c16.f90 (driver, :140-141 init, :218-232
                    full diagonalisation, :302-388 outer/inner loops, :379
                    convergence, :387 mcref, :412 ifail)
_start           -- Src/ditsp/ditsp_c16_start.f90:116-256
_loop            -- Src/ditsp/ditsp_c16_loop.f90:147-557
_ritz            -- Src/ditsp/ditsp_c16_ritz.f90:117-306
grsch_loop       -- Src/ditsp/grsch_loop_c16.f90:96-131
grsch_mm         -- Src/ditsp/grsch_mm_c16.f90 / grsch_mm_2_c16.f90 (one recursion)
grsch_mod        -- Src/ditsp/grsch_mod_c16.f90:77-147
grsch_shift      -- Src/ditsp/grsch_shift_c16.f90:57-69
diag_c16         -- Src/ditsp/diag_c16.f90 (LAPACK zheevd 'V','L')
diag_rq_jac      -- Src/omp/diag_rq_jac_c16.f90:67-79
ditsp_error      -- Src/ditsp/ditsp_error.f90:69-76
Ran2             -- Src/numeric/ran2.f90

Fortran default-real literals (0.2, 0.95, 0.9999, ...) are kept at their
single-precision values, as the reference compiles them.
"""
from __future__ import annotations

import numpy as np
from scipy.linalg import lapack


def _r4(x: float) -> float:
    return float(np.float32(x))


C_0P2, C_0P01, C_0P95, C_0P99 = _r4(0.2), _r4(0.01), _r4(0.95), _r4(0.99)
C_0P9999, C_1P2, C_EPS20 = _r4(0.9999), _r4(1.2), _r4(1.0e-20)
_TRACE = False


class Ran2:
    """Numerical-Recipes ran2 with SAVE state, Src/numeric/ran2.f90.

    A negative seed re-initialises the shuffle table (ditsp_c16 passes
    iseed = -1 on every call, ditsp_c16.f90:140).
    """
    M, IA, IC = 714025, 1366, 150889
    RM = 1.4005111865831e-6

    def __init__(self):
        self.ir = [0] * 97
        self.iy = 0
        self.iff = 0

    def __call__(self, idum: list) -> float:
        if idum[0] < 0 or self.iff == 0:
            self.iff = 1
            idum[0] = (self.IC - idum[0]) % self.M
            for j in range(97):
                idum[0] = (self.IA * idum[0] + self.IC) % self.M
                self.ir[j] = idum[0]
            idum[0] = (self.IA * idum[0] + self.IC) % self.M
            self.iy = idum[0]
        j = (97 * self.iy) // self.M
        if j > 96 or j < 0:
            raise RuntimeError("ran2: problems with random number generator")
        self.iy = self.ir[j]
        val = self.iy * self.RM
        idum[0] = (self.IA * idum[0] + self.IC) % self.M
        self.ir[j] = idum[0]
        return val


def diag_c16(ham: np.ndarray):
    """Eigen-decomposition of a Hermitian matrix with LAPACK zheevd('V','L')."""
    w, v, info = lapack.zheevd(np.asfortranarray(ham), compute_v=1, lower=1)
    if info != 0:
        raise RuntimeError(f"diag_c16 failed, info = {info}")
    return w, v


def diag_rq_jac(phi: np.ndarray, lam: np.ndarray, hdiag: np.ndarray):
    """Jacobi preconditioner: x = hdiag - lambda; x = 1 if x < 1 else 1/x; phi = -x phi."""
    x = hdiag[:, None] - lam[None, :]
    x = np.where(x < 1.0, 1.0, 1.0 / np.where(x < 1.0, 1.0, x))
    phi *= -x
    return phi


def ditsp_error(psi: np.ndarray, hpsi: np.ndarray) -> float:
    """xmax = max_n || H psi_n - <psi_n|H psi_n> psi_n ||^2."""
    if psi.shape[1] == 0:
        return 0.0
    eg = np.real(np.sum(psi.conj() * hpsi, axis=0))
    r = hpsi - psi * eg[None, :]
    return float(np.max(np.real(np.sum(r.conj() * r, axis=0))))


def grsch_mod(also, x, hx, irow, xscl):
    """Modified Gram-Schmidt for <= 10 vectors with a 1e-20 relative drop."""
    eps = C_EPS20
    peq = (1.0 / eps) * np.finfo(np.float64).tiny
    nvec = x.shape[1]
    for i in range(nvec):
        if i > 0:
            xni = float(np.real(np.vdot(x[:, i], x[:, i])))
            xnp = 0.0
            for j in range(i):
                prod = np.vdot(x[:, j], x[:, i])
                xnp += float(np.real(prod * np.conj(prod)))
                x[:, i] -= prod * x[:, j]
                if also:
                    hx[:, i] -= prod * hx[:, j]
            if xnp > C_0P9999 * xni:
                for j in range(i):
                    prod = np.vdot(x[:, j], x[:, i])
                    x[:, i] -= prod * x[:, j]
                    if also:
                        hx[:, i] -= prod * hx[:, j]
        suma = float(np.real(np.vdot(x[:, i], x[:, i])))
        if xscl[i] > peq:
            if suma < eps * xscl[i]:
                suma = 0.0
                irow[i] = 0
            else:
                suma = 1.0 / np.sqrt(suma)
        else:
            suma = 0.0
            irow[i] = 0
        x[:, i] *= suma
        if also:
            hx[:, i] *= suma


def grsch_mm(also, x, hx, irow, xscl):
    """Recursive block Gram-Schmidt (halves, CGS with one conditional repeat)."""
    nvec = x.shape[1]
    if nvec <= 10:
        grsch_mod(also, x, hx, irow, xscl)
        return
    nn = nvec // 2
    grsch_mm(also, x[:, :nn], hx[:, :nn] if also else None, irow[:nn], xscl[:nn])
    xnorm = np.real(np.sum(x[:, nn:].conj() * x[:, nn:], axis=0))
    t = x[:, :nn].conj().T @ x[:, nn:]
    x[:, nn:] -= x[:, :nn] @ t
    if also:
        hx[:, nn:] -= hx[:, :nn] @ t
    xsum = np.real(np.sum(t.conj() * t, axis=0))
    if np.any(xsum > C_0P9999 * xnorm):
        t = x[:, :nn].conj().T @ x[:, nn:]
        x[:, nn:] -= x[:, :nn] @ t
        if also:
            hx[:, nn:] -= hx[:, :nn] @ t
    grsch_mm(also, x[:, nn:], hx[:, nn:] if also else None, irow[nn:], xscl[nn:])


def grsch_loop(also, x, hx, nconv, nvec):
    """Orthonormalise columns nconv..nvec-1 against 0..nconv-1 (twice) and themselves."""
    irow = np.ones(max(nvec, 0), dtype=np.int64)
    if nvec <= nconv:
        return irow
    xscl = np.real(np.sum(x[:, nconv:nvec].conj() * x[:, nconv:nvec], axis=0))
    if nconv > 0:
        for _ in range(2):
            t = x[:, :nconv].conj().T @ x[:, nconv:nvec]
            x[:, nconv:nvec] -= x[:, :nconv] @ t
            if also:
                hx[:, nconv:nvec] -= hx[:, :nconv] @ t
    sub_irow = irow[nconv:nvec]
    grsch_mm(also, x[:, nconv:nvec], hx[:, nconv:nvec] if also else None, sub_irow, xscl)
    irow[nconv:nvec] = sub_irow
    return irow


def grsch_shift(x, nconv, nvec, irow) -> int:
    """Compact the columns with irow != 0 (from nconv on); returns ired."""
    j = nconv
    ired = 0
    for n in range(nconv, nvec):
        if irow[n] == 0:
            ired += 1
        else:
            if j < n:
                x[:, j] = x[:, n]
            j += 1
    return ired


class _State:
    pass


def _compact_eg_work(s, irow, lo, hi):
    n = lo
    for nac in range(lo, hi):
        if irow[nac] != 0:
            if n < nac:
                s.eg[n] = s.eg[nac]
                s.work[n] = s.work[nac]
            n += 1


def _degeneracy_trim(s, ntst):
    """The 'adjusts ntst for degeneracies' while-loop (ditsp_c16_loop.f90:263-290)."""
    for _ in range(s.nconv, ntst + 1):
        emax = max(s.eg[s.nconv:ntst]) if ntst > s.nconv else s.eg[s.nconv]
        emin = emax + 10.0 * s.epsa
        if ntst < s.niter:
            emin = min(emin, min(s.eg[ntst:s.niter]))
        if emax + s.epsa > emin:
            ntst -= 1
            if ntst <= s.nconv:
                break
    return ntst


def _first_unconverged(s, nmax, tol):
    ntst = s.nconv
    for n in range(s.nconv, nmax):
        if s.work[n] > tol:
            break
        ntst = n + 1
    return ntst


def ditsp_c16(hk, neig, mtxd, mtxds, psi, hpsi, hamsm, hdiag, epspsi=1e-5, icmax=40,
              iguess=0, mxdsml=None, mxdbnd=None):
    """Iterative diagonalisation; returns dict(ifail, ei, neig, ihkpsum, psi, hpsi).

    hk(X) applies H (hk_psi_c16) to the columns of X (mtxd x n). psi/hpsi are
    (mtxd, mxdbnd) arrays updated in place. hamsm is the leading mtxds block
    of H. mxdsml defaults to mtxds (h_kb_dia.f90 sets mxdsml = mtxds).
    """
    mxdsml = mtxds if mxdsml is None else mxdsml
    mxdbnd = psi.shape[1] if mxdbnd is None else mxdbnd
    ihkpsum = 0
    if neig < 1:
        return dict(ifail=0, ei=np.zeros(0), neig=neig, ihkpsum=0, psi=psi, hpsi=hpsi)
    if neig > mtxds or neig > mxdbnd or 3 * neig > mxdsml or mtxds > mxdsml:
        raise ValueError("ditsp_c16: array dimensions inconsistent with neig/mtxds")
    s = _State()
    s.eg = np.zeros(max(mtxd, mxdsml) + 2)
    s.work = np.zeros(mxdsml + 2)
    ifail = 0
    xmax = 1.0
    iseed = [-1]
    ran = Ran2()
    mcref = 2
    lconv = False
    if mtxds >= mtxd:
        w, v = diag_c16(hamsm[:mtxds, :mtxds])
        psi[:mtxd, :neig] = v[:mtxd, :neig]
        return dict(ifail=0, ei=w[:neig].copy(), neig=neig, ihkpsum=0, psi=psi, hpsi=hpsi,
                    lnoiter=True)
    bas = np.zeros((mtxd, mxdsml), dtype=np.complex128)
    hbas = np.zeros((mtxd, mxdsml), dtype=np.complex128)
    # ---- start (ditsp_c16_start.f90) ----
    et, tvec = diag_c16(hamsm[:mtxds, :mtxds])
    s.epsa = max(epspsi, abs((et[neig - 1] - et[0]) / float(50 * neig)))
    ndeg = neig
    for i in range(neig, mtxds):
        if abs(et[i] - et[i - 1]) > s.epsa:
            break
        ndeg = i + 1
    ndeg = min(ndeg, mxdbnd)
    niter = ndeg + 1
    if niter < mtxds:
        for i in range(ndeg + 1, mtxds):
            if abs(et[i] - et[i - 1]) > s.epsa:
                break
            niter = i + 1
    else:
        niter = mtxds
    niter = min(niter, mxdbnd)
    nexact = neig
    ecut = C_1P2 * et[neig - 1] - C_0P2 * et[0]
    for i in range(neig, mtxds):
        if et[i] > ecut:
            break
        nexact = i + 1
    nexact = min(nexact, mxdsml // 3, neig + 2 + neig // 5, mtxds // 2) + 3
    imax = nexact - 1
    for i in range(1, imax + 1):
        nexact -= 1
        # et(imax-i+2) - et(imax-i+1), 1-based
        if abs(et[imax - i + 1] - et[imax - i]) > s.epsa:
            break
    nexact = max(niter, nexact)
    if nexact + niter + niter // 5 + 2 > mxdsml:
        raise ValueError("ditsp_c16_start: increase mxdsml")
    bas[:mtxds, :nexact] = tvec[:, :nexact]
    hbas[:, :nexact] = hk(bas[:, :nexact])
    ihkpsum += nexact
    if iguess != 1:
        psi[:mtxd, :niter] = bas[:, :niter]
        hpsi[:mtxd, :niter] = hbas[:, :niter]
        lortho = True
        nitold = 0
    else:
        hpsi[:mtxd, :neig] = hk(psi[:mtxd, :neig])
        ihkpsum += neig
        bas[:, nexact:nexact + neig] = psi[:mtxd, :neig]
        hbas[:, nexact:nexact + neig] = hpsi[:mtxd, :neig]
        lortho = False
        nitold = neig
        if niter > neig:
            psi[:mtxd, neig:niter] = bas[:, neig:niter]
            hpsi[:mtxd, neig:niter] = hbas[:, neig:niter]
    s.nconv = 0
    s.niter = niter
    lsafe = False
    P = psi[:mtxd]
    HP = hpsi[:mtxd]
    for ic in range(1, icmax + 1):
        mcmax = mcref
        lexit = False
        lconv = False
        for mc in range(1, mcmax + 1):
            # ---- ditsp_c16_loop ----
            lconv = False
            lexit = False
            nconv, niter = s.nconv, s.niter
            for n in range(nconv, niter):
                s.eg[n] = float(np.real(np.vdot(P[:, n], HP[:, n])))
                r = HP[:, n] - s.eg[n] * P[:, n]
                s.work[n] = float(np.real(np.vdot(r, r)))
            xmold = xmax
            xmax = 0.0
            nmax = min(ndeg, niter)
            for n in range(nconv, nmax):
                xmax = max(xmax, s.work[n])
            if _TRACE:
                print(f"  oracle loop ic = {ic}  mc = {mc}  nconv = {nconv}  niter = {niter}  xmax = {xmax:.6e}")
            if mc > 1 and xmax > C_0P2 * xmold:
                mcref = mc
                lexit = True
            if not lexit:
                if xmax < epspsi * epspsi and lsafe and niter >= ndeg:
                    if lortho:
                        neig = ndeg
                        lconv = True
                    else:
                        irow = grsch_loop(True, P, HP, nconv, niter)
                        ired = grsch_shift(P, nconv, niter, irow)
                        grsch_shift(HP, nconv, niter, irow)
                        if ired > 0:
                            lsafe = False
                        _compact_eg_work(s, irow, nconv, niter)
                        niter -= ired
                        s.niter = niter
                        lortho = True
                        if nconv < niter:
                            xmax = 0.0
                            nmax = min(niter, ndeg)
                            for n in range(nconv, nmax):
                                xmax = max(xmax, s.work[n])
                            if xmax < epspsi * epspsi and lsafe and niter >= ndeg:
                                neig = ndeg
                                lconv = True
            if not lconv and not lexit and niter == nconv:
                lexit = True
            ntst = nconv
            tol = C_0P01 * epspsi * epspsi
            if not lconv and not lexit:
                ntst = _first_unconverged(s, niter, tol)
                if ntst > nconv:
                    ntst = _degeneracy_trim(s, ntst)
            if not lconv and not lexit:
                if ntst > nconv and not lortho:
                    irow = grsch_loop(True, P, HP, nconv, ntst)
                    irow = np.concatenate([irow, np.ones(max(0, niter - ntst), dtype=np.int64)])
                    ired = grsch_shift(P, nconv, niter, irow)
                    grsch_shift(HP, nconv, niter, irow)
                    if ired > 0:
                        lsafe = False
                    _compact_eg_work(s, irow, nconv, niter)
                    lortho = True
                    ntst -= ired
                    niter -= ired
                    s.niter = niter
                    if ntst > nconv:
                        nmax = ntst
                        ntst = _first_unconverged(s, nmax, tol)
                        if ntst > nconv:
                            ntst = _degeneracy_trim(s, ntst)
            if not lconv and not lexit and niter == nconv:
                lexit = True
            if not lconv and not lexit and ntst > nconv:
                k = ntst - nconv
                vsm = bas[:, nexact + nconv:nexact + ntst].conj().T @ P[:, nconv:ntst]
                for _ in range(10 * mxdbnd):
                    nmax = ntst
                    ntst = nconv
                    lxn = False
                    for n in range(nmax - nconv):
                        xn = float(np.real(np.vdot(vsm[:nmax - nconv, n], vsm[:nmax - nconv, n])))
                        if xn < C_0P95:
                            lxn = True
                            break
                        ntst = nconv + n + 1
                    if lxn:
                        if ntst <= nconv:
                            break
                    else:
                        emax = max(s.eg[nconv:ntst])
                        emin = emax + 10.0 * s.epsa
                        if ntst < niter:
                            emin = min(emin, min(s.eg[ntst:niter]))
                        if emax + s.epsa > emin:
                            ntst -= 1
                            if ntst <= nconv:
                                break
                        else:
                            break
                else:
                    raise RuntimeError("ditsp_c16_loop: span test did not terminate")
                del k
            if not lconv and not lexit:
                if ntst > nconv:
                    bas[:, nexact + nconv:nexact + ntst] = P[:, nconv:ntst]
                    irowb = grsch_loop(False, bas, hbas, nexact + nconv, nexact + ntst)
                    ired = grsch_shift(bas, nexact + nconv, nexact + ntst, irowb)
                    if ired > 0:
                        lsafe = False
                        irow = np.ones(niter, dtype=np.int64)
                        irow[nconv:ntst] = irowb[nexact + nconv:nexact + ntst]
                        grsch_shift(P, nconv, niter, irow)
                        grsch_shift(HP, nconv, niter, irow)
                        _compact_eg_work(s, irow, nconv, niter)
                    nnew = ntst - ired - nconv
                    hbas[:, nexact + nconv:nexact + nconv + nnew] = hk(bas[:, nexact + nconv:nexact + nconv + nnew])
                    ihkpsum += nnew
                    nconv = ntst - ired
                    niter = niter - ired
                    s.nconv, s.niter = nconv, niter
                # relaxation step (Jacobi)
                lam = s.eg[nconv:niter].copy()
                R = HP[:, nconv:niter] - P[:, nconv:niter] * lam[None, :]
                diag_rq_jac(R, lam, hdiag[:mtxd])
                P[:, nconv:niter] += R
                nrm = np.real(np.sum(P[:, nconv:niter].conj() * P[:, nconv:niter], axis=0))
                P[:, nconv:niter] *= (1.0 / np.sqrt(nrm))[None, :]
                lortho = False
                HP[:, nconv:niter] = hk(P[:, nconv:niter])
                ihkpsum += niter - nconv
            if lexit or lconv:
                break
        if not lsafe:
            mcref = 3
        # ---- ditsp_c16_ritz ----
        nconv, niter = s.nconv, s.niter
        lconv = False
        nsize = nexact + nitold + niter - nconv
        nlow = nexact + nitold - nconv
        if nsize > mxdsml:
            raise ValueError("ditsp_c16_ritz: change mxdsml")
        if nconv < niter:
            bas[:, nlow + nconv:nlow + niter] = P[:, nconv:niter]
        if (not lsafe) or niter == nconv:
            nsize += 1
            if nsize > mxdsml:
                raise ValueError("ditsp_c16_ritz: change mxdsml")
            vals = np.empty(2 * mtxd)
            for k in range(mtxd):
                vals[2 * k] = ran(iseed)
                vals[2 * k + 1] = ran(iseed)
            bas[:, nsize - 1] = vals[0::2] + 1j * vals[1::2]
        irowb = grsch_loop(False, bas, hbas, nexact + nconv, nsize)
        ired = grsch_shift(bas, nexact + nconv, nsize, irowb)
        nsize -= ired
        if nsize > mtxd:
            raise RuntimeError("ditsp_c16_ritz: problems with Gram-Schmidt")
        lo = nexact + nconv
        hbas[:, lo:nsize] = hk(bas[:, lo:nsize])
        ihkpsum += nsize - lo
        hsm = hbas[:, :nsize].conj().T @ bas[:, :nsize]
        egs, vsm = diag_c16(hsm)
        s.eg[:nsize] = egs
        ndeg = neig
        for i in range(neig, nsize):
            if abs(s.eg[i] - s.eg[i - 1]) > s.epsa:
                break
            ndeg = i + 1
        ndeg = min(ndeg, mxdbnd)
        niter = ndeg + 1
        if nsize > niter:
            for i in range(ndeg + 1, nsize):
                if abs(s.eg[i] - s.eg[i - 1]) > s.epsa:
                    break
                niter = i + 1
        nmax = (mxdsml - nexact + nconv) // 2
        niter = min(niter, nmax, nexact, mxdbnd)
        niter = max(niter, ndeg)
        if nconv > 0:
            for _ in range(nconv):
                nmax = nconv
                nconv = 0
                ljump = True
                for n in range(nmax):
                    xn = float(np.real(np.vdot(vsm[:nexact + nmax, n], vsm[:nexact + nmax, n])))
                    if xn < C_0P99:
                        ljump = False
                        break
                    nconv = n + 1
                if ljump:
                    if abs(s.eg[nconv] - s.eg[nconv - 1]) < s.epsa:
                        nconv -= 1
                        ljump = False
                if ljump or nconv == 0:
                    break
        P[:, :niter] = bas[:, :nsize] @ vsm[:, :niter]
        HP[:, :niter] = hbas[:, :nsize] @ vsm[:, :niter]
        bas[:, nexact + nconv:nexact + niter] = P[:, nconv:niter]
        hbas[:, nexact + nconv:nexact + niter] = HP[:, nconv:niter]
        if nconv >= ndeg:
            neig = ndeg
            lconv = True
        s.nconv, s.niter = nconv, niter
        xmax = ditsp_error(P[:, :neig], HP[:, :neig])
        if _TRACE:
            print(f"  oracle ritz ic = {ic}  nconv = {nconv}  niter = {niter}  nsize = {nsize}  ndeg = {ndeg}  "
                  f"xmax = {xmax:.6e}  e1 = {s.eg[0]:.12f}")
        lconv = xmax < epspsi * epspsi
        if lconv:
            break
        nitold = niter
        lortho = True
        lsafe = True
        if xmax < C_0P01:
            mcref = min(mcref + 2, 8)
    if not lconv:
        ifail = 1 + int(-np.log10(xmax))
        if ifail == 0:
            ifail = 1
    return dict(ifail=ifail, ei=s.eg[:neig].copy(), neig=neig, ihkpsum=ihkpsum, psi=psi,
                hpsi=hpsi, xmax=xmax, lnoiter=False)
