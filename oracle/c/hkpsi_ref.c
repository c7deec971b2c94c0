/*
 * C + OpenMP restatement of cpw2000's hk_psi_c16 -- TEST AND CPU-TIMING INFRASTRUCTURE ONLY.
 *
 * Follows the loop structure of Src/hk_psi/reference/hk_psi_c16.f90:176-231:
 * per band, zero the box, scatter psi into ipoint, backward pruned 3D FFT
 * (Src/fft/_cfft/cfft_wf_c16.f:246-410: x on the kept (y,z) pencils, y on the
 * kept z planes, z everywhere, zeroing the untrusted entries first), multiply
 * by vscr, forward pruned FFT (:123-242, scaled 1/N on the kept pencils),
 * gather, add ekpg*psi; then the two ZGEMMs of Src/cpw_lib/hk_psi_nl_c16.f90
 * (:82-97). As in the reference, OpenMP parallelises inside each band: over
 * the pencils of every FFT pass and over the elements of the pointwise loops.
 *
 * The 1D transforms are our own mixed-radix Stockham autosort FFT (radix 2, 3,
 * 4, 5 butterflies, generic O(p^2) for other primes), standing in for the
 * FFTPACK backend of Src/fft/_ncar (any exact FFT gives the same result to
 * rounding). The GEMMs are plain OpenMP loops, like the vendored netlib BLAS
 * of Src/LIBS/blas that the reference links when COMPBLAS=true, unless an
 * optimised cblas_zgemm is handed in with cpw_ref_set_zgemm (the reference's
 * default build, COMPBLAS=false at Src/config/make.inc:95, links an external
 * optimised BLAS).
 *
 * Build: see oracle/Makefile (gcc -O3 -fopenmp -shared).
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

typedef struct {
  int n;
  int nf;
  int fac[40];
  cplx* w; /* exp(-2 pi i k / n), k = 0..n-1 */
} plan1d;

static int plan_make(plan1d* p, int n) {
  p->n = n;
  p->nf = 0;
  int m = n;
  while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
  while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
  for (int f = 3; m > 1; f += 2)
    while (m % f == 0) { p->fac[p->nf++] = f; m /= f; }
  p->w = (cplx*)malloc(sizeof(cplx) * (size_t)n);
  if (!p->w) return -1;
  const long double tp = 6.283185307179586476925286766559005768L;
  for (int k = 0; k < n; ++k) {
    long double a = tp * k / n;
    p->w[k] = (double)cosl(a) - I * (double)sinl(a);
  }
  return 0;
}

static void plan_free(plan1d* p) { free(p->w); p->w = NULL; }

/* one radix-r pass of the Stockham autosort FFT; sign = +1 backward, -1 forward */
static void stockham_pass(const plan1d* p, int r, int ns, const cplx* in, cplx* out, int sign) {
  const int n = p->n, nr = n / r;
  cplx v[64];
  for (int j = 0; j < nr; ++j) {
    const int k = j % ns;
    for (int q = 0; q < r; ++q) {
      cplx x = in[j + q * nr];
      int t = (int)(((long long)k * q * (n / (ns * r))) % n);
      cplx w = p->w[t];
      if (sign > 0) w = conj(w);
      v[q] = (t == 0) ? x : x * w;
    }
    cplx o[64];
    if (r == 2) {
      o[0] = v[0] + v[1]; o[1] = v[0] - v[1];
    } else if (r == 4) {
      cplx a0 = v[0] + v[2], a1 = v[0] - v[2], b0 = v[1] + v[3];
      cplx b1 = (v[1] - v[3]) * (sign > 0 ? I : -I);
      o[0] = a0 + b0; o[2] = a0 - b0; o[1] = a1 + b1; o[3] = a1 - b1;
    } else if (r == 3) {
      const double h = 0.866025403784438646763723170752936183;
      cplx t1 = v[1] + v[2], t2 = v[0] - 0.5 * t1, t3 = (v[1] - v[2]) * (sign > 0 ? I : -I) * h;
      o[0] = v[0] + t1; o[1] = t2 + t3; o[2] = t2 - t3;
    } else {
      for (int a = 0; a < r; ++a) {
        cplx s = 0;
        for (int b = 0; b < r; ++b) {
          cplx w = p->w[((long long)a * b % r) * (n / r)];
          if (sign > 0) w = conj(w);
          s += v[b] * w;
        }
        o[a] = s;
      }
    }
    const int d = (j / ns) * ns * r + k;
    for (int q = 0; q < r; ++q) out[d + q * ns] = o[q];
  }
}

/* transform a contiguous line in place using work buffer tmp (length n) */
static void fft_line(const plan1d* p, cplx* x, cplx* tmp, int sign) {
  cplx* a = x;
  cplx* b = tmp;
  int ns = 1;
  for (int f = 0; f < p->nf; ++f) {
    stockham_pass(p, p->fac[f], ns, a, b, sign);
    ns *= p->fac[f];
    cplx* t = a; a = b; b = t;
  }
  if (a != x) memcpy(x, a, sizeof(cplx) * (size_t)p->n);
}

typedef struct {
  int n1, n2, n3, id, kd1, kd2, kd3;
  plan1d p1, p2, p3;
} box_t;

static int kept(int i, int n, int kd) { return i <= kd || i >= n - kd; }

/* cfft_wf_c16, MODE = -1 (sign +1) or MODE = +1 (sign -1, scaled) on chd(id, n2, n3) */
static void cfft_wf(box_t* B, cplx* chd, int mode) {
  const int n1 = B->n1, n2 = B->n2, n3 = B->n3, id = B->id;
  const int kd1 = B->kd1, kd2 = B->kd2, kd3 = B->kd3;
  const size_t sy = (size_t)id, sz = (size_t)id * n2;
  const int maxn = n1 > n2 ? (n1 > n3 ? n1 : n3) : (n2 > n3 ? n2 : n3);
  if (mode == -1) {
#pragma omp parallel
    {
      cplx* buf = (cplx*)malloc(sizeof(cplx) * 2 * (size_t)maxn);
      cplx* tmp = buf + maxn;
      /* dim 1 on the kept (y, z) pencils */
#pragma omp for schedule(static, 4)
      for (int zz = 0; zz < 2 * kd3 + 1; ++zz) {
        const int k = zz <= kd3 ? zz : n3 - (2 * kd3 + 1) + zz;
        for (int j = 0; j < n2; ++j) {
          if (!kept(j, n2, kd2)) continue;
          cplx* line = chd + k * sz + j * sy;
          for (int i = kd1 + 1; i < n1 - kd1; ++i) line[i] = 0;
          fft_line(&B->p1, line, tmp, +1);
        }
      }
      /* dim 2 on the kept z planes */
#pragma omp for schedule(static, 4)
      for (int zz = 0; zz < 2 * kd3 + 1; ++zz) {
        const int k = zz <= kd3 ? zz : n3 - (2 * kd3 + 1) + zz;
        for (int i = 0; i < n1; ++i) {
          cplx* base = chd + k * sz + i;
          for (int j = 0; j < n2; ++j) buf[j] = kept(j, n2, kd2) ? base[j * sy] : 0;
          fft_line(&B->p2, buf, tmp, +1);
          for (int j = 0; j < n2; ++j) base[j * sy] = buf[j];
        }
      }
      /* dim 3 everywhere */
#pragma omp for schedule(static, 4)
      for (int j = 0; j < n2; ++j) {
        for (int i = 0; i < n1; ++i) {
          cplx* base = chd + j * sy + i;
          for (int k = 0; k < n3; ++k) buf[k] = kept(k, n3, kd3) ? base[k * sz] : 0;
          fft_line(&B->p3, buf, tmp, +1);
          for (int k = 0; k < n3; ++k) base[k * sz] = buf[k];
        }
      }
      free(buf);
    }
  } else {
    const double fac = 1.0 / ((double)n1 * n2 * n3);
#pragma omp parallel
    {
      cplx* buf = (cplx*)malloc(sizeof(cplx) * 2 * (size_t)maxn);
      cplx* tmp = buf + maxn;
#pragma omp for schedule(static, 4)
      for (int j = 0; j < n2; ++j) {
        for (int i = 0; i < n1; ++i) {
          cplx* base = chd + j * sy + i;
          for (int k = 0; k < n3; ++k) buf[k] = base[k * sz];
          fft_line(&B->p3, buf, tmp, -1);
          for (int k = 0; k < n3; ++k) base[k * sz] = buf[k];
        }
      }
#pragma omp for schedule(static, 4)
      for (int zz = 0; zz < 2 * kd3 + 1; ++zz) {
        const int k = zz <= kd3 ? zz : n3 - (2 * kd3 + 1) + zz;
        for (int i = 0; i < n1; ++i) {
          cplx* base = chd + k * sz + i;
          for (int j = 0; j < n2; ++j) buf[j] = base[j * sy];
          fft_line(&B->p2, buf, tmp, -1);
          for (int j = 0; j < n2; ++j) base[j * sy] = buf[j];
        }
      }
#pragma omp for schedule(static, 4)
      for (int zz = 0; zz < 2 * kd3 + 1; ++zz) {
        const int k = zz <= kd3 ? zz : n3 - (2 * kd3 + 1) + zz;
        for (int j = 0; j < n2; ++j) {
          if (!kept(j, n2, kd2)) continue;
          cplx* line = chd + k * sz + j * sy;
          fft_line(&B->p1, line, tmp, -1);
          for (int i = 0; i < n1; ++i) line[i] *= fac;
        }
      }
      free(buf);
    }
  }
}

/* an optimised complex GEMM with the 64-bit-integer CBLAS interface (column-major) */
typedef void (*zgemm64_fn)(int order, int transa, int transb, long long m, long long n, long long k,
                           const void* alpha, const void* a, long long lda, const void* b, long long ldb,
                           const void* beta, void* c, long long ldc);
static zgemm64_fn g_zgemm = NULL;
void cpw_ref_set_zgemm(void* fn) { g_zgemm = (zgemm64_fn)fn; }
int cpw_ref_has_zgemm(void) { return g_zgemm != NULL; }

int cpw_ref_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/*
 * hpsi(:mtxd, :neig) = H psi. ipoint is 0-based (hk_psi_c16.f90:145-158 minus
 * one). psi/hpsi/anlga column-major complex(8) with leading dims ld/ldh/lda.
 * Returns 0, or -1 on allocation failure.
 */
int cpw_ref_hk_psi(int mtxd, int neig, const cplx* psi, int ld, cplx* hpsi, int ldh, const int* ipoint,
                   int kd1, int kd2, int kd3, int n1, int n2, int n3, int id, const double* vscr,
                   const double* ekpg, const cplx* anlga, int lda, const double* xnlkb, int nanl, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  box_t B;
  B.n1 = n1; B.n2 = n2; B.n3 = n3; B.id = id; B.kd1 = kd1; B.kd2 = kd2; B.kd3 = kd3;
  if (plan_make(&B.p1, n1) || plan_make(&B.p2, n2) || plan_make(&B.p3, n3)) return -1;
  const size_t ntot = (size_t)id * n2 * n3;
  cplx* chd = (cplx*)malloc(sizeof(cplx) * ntot);
  if (!chd) return -1;
  for (int n = 0; n < neig; ++n) {
    const cplx* ps = psi + (size_t)n * ld;
    cplx* hp = hpsi + (size_t)n * ldh;
#pragma omp parallel for
    for (long long i = 0; i < (long long)ntot; ++i) chd[i] = 0;
#pragma omp parallel for
    for (int i = 0; i < mtxd; ++i) chd[ipoint[i]] = ps[i];
    cfft_wf(&B, chd, -1);
#pragma omp parallel for
    for (long long i = 0; i < (long long)ntot; ++i) chd[i] *= vscr[i];
    cfft_wf(&B, chd, 1);
#pragma omp parallel for
    for (int i = 0; i < mtxd; ++i) hp[i] = chd[ipoint[i]] + ekpg[i] * ps[i];
  }
  free(chd);
  plan_free(&B.p1); plan_free(&B.p2); plan_free(&B.p3);
  if (nanl > 0 && neig > 0) {
    cplx* dhd = (cplx*)malloc(sizeof(cplx) * (size_t)nanl * neig);
    if (!dhd) return -1;
    if (g_zgemm) {
      /* the two ZGEMMs of hk_psi_nl_c16.f90:82 and :95 in the optimised BLAS (CblasColMajor 102,
         CblasNoTrans 111, CblasConjTrans 113) */
      const cplx one = 1.0, zero = 0.0;
      g_zgemm(102, 113, 111, nanl, neig, mtxd, &one, anlga, lda, psi, ld, &zero, dhd, nanl);
      for (int n = 0; n < neig; ++n)
        for (int a = 0; a < nanl; ++a) dhd[(size_t)n * nanl + a] *= xnlkb[a];
      g_zgemm(102, 111, 111, mtxd, neig, nanl, &one, anlga, lda, dhd, nanl, &one, hpsi, ldh);
      free(dhd);
      return 0;
    }
    /* dhd = anlga^H psi ; dhd = diag(xnlkb) dhd */
#pragma omp parallel for collapse(2) schedule(static)
    for (int n = 0; n < neig; ++n)
      for (int a = 0; a < nanl; ++a) {
        const cplx* x = anlga + (size_t)a * lda;
        const cplx* p = psi + (size_t)n * ld;
        cplx s = 0;
        for (int i = 0; i < mtxd; ++i) s += conj(x[i]) * p[i];
        dhd[(size_t)n * nanl + a] = xnlkb[a] * s;
      }
    /* hpsi += anlga dhd */
#pragma omp parallel for schedule(static)
    for (int n = 0; n < neig; ++n) {
      cplx* h = hpsi + (size_t)n * ldh;
      for (int a = 0; a < nanl; ++a) {
        const cplx t = dhd[(size_t)n * nanl + a];
        const cplx* x = anlga + (size_t)a * lda;
        for (int i = 0; i < mtxd; ++i) h[i] += x[i] * t;
      }
    }
    free(dhd);
  }
  return 0;
}
