// Block iterative eigensolver on the GPU, restating Src/ditsp (ditsp_c16 and
// its start/loop/ritz parts, the block Gram-Schmidt family, diag_c16,
// diag_rq_jac_c16 and ditsp_error). The control flow runs on the host with the
// reference's decisions and thresholds; every vector block (psi, hpsi, the
// iterative basis bas/hbas) stays in device memory. Dense products are cuBLAS
// ZGEMMs, the subspace eigensolve is cuSOLVER zheevd ('V', lower), and the
// column reductions / Jacobi relaxation are the kernels below. H|psi> is the
// context's operator (FP64 drop-in or the mixed-precision form).
#include <cusolverDn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <complex>
#include <string>
#include <vector>

#include "../../include/cpw_b200.h"
#include "context.hpp"

namespace cpwb {
namespace {

using Z = cuDoubleComplex;
using zc = std::complex<double>;

float r4(double x) { return (float)x; }
// Fortran default-real literals as the reference compiles them
const double C0P2 = r4(0.2), C0P01 = r4(0.01), C0P95 = r4(0.95), C0P99 = r4(0.99), C0P9999 = r4(0.9999);
const double C1P2 = r4(1.2), CEPS20 = r4(1.0e-20);

// --------------------------- column kernels ---------------------------
constexpr int kColThreads = 256;

// Sum over the block, returned to every thread (fixed order: deterministic).
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < (blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[32] = v;
  }
  __syncthreads();
  v = sh[32];
  __syncthreads();
  return v;
}

// out[j] = sum_i conj(x_ij) y_ij, one CTA per column (deterministic order)
__global__ void k_coldot(int m, const Z* __restrict__ x, long long ldx, const Z* __restrict__ y, long long ldy,
                         Z* __restrict__ out) {
  __shared__ double sh[33];
  const int j = blockIdx.x;
  const Z* a = x + (size_t)j * ldx;
  const Z* b = y + (size_t)j * ldy;
  double re = 0, im = 0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const Z u = a[i], v = b[i];
    re += u.x * v.x + u.y * v.y;
    im += u.x * v.y - u.y * v.x;
  }
  re = block_sum(re, sh);
  im = block_sum(im, sh);
  if (threadIdx.x == 0) out[j] = make_cuDoubleComplex(re, im);
}

// eg[j] = Re<p_j|h_j>; res[j] = || h_j - eg_j p_j ||^2 (two passes, no cancellation)
__global__ void k_rayleigh_residual(int m, const Z* __restrict__ p, long long ldp, const Z* __restrict__ h,
                                    long long ldh, double* __restrict__ eg, double* __restrict__ res) {
  __shared__ double sh[33];
  const int j = blockIdx.x;
  const Z* a = p + (size_t)j * ldp;
  const Z* b = h + (size_t)j * ldh;
  double re = 0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) re += a[i].x * b[i].x + a[i].y * b[i].y;
  const double e = block_sum(re, sh);
  double r = 0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const double dx = b[i].x - e * a[i].x, dy = b[i].y - e * a[i].y;
    r += dx * dx + dy * dy;
  }
  r = block_sum(r, sh);
  if (threadIdx.x == 0) {
    eg[j] = e;
    res[j] = r;
  }
}

// relaxation step (ditsp_c16_loop.f90:531-543 with diag_rq_jac_c16.f90:67-79):
// r = h - eg p; x = hdiag - eg; x = 1 if x < 1 else 1/x; p += -x r
__global__ void k_jacobi(int m, Z* __restrict__ p, long long ldp, const Z* __restrict__ h, long long ldh,
                         const double* __restrict__ eg, const double* __restrict__ hdiag) {
  const int j = blockIdx.y;
  const double e = eg[j];
  Z* a = p + (size_t)j * ldp;
  const Z* b = h + (size_t)j * ldh;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    double x = hdiag[i] - e;
    x = x < 1.0 ? 1.0 : 1.0 / x;
    const Z u = a[i], v = b[i];
    a[i] = make_cuDoubleComplex(u.x - x * (v.x - e * u.x), u.y - x * (v.y - e * u.y));
  }
}

// x_j *= s_j (real)
__global__ void k_colscale(int m, Z* __restrict__ x, long long ldx, const double* __restrict__ s) {
  const int j = blockIdx.y;
  const double f = s[j];
  Z* a = x + (size_t)j * ldx;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    a[i] = make_cuDoubleComplex(a[i].x * f, a[i].y * f);
}

// ---------------- device-side modified Gram-Schmidt (<= 10 vectors) ----------------
// One cooperative launch per block of vectors, restating grsch_mod_c16.f90:77-147
// with every decision taken on the device: sequential MGS projections, the
// repeat when xnp > 0.9999 xni, the drop below 1e-20 of the natural scale.
// Each CTA owns a slice of rows; reductions write per-CTA partial sums to a
// double-buffered array, pass a grid barrier, and every CTA reads the partials
// in parallel (one per thread) and adds them with the same fixed-order tree
// (deterministic, identical in all CTAs).
struct MgsArgs {
  int m, nvec, also;
  Z* x;
  Z* hx;
  const double* xscl;
  int* irow;
  double* partial;      // 2 * gridDim.x * 4 doubles
  unsigned* bar;        // [0] arrival count, [1] generation
  int* err;             // set to 1 when a barrier wait gives up
  double eps, peq, rep; // 1e-20 (as compiled), tiny/eps, 0.9999
  long long spin_limit; // polls of a grid-barrier wait before it gives up (2^24: ~1 s at ~64 ns per try)
};

// Grid barrier with a bounded wait: returns false (and sets *err) if the
// other CTAs did not arrive in time; all CTAs then leave the kernel.
__device__ bool grid_barrier(unsigned* bar, int* err, long long spin_limit) {
  __syncthreads();
  __shared__ int ok;
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = bar + 1;
    const unsigned g = *vgen;
    __threadfence();
    ok = 1;
    if (atomicAdd(&bar[0], 1u) == gridDim.x - 1) {
      atomicExch(&bar[0], 0u);
      __threadfence();
      atomicAdd(&bar[1], 1u);
    } else {
      long long it = 0;
      while (*vgen == g) {
        if (++it > spin_limit) {
          atomicExch(err, 1);
          ok = 0;
          break;
        }
        __nanosleep(40);
      }
    }
    __threadfence();
    if (*((volatile int*)err) != 0) ok = 0;
  }
  __syncthreads();
  return ok != 0;
}

// sums k (<= 4) per-thread values over the grid; result in out[0..k) for every thread
__device__ bool grid_sum(const MgsArgs& a, int& round, const double* v, int k, double* out, double* sh) {
  double* buf = a.partial + (size_t)(round & 1) * gridDim.x * 4;
  for (int t = 0; t < k; ++t) {
    const double s = block_sum(v[t], sh);
    if (threadIdx.x == 0) buf[(size_t)blockIdx.x * 4 + t] = s;
  }
  ++round;
  if (!grid_barrier(a.bar, a.err, a.spin_limit)) return false;
  for (int t = 0; t < k; ++t) {
    double s = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) s += ((volatile double*)buf)[(size_t)b * 4 + t];
    out[t] = block_sum(s, sh);
  }
  return true;
}

__global__ void __launch_bounds__(256) k_mgs(MgsArgs a) {
  __shared__ double sh[33];
  const int per = (a.m + gridDim.x - 1) / gridDim.x;
  const int r0 = blockIdx.x * per, r1 = min(a.m, r0 + per);
  int round = 0;
  double v[4], o[4];
  auto dot = [&](const Z* p, const Z* q, double& re, double& im) {
    re = 0;
    im = 0;
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      const Z u = p[r], w = q[r];
      re += u.x * w.x + u.y * w.y;
      im += u.x * w.y - u.y * w.x;
    }
  };
  auto axpy = [&](const Z* p, Z* q, double cr, double ci) {   // q -= c p
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      const Z u = p[r];
      q[r] = make_cuDoubleComplex(q[r].x - (cr * u.x - ci * u.y), q[r].y - (cr * u.y + ci * u.x));
    }
  };
  for (int i = 0; i < a.nvec; ++i) {
    Z* xi = a.x + (size_t)i * a.m;
    Z* hxi = a.also ? a.hx + (size_t)i * a.m : nullptr;
    if (i > 0) {
      double xni = 0, xnp = 0;
      for (int j = 0; j < i; ++j) {
        const Z* xj = a.x + (size_t)j * a.m;
        dot(xj, xi, v[0], v[1]);
        int k = 2;
        if (j == 0) {   // xni on the vector before any projection
          double re, im;
          dot(xi, xi, re, im);
          v[2] = re;
          k = 3;
        }
        if (!grid_sum(a, round, v, k, o, sh)) return;
        if (j == 0) xni = o[2];
        xnp += o[0] * o[0] + o[1] * o[1];
        axpy(xj, xi, o[0], o[1]);
        if (hxi) axpy(a.hx + (size_t)j * a.m, hxi, o[0], o[1]);
      }
      if (xnp > a.rep * xni) {
        for (int j = 0; j < i; ++j) {
          const Z* xj = a.x + (size_t)j * a.m;
          dot(xj, xi, v[0], v[1]);
          if (!grid_sum(a, round, v, 2, o, sh)) return;
          axpy(xj, xi, o[0], o[1]);
          if (hxi) axpy(a.hx + (size_t)j * a.m, hxi, o[0], o[1]);
        }
      }
    }
    double re, im;
    dot(xi, xi, re, im);
    v[0] = re;
    if (!grid_sum(a, round, v, 1, o, sh)) return;
    double suma = o[0];
    const double xs = a.xscl[i];
    int keep = 1;
    if (xs > a.peq) {
      if (suma < a.eps * xs) {
        suma = 0.0;
        keep = 0;
      } else {
        suma = 1.0 / sqrt(suma);
      }
    } else {
      suma = 0.0;
      keep = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && !keep) a.irow[i] = 0;
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      xi[r] = make_cuDoubleComplex(xi[r].x * suma, xi[r].y * suma);
      if (hxi) hxi[r] = make_cuDoubleComplex(hxi[r].x * suma, hxi[r].y * suma);
    }
  }
}

// G (k x k, lower triangle used) of a block whose columns idx[0..nd) were zeroed: their rows and
// columns become those of the identity, so the factorisation goes through and leaves them zero
__global__ void k_patch_gram(Z* G, int k, const int* idx, int nd) {
  const long long n = (long long)nd * k;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int d = idx[t / k], j = (int)(t % k);
    const Z v = make_cuDoubleComplex(j == d ? 1.0 : 0.0, 0.0);
    G[(size_t)j * k + d] = v;     // row d
    G[(size_t)d * k + j] = v;     // column d
  }
}

// out[i] = Re G(i, i): the diagonal of a k x k matrix in one contiguous block (a strided
// device-to-host copy of 16-byte pieces costs one transfer per element)
__global__ void k_diag_re(const Z* __restrict__ G, int k, double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) out[i] = G[(size_t)i * k + i].x;
}

// out = A^H for a k x k column-major matrix
__global__ void k_conj_transpose(const Z* __restrict__ A, int k, Z* __restrict__ out) {
  const long long n = (long long)k * k;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t % k), c = (int)(t / k);
    const Z v = A[(size_t)r * k + c];
    out[t] = make_cuDoubleComplex(v.x, -v.y);
  }
}

// zero the strictly upper triangle of a k x k column-major matrix
__global__ void k_zero_upper(Z* G, int k) {
  const long long n = (long long)k * k;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t % k), c = (int)(t / k);
    if (r < c) G[t] = make_cuDoubleComplex(0.0, 0.0);
  }
}

__global__ void k_diag_add(Z* G, int k, double shift) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x)
    G[(size_t)i * k + i].x += shift;
}

// --------------------------- solver state ---------------------------
struct Solver {
  cpw_b200_ctx* c;
  cudaStream_t st;
  cublasHandle_t blas;
  cusolverDnHandle_t sol = nullptr;
  int m;            // mtxd
  int mxdsml, mxdbnd;
  // The first zcols columns of bas are the small-matrix eigenvectors zero-padded below row zrows = mtxds
  // (ditsp_c16_start.f90:205-212) and never change: products with them run over zrows rows only.
  int zcols = 0, zrows = 0;
  long long ldp;    // leading dim of psi/hpsi (device)
  Z* P;             // psi   (ldp x mxdbnd)
  Z* HP;            // hpsi
  DevBuf bas, hbas, smallA, smallV, dvec, dvec2, dz, work, info, eg_d, hdiag_d;
  int lwork = 0;
  long long ihk = 0;
  int status = kOk;
  // wall-clock accounting per phase (printed when ipr > 1): 0 H|psi>, 1 Gram-Schmidt, 2 subspace eigensolve;
  // inside 1: 3 modified Gram-Schmidt leaves, 4 block passes against the converged vectors
  // outside 0-2: 5 residual norms of the inner loop, 6 span test, 7 relaxation (without H|psi>),
  // 8 Ritz subspace Hamiltonian, 9 Ritz rotations, copies and residual check
  // inside 3 (Cholesky QR): 10 Gram products, 11 factorisations with their host reads, 12 triangular solves
  double tphase[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  long long n_gs = 0, n_gs_vec = 0, n_leaf = 0;
  bool timing = false;
  struct Tick {
    Solver* s;
    int k;
    std::chrono::steady_clock::time_point t0;
    Tick(Solver* sv, int kk) : s(sv), k(kk) {
      if (s->timing) {
        cudaStreamSynchronize(s->st);
        t0 = std::chrono::steady_clock::now();
      }
    }
    void stop() {
      if (s->timing && k >= 0) {
        cudaStreamSynchronize(s->st);
        s->tphase[k] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      }
      k = -1;
    }
    ~Tick() { stop(); }
  };
  const Z one = make_cuDoubleComplex(1, 0), zero = make_cuDoubleComplex(0, 0), mone = make_cuDoubleComplex(-1, 0);

  Z* B(int j) { return (Z*)bas.p + (size_t)j * m; }
  Z* HB(int j) { return (Z*)hbas.p + (size_t)j * m; }
  Z* Pc(int j) { return P + (size_t)j * ldp; }
  Z* HPc(int j) { return HP + (size_t)j * ldp; }

  int ck(cudaError_t e, const char* w) { return e == cudaSuccess ? kOk : cuda_fail(e, w); }
  int ckb(cublasStatus_t s, const char* w) {
    return s == CUBLAS_STATUS_SUCCESS ? kOk : fail(kCublas, std::string(w) + ": cuBLAS status " + std::to_string((int)s));
  }

  int hk(Z* x, long long ldx, Z* hx, long long ldhx, int n) {
    if (n <= 0) return kOk;
    Tick tk(this, 0);
    ihk += n;
    return ctx_hkpsi_device(c, n, x, ldx, hx, ldhx, st, true, true);
  }

  // Basis-wide products of the mixed forms on the int8 tensor cores (FP64-accurate Ozaki GEMM,
  // oz.cu) instead of cuBLAS FP64; products below kI8MinFlops stay in cuBLAS (the splitting
  // launches cost more than they save there)
  bool basis_i8 = false;
  int oz_slices = 7;
  // which classes of basis-wide products take the int8 path when basis_i8 (CPW_B200_I8_PRODUCTS):
  // the class of a product is read from the prefix of its name
  enum : unsigned { kI8Chol = 1, kI8Mm = 2, kI8Conv = 4, kI8Span = 8, kI8Ham = 16, kI8Rot = 32, kI8Other = 64 };
  // default: the Cholesky QR, the Ritz subspace Hamiltonian and the Ritz rotations (large square or
  // tall products); the Gram-Schmidt passes against the converged block (many smaller products,
  // each paying the operand splits) measured faster in cuBLAS FP64
  unsigned i8_mask = kI8Chol | kI8Ham | kI8Rot;
  static unsigned i8_class(const char* w) {
    if (!strncmp(w, "cholqr", 6)) return kI8Chol;
    if (!strncmp(w, "grsch_mm", 8)) return kI8Mm;
    if (!strncmp(w, "grsch_loop", 10)) return kI8Conv;
    if (!strncmp(w, "span", 4)) return kI8Span;
    if (!strncmp(w, "ritz hamsm", 10)) return kI8Ham;
    if (!strncmp(w, "ritz", 4)) return kI8Rot;
    return kI8Other;
  }

  long long n_i8 = 0, n_cublas = 0;
  double kI8MinFlops = 2e9;    // CPW_B200_I8_MIN_GFLOP

  // C(m x n) = alpha * op(A) * op(B) + beta * C
  int gemm(cublasOperation_t ta, cublasOperation_t tb, int mm, int nn, int kk, Z alpha, const Z* A, long long lda,
           const Z* Bm, long long ldb, Z beta, Z* Cm, long long ldc, const char* w) {
    if (mm <= 0 || nn <= 0) return kOk;
    if (basis_i8 && (i8_mask & i8_class(w)) && kk > 0 && tb == CUBLAS_OP_N && (ta == CUBLAS_OP_N || ta == CUBLAS_OP_C) && alpha.y == 0 &&
        (alpha.x == 1.0 || alpha.x == -1.0) && beta.y == 0 && (beta.x == 0.0 || beta.x == 1.0) &&
        8.0 * mm * nn * kk >= kI8MinFlops) {
      ++n_i8;
      return oz_zgemm(c->ozs, ta == CUBLAS_OP_C, mm, nn, kk, A, lda, Bm, ldb, alpha.x, beta.x != 0.0, Cm, ldc,
                      oz_slices, c->tcs.wait_ns, st);
    }
    ++n_cublas;
    if (kk <= 0) {
      // C = beta C
      if (beta.x == 0 && beta.y == 0) {
        for (int j = 0; j < nn; ++j)
          if (int s = ck(cudaMemsetAsync(Cm + (size_t)j * ldc, 0, sizeof(Z) * mm, st), w)) return s;
      }
      return kOk;
    }
    return ckb(cublasZgemm(blas, ta, tb, mm, nn, kk, &alpha, A, (int)lda, Bm, (int)ldb, &beta, Cm, (int)ldc), w);
  }

  // a product of the Cholesky QR: on the int8 tensor cores with its triangular structure (OzTri),
  // else as gemm() routes it
  bool oz_tri = true;
  int chol_gemm(cublasOperation_t ta, int mm, int nn, int kk, const Z* A, long long lda, const Z* Bm, long long ldb,
                Z* Cm, long long ldc, int tri, const char* w) {
    if (basis_i8 && (i8_mask & kI8Chol) && 8.0 * mm * nn * kk >= kI8MinFlops) {
      ++n_i8;
      return oz_zgemm(c->ozs, ta == CUBLAS_OP_C, mm, nn, kk, A, lda, Bm, ldb, 1.0, false, Cm, ldc, oz_slices,
                      c->tcs.wait_ns, st, oz_tri ? tri : kOzFull);
    }
    return gemm(ta, CUBLAS_OP_N, mm, nn, kk, one, A, lda, Bm, ldb, zero, Cm, ldc, w);
  }

  // host copies of per-column dots  out[j] = <x_j|y_j>
  int coldots(const Z* x, long long ldx, const Z* y, long long ldy, int n, std::vector<zc>& out) {
    out.assign(n, zc(0, 0));
    if (n <= 0) return kOk;
    if (int s = dz.ensure(sizeof(Z) * n)) return s;
    k_coldot<<<n, kColThreads, 0, st>>>(m, x, ldx, y, ldy, (Z*)dz.p);
    if (int s = ck(cudaMemcpyAsync(out.data(), dz.p, sizeof(Z) * n, cudaMemcpyDeviceToHost, st), "coldots")) return s;
    return ck(cudaStreamSynchronize(st), "coldots");
  }

  int colscale(Z* x, long long ldx, int n, const std::vector<double>& s) {
    if (n <= 0) return kOk;
    if (int r = dvec2.ensure(sizeof(double) * n)) return r;
    if (int r = ck(cudaMemcpyAsync(dvec2.p, s.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st), "colscale"))
      return r;
    dim3 g((unsigned)std::min(64, (m + 255) / 256), n);
    k_colscale<<<g, 256, 0, st>>>(m, x, ldx, (const double*)dvec2.p);
    // the host vector may go out of scope: wait for the copy
    return ck(cudaStreamSynchronize(st), "colscale");
  }

  int copycols(Z* dst, long long ldd, const Z* src, long long lds, int n) {
    if (n <= 0) return kOk;
    return ck(cudaMemcpy2DAsync(dst, ldd * sizeof(Z), src, lds * sizeof(Z), m * sizeof(Z), n,
                                cudaMemcpyDeviceToDevice, st),
              "copycols");
  }

  // Hermitian eigen-decomposition of the n x n device matrix A (ld n) with
  // zheevd('V','L'): eigenvalues to host w, eigenvectors overwrite A. With 0 < nlow < n only the
  // nlow lowest pairs are computed (zheevdx, range 'I'): w gets nlow values, A their vectors in
  // its leading nlow columns.
  int diag(Z* A, int n, std::vector<double>& w, int nlow = 0) {
    w.assign(n, 0.0);
    if (n <= 0) return kOk;
    Tick tk(this, 2);
    if (!sol) {
      if (cusolverDnCreate(&sol) != CUSOLVER_STATUS_SUCCESS) return fail(kCusolver, "cusolverDnCreate failed");
    }
    cusolverDnSetStream(sol, st);
    if (nlow > 0 && nlow < n) {
      int lw = 0, meig = 0;
      if (cusolverDnZheevdx_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUSOLVER_EIG_RANGE_I, CUBLAS_FILL_MODE_LOWER, n,
                                       A, n, 0.0, 0.0, 1, nlow, &meig, (double*)eg_d.p,
                                       &lw) != CUSOLVER_STATUS_SUCCESS)
        return fail(kCusolver, "zheevdx buffer size");
      if (int s = work.ensure(sizeof(Z) * (size_t)std::max(lw, 1))) return s;
      if (int s = info.ensure(sizeof(int))) return s;
      if (cusolverDnZheevdx(sol, CUSOLVER_EIG_MODE_VECTOR, CUSOLVER_EIG_RANGE_I, CUBLAS_FILL_MODE_LOWER, n, A, n, 0.0,
                            0.0, 1, nlow, &meig, (double*)eg_d.p, (Z*)work.p, lw,
                            (int*)info.p) != CUSOLVER_STATUS_SUCCESS)
        return fail(kCusolver, "zheevdx");
      int inf = 0;
      w.resize(nlow);
      if (int s = ck(cudaMemcpyAsync(&inf, info.p, sizeof(int), cudaMemcpyDeviceToHost, st), "zheevdx info")) return s;
      if (int s = ck(cudaMemcpyAsync(w.data(), eg_d.p, sizeof(double) * nlow, cudaMemcpyDeviceToHost, st),
                     "zheevdx w"))
        return s;
      if (int s = ck(cudaStreamSynchronize(st), "zheevdx")) return s;
      if (inf != 0 || meig != nlow) return fail(kCusolver, "diag_c16 (partial) failed, info = " + std::to_string(inf));
      return kOk;
    }
    int lw = 0;
    if (cusolverDnZheevd_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, A, n,
                                    (double*)eg_d.p, &lw) != CUSOLVER_STATUS_SUCCESS)
      return fail(kCusolver, "zheevd buffer size");
    if (int s = work.ensure(sizeof(Z) * (size_t)std::max(lw, 1))) return s;
    if (int s = info.ensure(sizeof(int))) return s;
    if (cusolverDnZheevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, A, n, (double*)eg_d.p,
                         (Z*)work.p, lw, (int*)info.p) != CUSOLVER_STATUS_SUCCESS)
      return fail(kCusolver, "zheevd");
    int inf = 0;
    if (int s = ck(cudaMemcpyAsync(&inf, info.p, sizeof(int), cudaMemcpyDeviceToHost, st), "zheevd info")) return s;
    if (int s = ck(cudaMemcpyAsync(w.data(), eg_d.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st), "zheevd w"))
      return s;
    if (int s = ck(cudaStreamSynchronize(st), "zheevd")) return s;
    if (inf != 0) return fail(kCusolver, "diag_c16 failed, info = " + std::to_string(inf));
    return kOk;
  }

  // ---- Cholesky QR, twice: the in-block orthonormalisation of the mixed form ----
  // X <- X (L^H)^-1 with X^H X = L L^H, two passes. Before the first pass changes X, a
  // failed factorisation, a pivot L_ii^2 below 1e-20 xscl_i (a vector the reference's drop
  // rule removes, grsch_mod_c16.f90) or below kCholCond G_ii (the block itself nearly
  // dependent, beyond what Cholesky QR resolves) sets *fallback and leaves X to the
  // reference's recursive Gram-Schmidt.
  // Ritz subspace Hamiltonian reuse: the leading ham_clean columns of bas/hbas are unchanged
  // since the last hbas^H bas, whose lower triangle (order ham_prev_n) is kept in ham_prev
  int ham_clean = 0, ham_prev_n = 0;
  long long ham_reused = 0, ham_full = 0;
  DevBuf ham_prev;
  void touch(int c0) { ham_clean = std::max(0, std::min(ham_clean, c0)); }
  bool chol = false;
  bool ham_full_gemm = false;  // Ritz subspace Hamiltonian block as a full product instead of zherkx
  bool partial_eig = false;    // Ritz step: only the eigenpairs its decisions and rotations read
  long long n_eig_full_again = 0;
  bool tc_rot = false;   // Ritz rotations on the tensor cores (mixed form with tensor-core projectors)
  long long n_chol = 0, n_chol_fallback = 0, n_fb_info = 0, n_fb_drop = 0, n_fb_cond = 0;
  DevBuf chol_g, chol_work, chol_info, chol_idx, chol_diag, chol_tmp, chol_tri, chol_lh;
  bool chol_gram_gemm = true, chol_apply_gemm = true;
  // L (lower, k x k in G) -> L^-1 in place, strictly upper part zeroed
  int chol_inverse(Z* G, int k) {
    size_t dbytes = 0, hbytes = 0;
    if (cusolverDnXtrtri_bufferSize(sol, CUBLAS_FILL_MODE_LOWER, CUBLAS_DIAG_NON_UNIT, k, CUDA_C_64F, G, k, &dbytes,
                                    &hbytes) != CUSOLVER_STATUS_SUCCESS)
      return fail(kCusolver, "trtri workspace");
    std::vector<unsigned char> hwork(std::max<size_t>(hbytes, 1));
    if (int s = chol_tri.ensure(std::max<size_t>(dbytes, 16))) return s;
    if (cusolverDnXtrtri(sol, CUBLAS_FILL_MODE_LOWER, CUBLAS_DIAG_NON_UNIT, k, CUDA_C_64F, G, k, chol_tri.p, dbytes,
                         hwork.data(), hbytes, (int*)chol_info.p) != CUSOLVER_STATUS_SUCCESS)
      return fail(kCusolver, "trtri");
    k_zero_upper<<<std::max(1, std::min(1184, (int)(((long long)k * k + 255) / 256))), 256, 0, st>>>(G, k);
    int inf = 0;
    if (int s = ck(cudaMemcpyAsync(&inf, chol_info.p, sizeof(int), cudaMemcpyDeviceToHost, st), "trtri info")) return s;
    if (int s = ck(cudaStreamSynchronize(st), "trtri")) return s;
    if (inf != 0) return fail(kCusolver, "cholqr: trtri failed, info = " + std::to_string(inf));
    return kOk;
  }
  // x (m x k) <- x Li^H for the lower-triangular Li stored full (k x k)
  int apply_right_lh(Z* x, int k, const Z* Li) {
    if (int s = chol_tmp.ensure(sizeof(Z) * (size_t)m * k)) return s;
    Z* t = (Z*)chol_tmp.p;
    if (basis_i8 && (i8_mask & kI8Chol)) {
      // the int8 GEMM takes B as stored: form Li^H
      if (int s = chol_lh.ensure(sizeof(Z) * (size_t)k * k)) return s;
      k_conj_transpose<<<std::max(1, std::min(1184, (int)(((long long)k * k + 255) / 256))), 256, 0, st>>>(
          Li, k, (Z*)chol_lh.p);
      if (int s = chol_gemm(CUBLAS_OP_N, m, k, k, x, m, (const Z*)chol_lh.p, k, t, m, kOzUpperB, "cholqr apply"))
        return s;
    } else if (int s = gemm(CUBLAS_OP_N, CUBLAS_OP_C, m, k, k, one, x, m, Li, k, zero, t, m, "cholqr apply")) {
      return s;
    }
    return ck(cudaMemcpyAsync(x, t, sizeof(Z) * (size_t)m * k, cudaMemcpyDeviceToDevice, st), "cholqr apply");
  }
  // the real diagonal of G (k x k) into host h (k doubles)
  int diag_to_host(const Z* G, int k, double* h) {
    if (int s = chol_diag.ensure(sizeof(double) * (size_t)k)) return s;
    k_diag_re<<<std::max(1, std::min(64, (k + 255) / 256)), 256, 0, st>>>(G, k, (double*)chol_diag.p);
    return ck(cudaMemcpyAsync(h, chol_diag.p, sizeof(double) * (size_t)k, cudaMemcpyDeviceToHost, st), "cholqr diag");
  }
  long long n_chol_dropped = 0, n_chol_shifted = 0;
  static constexpr double kCholCond = 1e-12;
  int cholqr(bool also, Z* x, Z* hx, int k, int* irow, const double* xscl, bool* fallback) {
    *fallback = false;
    if (k <= 0) return kOk;
    Tick tk(this, 3);
    ++n_chol;
    if (!sol) {
      if (cusolverDnCreate(&sol) != CUSOLVER_STATUS_SUCCESS) return fail(kCusolver, "cusolverDnCreate failed");
      cusolverDnSetStream(sol, st);
    }
    int s;
    if ((s = chol_g.ensure(sizeof(Z) * (size_t)k * k)) || (s = chol_info.ensure(sizeof(int))) ||
        (s = chol_idx.ensure(sizeof(int) * (size_t)k)))
      return s;
    Z* G = (Z*)chol_g.p;
    int lw = 0;
    if (cusolverDnZpotrf_bufferSize(sol, CUBLAS_FILL_MODE_LOWER, k, G, k, &lw) != CUSOLVER_STATUS_SUCCESS)
      return fail(kCusolver, "zpotrf workspace");
    if ((s = chol_work.ensure(sizeof(Z) * (size_t)std::max(lw, 1)))) return s;
    std::vector<double> dg(k), dg0(k);
    std::vector<int> dropped;
    // two plain passes; when the first plain factorisation fails (a nearly dependent block),
    // one shifted pass first (factor G + s I, s = 11 (m k + k (k + 1)) u trace(G), as in the
    // published shifted Cholesky QR 3) brings the block to a condition Cholesky QR resolves
    bool first = true, shift_now = false, shifted = false;
    int done = 0;
    while (done < 2) {
      {
        Tick tg(this, 10);
        if (chol_gram_gemm) {
          // X^H X as a full product: cuBLAS's zherk for a block of a few hundred vectors over
          // ~1e5 rows runs at a fraction of the ZGEMM rate (measured: 6 ms against ~1 ms)
          // (the factorisation reads the lower triangle only)
          if ((s = chol_gemm(CUBLAS_OP_C, k, k, m, x, m, x, m, G, k, kOzLowerOut, "cholqr gram"))) return s;
        } else {
          const double a1 = 1.0, b0 = 0.0;   // lower triangle of X^H X
          if (cublasZherk(blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_C, k, m, &a1, x, m, &b0, G, k) !=
              CUBLAS_STATUS_SUCCESS)
            return fail(kCublas, "cholqr gram");
        }
      }
      Tick tf(this, 11);
      // squared norms of the block's vectors (the Gram diagonal, before the factorisation)
      if ((s = diag_to_host(G, k, dg0.data()))) return s;
      if (first || shift_now) {
        if ((s = ck(cudaStreamSynchronize(st), "cholqr norms"))) return s;
      }
      if (first) {
        // the reference's drop rule (grsch_mod_c16.f90: norm^2 below 1e-20 of the norm^2 before
        // the passes against the converged vectors) removes vectors those passes reduced to
        // rounding noise: zero and flag them
        for (int i = 0; i < k; ++i)
          if (!(dg0[i] >= CEPS20 * xscl[i]) || !(xscl[i] > 0.0)) dropped.push_back(i);
        for (int i : dropped) {
          irow[i] = 0;
          if ((s = ck(cudaMemsetAsync(x + (size_t)i * m, 0, sizeof(Z) * m, st), "cholqr drop")) ||
              (also && (s = ck(cudaMemsetAsync(hx + (size_t)i * m, 0, sizeof(Z) * m, st), "cholqr drop"))))
            return s;
        }
        if (!dropped.empty()) {
          n_chol_dropped += (long long)dropped.size();
          if ((s = ck(cudaMemcpyAsync(chol_idx.p, dropped.data(), sizeof(int) * dropped.size(),
                                      cudaMemcpyHostToDevice, st),
                      "cholqr drop")))
            return s;
        }
      }
      if (!dropped.empty())
        k_patch_gram<<<std::max(1, std::min(1184, (int)((dropped.size() * k + 255) / 256))), 256, 0, st>>>(
            G, k, (const int*)chol_idx.p, (int)dropped.size());
      if (shift_now) {
        double tr = 0.0;
        for (int i = 0; i < k; ++i) tr += dg0[i];
        const double sh = 11.0 * ((double)m * k + (double)k * (k + 1)) * 1.1102230246251565e-16 * tr;
        k_diag_add<<<std::max(1, std::min(1184, (k + 255) / 256)), 256, 0, st>>>(G, k, sh);
      }
      if (cusolverDnZpotrf(sol, CUBLAS_FILL_MODE_LOWER, k, G, k, (Z*)chol_work.p, lw, (int*)chol_info.p) !=
          CUSOLVER_STATUS_SUCCESS)
        return fail(kCusolver, "zpotrf");
      int info = 0;
      if ((s = ck(cudaMemcpyAsync(&info, chol_info.p, sizeof(int), cudaMemcpyDeviceToHost, st), "cholqr info")) ||
          (s = diag_to_host(G, k, dg.data())) || (s = ck(cudaStreamSynchronize(st), "cholqr")))
        return s;
      first = false;
      bool bad = info != 0;
      int why = bad ? 1 : 0;        // 1 factorisation, 2 drop rule, 3 conditioning
      for (int i = 0; i < k && !bad && done == 0 && !shift_now; ++i) {
        if (irow[i] == 0) continue;
        const double piv = dg[i] * dg[i];
        if (!(piv > CEPS20 * xscl[i])) {
          bad = true;
          why = 2;
        } else if (!(piv > kCholCond * dg0[i])) {
          bad = true;
          why = 3;
        }
      }
      if (bad && done == 0 && !shifted && !shift_now) {
        // X is unchanged: factor again with the shift
        shift_now = true;
        shifted = true;
        ++n_chol_shifted;
        continue;
      }
      if (bad && done == 0) {
        if (why == 1) ++n_fb_info;
        if (why == 2) ++n_fb_drop;
        if (why == 3) ++n_fb_cond;
      }
      if (bad) {
        if (done == 0) {
          // the zeroed vectors stay dropped; the recursive Gram-Schmidt takes the block
          *fallback = true;
          ++n_chol_fallback;
          return kOk;
        }
        return fail(kCusolver, "cholqr: second Cholesky pass failed");
      }
      tf.stop();
      Tick tt(this, 12);
      if (chol_apply_gemm) {
        // X <- X L^-H as one ZGEMM with the explicit inverse (trtri, then the strictly upper part
        // zeroed): the triangular solve of a tall block runs far below the ZGEMM rate
        if ((s = chol_inverse(G, k))) return s;
        if ((s = apply_right_lh(x, k, G)) || (also && (s = apply_right_lh(hx, k, G)))) return s;
      } else {
        if (cublasZtrsm(blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_C, CUBLAS_DIAG_NON_UNIT, m, k,
                        &one, G, k, x, m) != CUBLAS_STATUS_SUCCESS)
          return fail(kCublas, "cholqr trsm");
        if (also && cublasZtrsm(blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_C, CUBLAS_DIAG_NON_UNIT, m,
                                k, &one, G, k, hx, m) != CUBLAS_STATUS_SUCCESS)
          return fail(kCublas, "cholqr trsm");
      }
      if (shift_now) {
        shift_now = false;      // the shifted pass conditions the block; two plain passes follow
        continue;
      }
      ++done;
    }
    return kOk;
  }

  // ---- block Gram-Schmidt family (grsch_mod / grsch_mm / grsch_loop / grsch_shift) ----
  // grsch_mod on the device (k_mgs); irow/xscl are host arrays of nvec entries
  DevBuf mgs_part, mgs_bar, mgs_irow, mgs_xscl;
  int mgs_grid = 0;
  int grsch_mod(bool also, Z* x, Z* hx, int nvec, int* irow, const double* xscl) {
    if (nvec <= 0) return kOk;
    Tick tk(this, 3);
    ++n_leaf;
    if (!mgs_grid) {
      int dev = 0, nsm = 0, per = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_mgs, 256, 0);
      mgs_grid = std::max(1, std::min(nsm * std::max(per, 1), nsm));
    }
    const int grid = std::max(1, std::min(mgs_grid, (m + 511) / 512));
    int s;
    if ((s = mgs_part.ensure(sizeof(double) * 8 * (size_t)mgs_grid)) || (s = mgs_bar.ensure(sizeof(unsigned) * 4)) ||
        (s = mgs_irow.ensure(sizeof(int) * 16)) || (s = mgs_xscl.ensure(sizeof(double) * 16)))
      return s;
    if ((s = ck(cudaMemsetAsync(mgs_bar.p, 0, sizeof(unsigned) * 4, st), "mgs"))) return s;
    if ((s = ck(cudaMemcpyAsync(mgs_irow.p, irow, sizeof(int) * nvec, cudaMemcpyHostToDevice, st), "mgs"))) return s;
    if ((s = ck(cudaMemcpyAsync(mgs_xscl.p, xscl, sizeof(double) * nvec, cudaMemcpyHostToDevice, st), "mgs")))
      return s;
    MgsArgs a;
    a.m = m;
    a.nvec = nvec;
    a.also = also ? 1 : 0;
    a.x = x;
    a.hx = hx;
    a.xscl = (const double*)mgs_xscl.p;
    a.irow = (int*)mgs_irow.p;
    a.partial = (double*)mgs_part.p;
    a.bar = (unsigned*)mgs_bar.p;
    a.err = (int*)mgs_bar.p + 2;
    a.eps = CEPS20;
    a.peq = (1.0 / CEPS20) * 2.2250738585072014e-308;
    a.rep = C0P9999;
    a.spin_limit = c->grid_polls;
    void* args[] = {&a};
    if ((s = ck(cudaLaunchCooperativeKernel((const void*)k_mgs, dim3(grid), dim3(256), args, 0, st), "mgs launch")))
      return s;
    int err = 0;
    if ((s = ck(cudaMemcpyAsync(irow, mgs_irow.p, sizeof(int) * nvec, cudaMemcpyDeviceToHost, st), "mgs"))) return s;
    if ((s = ck(cudaMemcpyAsync(&err, (int*)mgs_bar.p + 2, sizeof(int), cudaMemcpyDeviceToHost, st), "mgs"))) return s;
    if ((s = ck(cudaStreamSynchronize(st), "mgs"))) return s;
    if (err) return fail(kTimeout, "grsch_mod: a grid barrier wait gave up");
    return kOk;
  }

  int grsch_mm(bool also, Z* x, Z* hx, int nvec, int* irow, const double* xscl) {
    if (nvec <= 10) return grsch_mod(also, x, hx, nvec, irow, xscl);
    const int nn = nvec / 2, nn2 = nvec - nn;
    if (int s = grsch_mm(also, x, hx, nn, irow, xscl)) return s;
    std::vector<zc> xn;
    if (int s = coldots(x + (size_t)nn * m, m, x + (size_t)nn * m, m, nn2, xn)) return s;
    if (int s = smallA.ensure(sizeof(Z) * (size_t)nn * nn2)) return s;
    Z* t = (Z*)smallA.p;
    if (int s = gemm(CUBLAS_OP_C, CUBLAS_OP_N, nn, nn2, m, one, x, m, x + (size_t)nn * m, m, zero, t, nn, "grsch_mm t"))
      return s;
    if (int s = gemm(CUBLAS_OP_N, CUBLAS_OP_N, m, nn2, nn, mone, x, m, t, nn, one, x + (size_t)nn * m, m, "grsch_mm x"))
      return s;
    if (also)
      if (int s = gemm(CUBLAS_OP_N, CUBLAS_OP_N, m, nn2, nn, mone, hx, m, t, nn, one, hx + (size_t)nn * m, m,
                       "grsch_mm hx"))
        return s;
    std::vector<Z> th((size_t)nn * nn2);
    if (int s = ck(cudaMemcpyAsync(th.data(), t, sizeof(Z) * th.size(), cudaMemcpyDeviceToHost, st), "grsch_mm t"))
      return s;
    if (int s = ck(cudaStreamSynchronize(st), "grsch_mm")) return s;
    bool rep = false;
    for (int n = 0; n < nn2; ++n) {
      double xs = 0;
      for (int i = 0; i < nn; ++i) xs += th[(size_t)n * nn + i].x * th[(size_t)n * nn + i].x +
                                         th[(size_t)n * nn + i].y * th[(size_t)n * nn + i].y;
      if (xs > C0P9999 * xn[n].real()) rep = true;
    }
    if (rep) {
      if (int s = gemm(CUBLAS_OP_C, CUBLAS_OP_N, nn, nn2, m, one, x, m, x + (size_t)nn * m, m, zero, t, nn,
                       "grsch_mm t2"))
        return s;
      if (int s = gemm(CUBLAS_OP_N, CUBLAS_OP_N, m, nn2, nn, mone, x, m, t, nn, one, x + (size_t)nn * m, m,
                       "grsch_mm x2"))
        return s;
      if (also)
        if (int s = gemm(CUBLAS_OP_N, CUBLAS_OP_N, m, nn2, nn, mone, hx, m, t, nn, one, hx + (size_t)nn * m, m,
                         "grsch_mm hx2"))
          return s;
    }
    return grsch_mm(also, x + (size_t)nn * m, also ? hx + (size_t)nn * m : nullptr, nn2, irow + nn, xscl + nn);
  }

  // orthonormalise columns [nconv, nvec) of x (ld m) against [0, nconv) twice and among themselves;
  // structured: x is bas, whose leading zcols columns vanish below row zrows (hx, when updated, has no
  // such structure)
  int grsch_loop(bool also, Z* x, Z* hx, int nconv, int nvec, std::vector<int>& irow, bool structured = false) {
    Tick tk(this, 1);
    irow.assign(std::max(nvec, 0), 1);
    if (nvec <= nconv) return kOk;
    const int k = nvec - nconv;
    ++n_gs;
    n_gs_vec += k;
    std::vector<zc> d;
    if (int s = coldots(x + (size_t)nconv * m, m, x + (size_t)nconv * m, m, k, d)) return s;
    std::vector<double> xscl(k);
    for (int i = 0; i < k; ++i) xscl[i] = d[i].real();
    if (nconv > 0) {
      Tick tk4(this, 4);
      if (int s = smallA.ensure(sizeof(Z) * (size_t)nconv * k)) return s;
      Z* t = (Z*)smallA.p;
      // leading columns with zero rows below zrows: their products run over zrows rows
      const int c0 = structured ? std::min(zcols, nconv) : 0;
      Z* y = x + (size_t)nconv * m;
      const Z* xc = x + (size_t)c0 * m;
      // on the int8 tensor cores the converged block is split once for both passes: as A^H for
      // T = X^H Y, as A for Y -= X T (and H X for H Y -= H X T)
      const bool i8 = basis_i8 && (i8_mask & kI8Conv) && 8.0 * (nconv - c0) * k * m >= kI8MinFlops;
      // (the splits live in the context: freeing device memory per call would synchronise the device)
      OzOperand& x_cn = c->oz_gs[0];
      OzOperand& x_nn = c->oz_gs[1];
      OzOperand& hx_nn = c->oz_gs[2];
      if (i8) {
        ++n_i8;
        if (int s = oz_prepare_a(x_cn, true, nconv - c0, m, xc, m, oz_slices, st)) return s;
        if (int s = oz_prepare_a(x_nn, false, m, nconv - c0, xc, m, oz_slices, st)) return s;
        if (also)
          if (int s = oz_prepare_a(hx_nn, false, m, nconv, hx, m, oz_slices, st)) return s;
      }
      for (int pass = 0; pass < 2; ++pass) {
        if (c0 > 0)
          if (int s = gemm(CUBLAS_OP_C, CUBLAS_OP_N, c0, k, zrows, one, x, m, y, m, zero, t, nconv, "grsch_loop t0"))
            return s;
        if (i8) {
          if (int s = oz_gemm_prepared(c->ozs, x_cn, k, y, m, 1.0, false, t + c0, nconv, c->tcs.wait_ns, st))
            return s;
          if (int s = oz_gemm_prepared(c->ozs, x_nn, k, t + c0, nconv, -1.0, true, y, m, c->tcs.wait_ns, st))
            return s;
        } else {
          if (int s = gemm(CUBLAS_OP_C, CUBLAS_OP_N, nconv - c0, k, m, one, xc, m, y, m, zero, t + c0, nconv,
                           "grsch_loop t"))
            return s;
          if (int s = gemm(CUBLAS_OP_N, CUBLAS_OP_N, m, k, nconv - c0, mone, xc, m, t + c0, nconv, one, y, m,
                           "grsch_loop x"))
            return s;
        }
        if (c0 > 0)
          if (int s = gemm(CUBLAS_OP_N, CUBLAS_OP_N, zrows, k, c0, mone, x, m, t, nconv, one, y, m, "grsch_loop x0"))
            return s;
        if (also) {
          if (i8) {
            if (int s = oz_gemm_prepared(c->ozs, hx_nn, k, t, nconv, -1.0, true, hx + (size_t)nconv * m, m,
                                         c->tcs.wait_ns, st))
              return s;
          } else if (int s = gemm(CUBLAS_OP_N, CUBLAS_OP_N, m, k, nconv, mone, hx, m, t, nconv, one,
                                  hx + (size_t)nconv * m, m, "grsch_loop hx")) {
            return s;
          }
        }
      }
    }
    if (chol) {
      bool fb = false;
      if (int s = cholqr(also, x + (size_t)nconv * m, also ? hx + (size_t)nconv * m : nullptr, k, irow.data() + nconv,
                         xscl.data(), &fb))
        return s;
      if (!fb) return kOk;
    }
    return grsch_mm(also, x + (size_t)nconv * m, also ? hx + (size_t)nconv * m : nullptr, k, irow.data() + nconv,
                    xscl.data());
  }

  int grsch_shift(Z* x, long long ldx, int nconv, int nvec, const std::vector<int>& irow, int* ired) {
    int j = nconv;
    *ired = 0;
    for (int n = nconv; n < nvec; ++n) {
      if (irow[n] == 0) {
        ++*ired;
      } else {
        if (j < n)
          if (int s = copycols(x + (size_t)j * ldx, ldx, x + (size_t)n * ldx, ldx, 1)) return s;
        ++j;
      }
    }
    return kOk;
  }

  // psi/hpsi live with leading dimension ldp; the GS routines work on ld m, so
  // when ldp != m the block is staged through bas-sized scratch (dvec).
  int rayleigh(int lo, int hi, std::vector<double>& eg, std::vector<double>& res) {
    const int n = hi - lo;
    if (n <= 0) return kOk;
    if (int s = dvec.ensure(sizeof(double) * 2 * n)) return s;
    double* e = (double*)dvec.p;
    k_rayleigh_residual<<<n, kColThreads, 0, st>>>(m, Pc(lo), ldp, HPc(lo), ldp, e, e + n);
    std::vector<double> h(2 * n);
    if (int s = ck(cudaMemcpyAsync(h.data(), e, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, st), "rayleigh"))
      return s;
    if (int s = ck(cudaStreamSynchronize(st), "rayleigh")) return s;
    for (int i = 0; i < n; ++i) {
      eg[lo + i] = h[i];
      res[lo + i] = h[n + i];
    }
    return kOk;
  }

  double xmax_error(int neig) {
    std::vector<double> eg(neig), res(neig);
    if (rayleigh(0, neig, eg, res)) return -1.0;
    double x = 0;
    for (int i = 0; i < neig; ++i) x = std::max(x, res[i]);
    return x;
  }
};

// The solver's device buffers and cuSOLVER handle live in the context between calls: allocating
// and freeing them per call costs milliseconds and cudaFree synchronises the whole device, which
// would serialise contexts that solve different k-points at the same time.
struct SolverPool {
  Solver& S;
  static constexpr int kN = 24;
  DevBuf* m[kN];
  explicit SolverPool(Solver& s) : S(s) {
    DevBuf* l[kN] = {&S.bas,  &S.hbas,      &S.smallA,    &S.smallV,   &S.dvec,     &S.dvec2,    &S.dz,
                     &S.work, &S.info,      &S.eg_d,      &S.hdiag_d,  &S.ham_prev, &S.chol_g,   &S.chol_work,
                     &S.chol_info, &S.chol_idx, &S.mgs_part, &S.mgs_bar, &S.mgs_irow, &S.mgs_xscl, &S.chol_diag,
                     &S.chol_tmp, &S.chol_tri, &S.chol_lh};
    for (int i = 0; i < kN; ++i) {
      m[i] = l[i];
      swap(*m[i], S.c->ditsp_pool[i]);
    }
    S.sol = (cusolverDnHandle_t)S.c->ditsp_sol;
    if (S.sol) cusolverDnSetStream(S.sol, S.st);
  }
  ~SolverPool() {
    for (int i = 0; i < kN; ++i) swap(*m[i], S.c->ditsp_pool[i]);
    S.c->ditsp_sol = (void*)S.sol;
    S.sol = nullptr;
  }
  static void swap(DevBuf& a, DevBuf& b) {
    std::swap(a.p, b.p);
    std::swap(a.bytes, b.bytes);
  }
};

struct Trim {
  std::vector<double>* eg;
  int nconv, niter;
  double epsa;
  // the 'adjusts ntst for degeneracies' loop (ditsp_c16_loop.f90:263-290); the
  // trip count is fixed on entry, as a Fortran DO loop's
  int degeneracy(int ntst) const {
    const int trips = ntst - nconv + 1;
    for (int it = 0; it < trips; ++it) {
      double emax = (*eg)[nconv];
      for (int n = nconv; n < ntst; ++n) emax = std::max(emax, (*eg)[n]);
      double emin = emax + 10.0 * epsa;
      for (int n = ntst; n < niter; ++n) emin = std::min(emin, (*eg)[n]);
      if (emax + epsa > emin) {
        --ntst;
        if (ntst <= nconv) break;
      }
    }
    return ntst;
  }
};

}  // namespace

// The driver. psi/hpsi: device complex128 (ldp >= mtxd), mxdbnd columns.
// hamsm: host complex(8) (mxdsml, mxdsml) column-major (first mtxds used).
// hdiag: host real(mtxd). ei: host real(mxdbnd).
int ditsp_device(cpw_b200_ctx* c, int ipr, int* ifail, int icmax, int iguess, double epspsi, int* neig_io, int mtxds,
                 void* psi, long long ldp, void* hpsi, const double* hamsm, int mxdsml, const double* hdiag,
                 int mxdbnd, double* ei, long long* ihkpsum, cudaStream_t st, double* itlog, int itlog_rows) {
  if (!c->have_basis || !c->have_pot) return fail(kNotReady, "ditsp_c16: basis and potential must be set");
  const int mtxd = c->mtxd;
  int neig = *neig_io;
  *ifail = 0;
  *ihkpsum = 0;
  if (neig < 1) return kOk;
  if (neig > mtxds) return fail(kBadArg, "ditsp_c16: neig is greater than mtxds");
  if (neig > mxdbnd) return fail(kBadArg, "ditsp_c16: neig is greater than mxdbnd");
  if (3 * neig > mxdsml) return fail(kBadArg, "ditsp_c16: 3*neig is greater than mxdsml");
  if (mtxds > mxdsml) return fail(kBadArg, "ditsp_c16: mtxds is greater than mxdsml");
  if (ldp < mtxd) return fail(kBadArg, "ditsp_c16: leading dimension smaller than mtxd");

  Solver S;
  S.c = c;
  S.st = st;
  S.blas = c->blas;
  cublasSetStream(S.blas, st);
  S.m = mtxd;
  S.mxdsml = mxdsml;
  S.mxdbnd = mxdbnd;
  S.ldp = ldp;
  S.P = (Z*)psi;
  S.HP = (Z*)hpsi;
  S.timing = ipr > 1;
  SolverPool pool(S);
  // in-block orthonormalisation: the reference's recursive Gram-Schmidt for the FP64 drop-in,
  // Cholesky QR twice for the mixed form; CPW_B200_ORTHO=mgs|cholqr overrides
  S.chol = c->precision != 0;
  S.tc_rot = c->precision == 2 && !(getenv("CPW_B200_TC_ROT") && !strcmp(getenv("CPW_B200_TC_ROT"), "0"));
  // partial subspace eigensolve (zheevdx, lowest pairs only): measured no faster than zheevd on the
  // Si216 Ritz matrices (~1100), so off unless CPW_B200_EIG_PARTIAL=1
  S.partial_eig = getenv("CPW_B200_EIG_PARTIAL") && !strcmp(getenv("CPW_B200_EIG_PARTIAL"), "1");
  // basis-wide products: FP64 cuBLAS in the drop-in, the FP64-accurate int8 tensor-core GEMM in the
  // mixed forms; CPW_B200_BASIS_GEMM=fp64|i8 overrides, CPW_B200_OZ_SLICES sets its slices (1..8)
  S.basis_i8 = c->precision != 0;
  if (const char* v = getenv("CPW_B200_BASIS_GEMM")) {
    if (!strcmp(v, "fp64")) S.basis_i8 = false;
    if (!strcmp(v, "i8")) S.basis_i8 = true;
  }
  if (const char* v = getenv("CPW_B200_OZ_SLICES")) S.oz_slices = std::max(1, std::min(8, atoi(v)));
  if (const char* v = getenv("CPW_B200_I8_PRODUCTS")) {
    // comma list of chol, mm, conv, span, ham, rot, other, or all
    const std::string l = std::string(",") + v + ",";
    auto has = [&](const char* n) { return l.find(std::string(",") + n + ",") != std::string::npos; };
    if (has("all")) {
      S.i8_mask = ~0u;
    } else {
      S.i8_mask = (has("chol") ? Solver::kI8Chol : 0u) | (has("mm") ? Solver::kI8Mm : 0u) |
                  (has("conv") ? Solver::kI8Conv : 0u) | (has("span") ? Solver::kI8Span : 0u) |
                  (has("ham") ? Solver::kI8Ham : 0u) | (has("rot") ? Solver::kI8Rot : 0u) |
                  (has("other") ? Solver::kI8Other : 0u);
    }
  }
  S.ham_full_gemm = S.basis_i8 && (S.i8_mask & Solver::kI8Ham);
  if (const char* v = getenv("CPW_B200_HAM_BLOCK")) {
    if (!strcmp(v, "herkx")) S.ham_full_gemm = false;
    if (!strcmp(v, "gemm")) S.ham_full_gemm = true;
  }
  S.chol_gram_gemm = !(getenv("CPW_B200_CHOL_GRAM") && !strcmp(getenv("CPW_B200_CHOL_GRAM"), "herk"));
  S.chol_apply_gemm = !(getenv("CPW_B200_CHOL_APPLY") && !strcmp(getenv("CPW_B200_CHOL_APPLY"), "trsm"));
  S.oz_tri = !(getenv("CPW_B200_OZ_TRI") && !strcmp(getenv("CPW_B200_OZ_TRI"), "0"));
  if (const char* v = getenv("CPW_B200_I8_MIN_GFLOP")) S.kI8MinFlops = std::max(0.0, atof(v)) * 1e9;
  if (const char* o = getenv("CPW_B200_ORTHO")) {
    if (!strcmp(o, "mgs")) S.chol = false;
    if (!strcmp(o, "cholqr")) S.chol = true;
  }
  const auto t_start = std::chrono::steady_clock::now();
  int s;
  if ((s = S.eg_d.ensure(sizeof(double) * (size_t)std::max(mxdsml, 1)))) return s;

  // upload hamsm (leading mtxds block) once
  auto load_small = [&](DevBuf& buf, int n) -> int {
    int r = buf.ensure(sizeof(Z) * (size_t)n * n);
    if (r) return r;
    return S.ck(cudaMemcpy2DAsync(buf.p, sizeof(Z) * n, hamsm, sizeof(Z) * (size_t)mxdsml, sizeof(Z) * n, n,
                                  cudaMemcpyHostToDevice, st),
                "hamsm upload");
  };

  std::vector<double> eg(std::max(mtxd, mxdsml) + 2, 0.0), work(mxdsml + 2, 0.0);
  std::vector<double> et;

  if (mtxds >= mtxd) {
    // non-iterative diagonalisation (ditsp_c16.f90:218-232)
    if ((s = load_small(S.smallV, mtxds))) return s;
    if ((s = S.diag((Z*)S.smallV.p, mtxds, et))) return s;
    if ((s = S.copycols(S.P, ldp, (Z*)S.smallV.p, mtxds, neig))) return s;
    for (int i = 0; i < neig; ++i) ei[i] = et[i];
    return S.ck(cudaStreamSynchronize(st), "ditsp");
  }

  if ((s = S.bas.ensure(sizeof(Z) * (size_t)mtxd * mxdsml))) return s;
  if ((s = S.hbas.ensure(sizeof(Z) * (size_t)mtxd * mxdsml))) return s;
  if ((s = S.ck(cudaMemsetAsync(S.bas.p, 0, sizeof(Z) * (size_t)mtxd * mxdsml, st), "bas"))) return s;
  if ((s = S.hdiag_d.ensure(sizeof(double) * mtxd))) return s;
  if ((s = S.ck(cudaMemcpyAsync(S.hdiag_d.p, hdiag, sizeof(double) * mtxd, cudaMemcpyHostToDevice, st), "hdiag")))
    return s;

  // ---- start (ditsp_c16_start.f90) ----
  if ((s = load_small(S.smallV, mtxds))) return s;
  if ((s = S.diag((Z*)S.smallV.p, mtxds, et))) return s;
  double epsa = std::max(epspsi, fabs((et[neig - 1] - et[0]) / (double)(50 * neig)));
  int ndeg = neig;
  for (int i = neig; i < mtxds; ++i) {
    if (fabs(et[i] - et[i - 1]) > epsa) break;
    ndeg = i + 1;
  }
  ndeg = std::min(ndeg, mxdbnd);
  int niter = ndeg + 1;
  if (niter < mtxds) {
    for (int i = ndeg + 1; i < mtxds; ++i) {
      if (fabs(et[i] - et[i - 1]) > epsa) break;
      niter = i + 1;
    }
  } else {
    niter = mtxds;
  }
  niter = std::min(niter, mxdbnd);
  int nexact = neig;
  const double ecut = C1P2 * et[neig - 1] - C0P2 * et[0];
  for (int i = neig; i < mtxds; ++i) {
    if (et[i] > ecut) break;
    nexact = i + 1;
  }
  nexact = std::min(std::min(nexact, mxdsml / 3), std::min(neig + 2 + neig / 5, mtxds / 2)) + 3;
  {
    const int imax = nexact - 1;
    for (int i = 1; i <= imax; ++i) {
      --nexact;
      if (fabs(et[imax - i + 1] - et[imax - i]) > epsa) break;
    }
  }
  nexact = std::max(niter, nexact);
  if (nexact + niter + niter / 5 + 2 > mxdsml) return fail(kBadArg, "ditsp_c16_start: increase mxdsml");
  // bas(:, 1:nexact) = small eigenvectors zero-padded; hbas = H bas
  if ((s = S.ck(cudaMemcpy2DAsync(S.bas.p, sizeof(Z) * mtxd, S.smallV.p, sizeof(Z) * mtxds, sizeof(Z) * mtxds, nexact,
                                  cudaMemcpyDeviceToDevice, st),
                "start basis")))
    return s;
  if ((s = S.hk(S.B(0), mtxd, S.HB(0), mtxd, nexact))) return s;
  if (!(getenv("CPW_B200_ZERO_BLOCKS") && !strcmp(getenv("CPW_B200_ZERO_BLOCKS"), "0"))) {
    S.zcols = nexact;
    S.zrows = mtxds;
  }
  int nitold;
  bool lortho;
  if (iguess != 1) {
    if ((s = S.copycols(S.P, ldp, S.B(0), mtxd, niter))) return s;
    if ((s = S.copycols(S.HP, ldp, S.HB(0), mtxd, niter))) return s;
    lortho = true;
    nitold = 0;
  } else {
    if ((s = S.hk(S.P, ldp, S.HP, ldp, neig))) return s;
    if ((s = S.copycols(S.B(nexact), mtxd, S.P, ldp, neig))) return s;
    if ((s = S.copycols(S.HB(nexact), mtxd, S.HP, ldp, neig))) return s;
    lortho = false;
    nitold = neig;
    if (niter > neig) {
      if ((s = S.copycols(S.Pc(neig), ldp, S.B(neig), mtxd, niter - neig))) return s;
      if ((s = S.copycols(S.HPc(neig), ldp, S.HB(neig), mtxd, niter - neig))) return s;
    }
  }

  // P/HP are handled by the GS routines with leading dimension m: stage them
  // through a packed copy when ldp != m.
  DevBuf pk, hpk;
  const bool packed = ldp != mtxd;
  Z* PP = S.P;
  Z* HPP = S.HP;
  if (packed) {
    if ((s = pk.ensure(sizeof(Z) * (size_t)mtxd * mxdbnd)) || (s = hpk.ensure(sizeof(Z) * (size_t)mtxd * mxdbnd)))
      return s;
    if ((s = S.copycols((Z*)pk.p, mtxd, S.P, ldp, mxdbnd)) || (s = S.copycols((Z*)hpk.p, mtxd, S.HP, ldp, mxdbnd)))
      return s;
    PP = (Z*)pk.p;
    HPP = (Z*)hpk.p;
    S.P = PP;
    S.HP = HPP;
    S.ldp = mtxd;
  }

  int nconv = 0;
  bool lsafe = false, lconv = false;
  double xmax = 1.0;
  int mcref = 2;
  int iseed = -1;
  // ran2 state (Src/numeric/ran2.f90), re-initialised by the negative seed
  int ir[97];
  int iy = 0, iff = 0;
  auto ran2 = [&](int& idum) -> double {
    const int M = 714025, IA = 1366, IC = 150889;
    if (idum < 0 || iff == 0) {
      iff = 1;
      idum = (IC - idum) % M;
      for (int j = 0; j < 97; ++j) {
        idum = (int)(((long long)IA * idum + IC) % M);
        ir[j] = idum;
      }
      idum = (int)(((long long)IA * idum + IC) % M);
      iy = idum;
    }
    const int j = (int)((97LL * iy) / M);
    iy = ir[j];
    const double v = iy * 1.4005111865831e-6;
    idum = (int)(((long long)IA * idum + IC) % M);
    ir[j] = idum;
    return v;
  };

  auto compact_eg = [&](const std::vector<int>& irow, int lo, int hi) {
    int n = lo;
    for (int nac = lo; nac < hi; ++nac) {
      if (irow[nac] != 0) {
        if (n < nac) {
          eg[n] = eg[nac];
          work[n] = work[nac];
        }
        ++n;
      }
    }
  };
  auto first_unconverged = [&](int nmax, double tol) {
    int ntst = nconv;
    for (int n = nconv; n < nmax; ++n) {
      if (work[n] > tol) break;
      ntst = n + 1;
    }
    return ntst;
  };

  std::vector<int> irow;
  for (int ic = 1; ic <= icmax; ++ic) {
    const int mcmax = mcref;
    bool lexit = false;
    lconv = false;
    for (int mc = 1; mc <= mcmax; ++mc) {
      // ---- ditsp_c16_loop ----
      lconv = false;
      lexit = false;
      {
        Solver::Tick tk5(&S, 5);
        if ((s = S.rayleigh(nconv, niter, eg, work))) return s;
      }
      const double xmold = xmax;
      xmax = 0.0;
      for (int n = nconv; n < std::min(ndeg, niter); ++n) xmax = std::max(xmax, work[n]);
      if (ipr > 3)
        printf("  ditsp_c16_loop ic = %d  mc = %d  nconv = %d  niter = %d  xmax = %.6e\n", ic, mc, nconv, niter, xmax);
      if (mc > 1 && xmax > C0P2 * xmold) {
        mcref = mc;
        lexit = true;
      }
      if (!lexit && xmax < epspsi * epspsi && lsafe && niter >= ndeg) {
        if (lortho) {
          neig = ndeg;
          lconv = true;
        } else {
          if ((s = S.grsch_loop(true, PP, HPP, nconv, niter, irow))) return s;
          int ired;
          if ((s = S.grsch_shift(PP, mtxd, nconv, niter, irow, &ired))) return s;
          if ((s = S.grsch_shift(HPP, mtxd, nconv, niter, irow, &ired))) return s;
          if (ired > 0) lsafe = false;
          compact_eg(irow, nconv, niter);
          niter -= ired;
          lortho = true;
          if (nconv < niter) {
            xmax = 0.0;
            for (int n = nconv; n < std::min(niter, ndeg); ++n) xmax = std::max(xmax, work[n]);
            if (xmax < epspsi * epspsi && lsafe && niter >= ndeg) {
              neig = ndeg;
              lconv = true;
            }
          }
        }
      }
      if (!lconv && !lexit && niter == nconv) lexit = true;
      const double tol = C0P01 * epspsi * epspsi;
      int ntst = nconv;
      if (!lconv && !lexit) {
        ntst = first_unconverged(niter, tol);
        if (ntst > nconv) ntst = Trim{&eg, nconv, niter, epsa}.degeneracy(ntst);
      }
      if (!lconv && !lexit && ntst > nconv && !lortho) {
        if ((s = S.grsch_loop(true, PP, HPP, nconv, ntst, irow))) return s;
        irow.resize(std::max(niter, ntst), 1);
        for (int n = ntst; n < niter; ++n) irow[n] = 1;
        int ired;
        if ((s = S.grsch_shift(PP, mtxd, nconv, niter, irow, &ired))) return s;
        if ((s = S.grsch_shift(HPP, mtxd, nconv, niter, irow, &ired))) return s;
        if (ired > 0) lsafe = false;
        compact_eg(irow, nconv, niter);
        lortho = true;
        ntst -= ired;
        niter -= ired;
        if (ntst > nconv) {
          const int nmax = ntst;
          ntst = first_unconverged(nmax, tol);
          if (ntst > nconv) ntst = Trim{&eg, nconv, niter, epsa}.degeneracy(ntst);
        }
      }
      if (!lconv && !lexit && niter == nconv) lexit = true;
      if (!lconv && !lexit && ntst > nconv) {
        // span test against the previous basis vectors (ditsp_c16_loop.f90:396-461)
        Solver::Tick tk6(&S, 6);
        const int k = ntst - nconv;
        if ((s = S.smallA.ensure(sizeof(Z) * (size_t)k * k))) return s;
        if ((s = S.gemm(CUBLAS_OP_C, CUBLAS_OP_N, k, k, mtxd, S.one, S.B(nexact + nconv), mtxd, PP + (size_t)nconv * mtxd,
                        mtxd, S.zero, (Z*)S.smallA.p, k, "span test")))
          return s;
        std::vector<Z> vs((size_t)k * k);
        if ((s = S.ck(cudaMemcpyAsync(vs.data(), S.smallA.p, sizeof(Z) * vs.size(), cudaMemcpyDeviceToHost, st), "span")))
          return s;
        if ((s = S.ck(cudaStreamSynchronize(st), "span"))) return s;
        bool done = false;
        for (int it = 0; it < 10 * mxdbnd && !done; ++it) {
          const int nmax = ntst;
          ntst = nconv;
          bool lxn = false;
          for (int n = 0; n < nmax - nconv; ++n) {
            double xn = 0;
            for (int i = 0; i < nmax - nconv; ++i)
              xn += vs[(size_t)n * k + i].x * vs[(size_t)n * k + i].x + vs[(size_t)n * k + i].y * vs[(size_t)n * k + i].y;
            if (xn < C0P95) {
              lxn = true;
              break;
            }
            ntst = nconv + n + 1;
          }
          if (lxn) {
            if (ntst <= nconv) done = true;
          } else {
            double emax = eg[nconv];
            for (int n = nconv; n < ntst; ++n) emax = std::max(emax, eg[n]);
            double emin = emax + 10.0 * epsa;
            for (int n = ntst; n < niter; ++n) emin = std::min(emin, eg[n]);
            if (emax + epsa > emin) {
              --ntst;
              if (ntst <= nconv) done = true;
            } else {
              done = true;
            }
          }
          if (!done && it == 10 * mxdbnd - 1) return fail(kBadArg, "ditsp_c16_loop: span test did not terminate");
        }
      }
      if (!lconv && !lexit) {
        if (ntst > nconv) {
          S.touch(nexact + nconv);
          if ((s = S.copycols(S.B(nexact + nconv), mtxd, PP + (size_t)nconv * mtxd, mtxd, ntst - nconv))) return s;
          std::vector<int> irowb;
          if ((s = S.grsch_loop(false, (Z*)S.bas.p, (Z*)S.hbas.p, nexact + nconv, nexact + ntst, irowb, true)))
            return s;
          int ired;
          if ((s = S.grsch_shift((Z*)S.bas.p, mtxd, nexact + nconv, nexact + ntst, irowb, &ired))) return s;
          if (ired > 0) {
            lsafe = false;
            std::vector<int> ir2(niter, 1);
            for (int n = nconv; n < ntst; ++n) ir2[n] = irowb[nexact + n];
            int r2;
            if ((s = S.grsch_shift(PP, mtxd, nconv, niter, ir2, &r2))) return s;
            if ((s = S.grsch_shift(HPP, mtxd, nconv, niter, ir2, &r2))) return s;
            compact_eg(ir2, nconv, niter);
          }
          const int nnew = ntst - ired - nconv;
          S.touch(nexact + nconv);
          if ((s = S.hk(S.B(nexact + nconv), mtxd, S.HB(nexact + nconv), mtxd, nnew))) return s;
          nconv = ntst - ired;
          niter -= ired;
        }
        // relaxation step
        const int nr = niter - nconv;
        if (nr > 0) {
          Solver::Tick tk7(&S, 7);
          if ((s = S.dvec2.ensure(sizeof(double) * nr))) return s;
          if ((s = S.ck(cudaMemcpyAsync(S.dvec2.p, eg.data() + nconv, sizeof(double) * nr, cudaMemcpyHostToDevice, st),
                        "eg")))
            return s;
          dim3 g((unsigned)std::min(64, (mtxd + 255) / 256), nr);
          k_jacobi<<<g, 256, 0, st>>>(mtxd, PP + (size_t)nconv * mtxd, mtxd, HPP + (size_t)nconv * mtxd, mtxd,
                                      (const double*)S.dvec2.p, (const double*)S.hdiag_d.p);
          std::vector<zc> nrm;
          if ((s = S.coldots(PP + (size_t)nconv * mtxd, mtxd, PP + (size_t)nconv * mtxd, mtxd, nr, nrm))) return s;
          std::vector<double> sc(nr);
          for (int i = 0; i < nr; ++i) sc[i] = 1.0 / sqrt(nrm[i].real());
          if ((s = S.colscale(PP + (size_t)nconv * mtxd, mtxd, nr, sc))) return s;
          lortho = false;
          tk7.stop();
          if ((s = S.hk(PP + (size_t)nconv * mtxd, mtxd, HPP + (size_t)nconv * mtxd, mtxd, nr))) return s;
        }
      }
      if (lexit || lconv) break;
    }
    if (!lsafe) mcref = 3;
    // ---- ditsp_c16_ritz ----
    lconv = false;
    int nsize = nexact + nitold + niter - nconv;
    const int nlow = nexact + nitold - nconv;
    if (nsize > mxdsml) return fail(kBadArg, "ditsp_c16_ritz: change mxdsml");
    if (nconv < niter)
    {
      S.touch(nlow + nconv);
      if ((s = S.copycols(S.B(nlow + nconv), mtxd, PP + (size_t)nconv * mtxd, mtxd, niter - nconv))) return s;
    }
    if (!lsafe || niter == nconv) {
      ++nsize;
      if (nsize > mxdsml) return fail(kBadArg, "ditsp_c16_ritz: change mxdsml");
      std::vector<Z> rv(mtxd);
      for (int k = 0; k < mtxd; ++k) {
        const double xr = ran2(iseed);
        const double xi = ran2(iseed);
        rv[k] = make_cuDoubleComplex(xr, xi);
      }
      S.touch(nsize - 1);
      if ((s = S.ck(cudaMemcpyAsync(S.B(nsize - 1), rv.data(), sizeof(Z) * mtxd, cudaMemcpyHostToDevice, st), "ran")))
        return s;
      if ((s = S.ck(cudaStreamSynchronize(st), "ran"))) return s;
    }
    {
      std::vector<int> irowb;
      S.touch(nexact + nconv);
      if ((s = S.grsch_loop(false, (Z*)S.bas.p, (Z*)S.hbas.p, nexact + nconv, nsize, irowb, true))) return s;
      int ired;
      if ((s = S.grsch_shift((Z*)S.bas.p, mtxd, nexact + nconv, nsize, irowb, &ired))) return s;
      nsize -= ired;
    }
    if (nsize > mtxd) return fail(kBadArg, "ditsp_c16_ritz: problems with Gram-Schmidt");
    const int lo = nexact + nconv;
    S.touch(lo);
    if ((s = S.hk(S.B(lo), mtxd, S.HB(lo), mtxd, nsize - lo))) return s;
    if ((s = S.smallV.ensure(sizeof(Z) * (size_t)nsize * nsize))) return s;
    // hamsm = hbas^H bas (ditsp_c16_ritz.f90:195); zheevd reads its lower triangle only, which
    // zherkx computes at half the cost of the full product
    {
      Solver::Tick tk8(&S, 8);
      const double b0 = 0.0;
      Z* H = (Z*)S.smallV.p;
      // the leading block over columns untouched since the previous Ritz step is that step's
      // (the same products); only the rows of the new columns are computed
      const int c = std::min(S.ham_clean, std::min(S.ham_prev_n, nsize));
      if (c > 0) {
        ++S.ham_reused;
        if ((s = S.ck(cudaMemcpy2DAsync(H, sizeof(Z) * (size_t)nsize, S.ham_prev.p, sizeof(Z) * (size_t)S.ham_prev_n,
                                        sizeof(Z) * (size_t)c, c, cudaMemcpyDeviceToDevice, st),
                      "ritz hamsm reuse")))
          return s;
      } else {
        ++S.ham_full;
      }
      // rows [c, nsize) of the lower triangle. Columns j < zcols of bas vanish below row zrows, so
      // hbas(:, i)^H bas(:, j) for those columns runs over zrows rows: one product over zrows rows
      // for the columns below zcols (the rectangle, upper entries of its diagonal block included, which
      // zheevd does not read), one over mtxd rows for the columns [zcols, c), and zherkx (the lower
      // triangle) for the columns [max(c, zcols), nsize).
      if (c < nsize) {
        const int cz = std::min(S.zcols, nsize);
        if (cz > 0 &&
            (s = S.gemm(CUBLAS_OP_C, CUBLAS_OP_N, nsize - c, cz, S.zrows, S.one, S.HB(c), mtxd, S.B(0), mtxd, S.zero,
                        H + c, nsize, "ritz hamsm zero-padded columns")))
          return s;
        if (c > cz &&
            (s = S.gemm(CUBLAS_OP_C, CUBLAS_OP_N, nsize - c, c - cz, mtxd, S.one, S.HB(c), mtxd, S.B(cz), mtxd,
                        S.zero, H + (size_t)cz * nsize + c, nsize, "ritz hamsm rows")))
            return s;
        const int d0 = std::max(c, cz);
        if (d0 < nsize && S.ham_full_gemm) {
          // the whole square (twice the products of the triangle, at the full GEMM rate)
          if ((s = S.gemm(CUBLAS_OP_C, CUBLAS_OP_N, nsize - d0, nsize - d0, mtxd, S.one, S.HB(d0), mtxd, S.B(d0),
                          mtxd, S.zero, H + (size_t)d0 * nsize + d0, nsize, "ritz hamsm block")))
            return s;
        } else if (d0 < nsize && cublasZherkx(S.blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_C, nsize - d0, mtxd, &S.one,
                                              S.HB(d0), mtxd, S.B(d0), mtxd, &b0, H + (size_t)d0 * nsize + d0,
                                              nsize) != CUBLAS_STATUS_SUCCESS) {
          return fail(kCublas, "ritz hamsm");
        }
      }
      // keep it for the next Ritz step (zheevd overwrites smallV)
      if ((s = S.ham_prev.ensure(sizeof(Z) * (size_t)nsize * nsize)) ||
          (s = S.ck(cudaMemcpyAsync(S.ham_prev.p, H, sizeof(Z) * (size_t)nsize * nsize, cudaMemcpyDeviceToDevice, st),
                    "ritz hamsm keep")))
        return s;
      S.ham_prev_n = nsize;
      S.ham_clean = nsize;
    }
    // The decisions below read the eigenvalues up to the first gap above epsa past ndeg and niter,
    // and niter is capped at nitcap; psi and hpsi use the first niter eigenvectors. So only the
    // lowest nitcap + 2 pairs are computed (zheevdx), unless the degeneracy count ndeg runs into
    // that bound, when the full decomposition is taken (the reference computes all pairs,
    // ditsp_c16_ritz.f90:200; the decisions are the same).
    const int nitcap = std::min(std::min((mxdsml - nexact + nconv) / 2, nexact), mxdbnd);
    int nval = S.partial_eig ? std::min(nsize, nitcap + 2) : nsize;
    std::vector<double> egs;
    if (nval < nsize) {
      // if the full decomposition is needed after all, ham_prev still holds the matrix
      if ((s = S.diag((Z*)S.smallV.p, nsize, egs, nval))) return s;
    } else {
      if ((s = S.diag((Z*)S.smallV.p, nsize, egs))) return s;
    }
    auto count_ndeg = [&](int nv) {
      int nd = neig;
      for (int i = neig; i < nv; ++i) {
        if (fabs(egs[i] - egs[i - 1]) > epsa) break;
        nd = i + 1;
      }
      return nd;
    };
    ndeg = count_ndeg(nval);
    if (nval < nsize && ndeg == nval) {
      // a degenerate cluster reaches the computed pairs: decompose fully
      if ((s = S.ck(cudaMemcpyAsync(S.smallV.p, S.ham_prev.p, sizeof(Z) * (size_t)nsize * nsize,
                                    cudaMemcpyDeviceToDevice, st),
                    "ritz hamsm again")))
        return s;
      ++S.n_eig_full_again;
      if ((s = S.diag((Z*)S.smallV.p, nsize, egs))) return s;
      nval = nsize;
      ndeg = count_ndeg(nval);
    }
    for (int i = 0; i < nsize; ++i) eg[i] = i < nval ? egs[i] : 0.0;
    ndeg = std::min(ndeg, mxdbnd);
    niter = ndeg + 1;
    if (nsize > niter) {
      for (int i = ndeg + 1; i < nval; ++i) {       // beyond nval niter exceeds nitcap: capped below
        if (fabs(eg[i] - eg[i - 1]) > epsa) break;
        niter = i + 1;
      }
    }
    niter = std::max(std::min(niter, nitcap), ndeg);
    if (nconv > 0) {
      // the test reads rows [0, nexact + nconv) of the first nconv eigenvectors only
      const int vrows = std::min(nsize, nexact + nconv);
      std::vector<Z> vh((size_t)nsize * nconv);
      if ((s = S.ck(cudaMemcpy2DAsync(vh.data(), sizeof(Z) * (size_t)nsize, S.smallV.p, sizeof(Z) * (size_t)nsize,
                                      sizeof(Z) * (size_t)vrows, nconv, cudaMemcpyDeviceToHost, st),
                    "vsm")))
        return s;
      if ((s = S.ck(cudaStreamSynchronize(st), "vsm"))) return s;
      const int kmax = nconv;
      for (int k = 0; k < kmax; ++k) {
        const int nmax = nconv;
        nconv = 0;
        bool ljump = true;
        for (int n = 0; n < nmax; ++n) {
          double xn = 0;
          for (int i = 0; i < nexact + nmax; ++i)
            xn += vh[(size_t)n * nsize + i].x * vh[(size_t)n * nsize + i].x +
                  vh[(size_t)n * nsize + i].y * vh[(size_t)n * nsize + i].y;
          if (xn < C0P99) {
            ljump = false;
            break;
          }
          nconv = n + 1;
        }
        if (ljump && fabs(eg[nconv] - eg[nconv - 1]) < epsa) {
          --nconv;
          ljump = false;
        }
        if (ljump || nconv == 0) break;
      }
    }
    // psi = bas V, hpsi = hbas V (ditsp_c16_ritz.f90:284-287): split-TF32 tensor-core products in the
    // mixed form (V and the subspace Hamiltonian stay FP64), FP64 ZGEMM otherwise
    Solver::Tick tk9(&S, 9);
    // psi: the leading zcols columns of bas vanish below row zrows, so their share of bas V is added
    // to the first zrows rows only
    const int cz = std::min(S.zcols, nsize);
    const Z* V = (const Z*)S.smallV.p;
    if (S.tc_rot && !(S.basis_i8 && (S.i8_mask & Solver::kI8Rot))) {
      if ((s = tc_zgemm_nn(c, mtxd, niter, nsize - cz, S.B(cz), mtxd, V + cz, nsize, PP, mtxd, st)) ||
          (cz > 0 && (s = tc_zgemm_nn(c, S.zrows, niter, cz, S.bas.p, mtxd, V, nsize, PP, mtxd, st, true))) ||
          (s = tc_zgemm_nn(c, mtxd, niter, nsize, S.hbas.p, mtxd, S.smallV.p, nsize, HPP, mtxd, st)))
        return s;
    } else {
      if ((s = S.gemm(CUBLAS_OP_N, CUBLAS_OP_N, mtxd, niter, nsize - cz, S.one, S.B(cz), mtxd, V + cz, nsize,
                      S.zero, PP, mtxd, "ritz psi")))
        return s;
      if (cz > 0 && (s = S.gemm(CUBLAS_OP_N, CUBLAS_OP_N, S.zrows, niter, cz, S.one, (Z*)S.bas.p, mtxd, V, nsize, S.one,
                                PP, mtxd, "ritz psi zero-padded columns")))
        return s;
      if ((s = S.gemm(CUBLAS_OP_N, CUBLAS_OP_N, mtxd, niter, nsize, S.one, (Z*)S.hbas.p, mtxd, (Z*)S.smallV.p, nsize,
                      S.zero, HPP, mtxd, "ritz hpsi")))
        return s;
    }
    if (niter > nconv) {
      S.touch(nexact + nconv);
      if ((s = S.copycols(S.B(nexact + nconv), mtxd, PP + (size_t)nconv * mtxd, mtxd, niter - nconv))) return s;
      if ((s = S.copycols(S.HB(nexact + nconv), mtxd, HPP + (size_t)nconv * mtxd, mtxd, niter - nconv))) return s;
    }
    if (nconv >= ndeg) neig = ndeg;
    xmax = S.xmax_error(neig);
    if (xmax < 0) return fail(kCuda, "ditsp_c16: residual evaluation failed");
    tk9.stop();
    if (itlog && ic <= itlog_rows) {
      // iteration log row: elapsed s, xmax, nconv, H|psi> products so far, eg(1:mxdbnd)
      double* row = itlog + (size_t)(ic - 1) * (4 + mxdbnd);
      row[0] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
      row[1] = xmax;
      row[2] = nconv;
      row[3] = (double)S.ihk;
      for (int i = 0; i < mxdbnd; ++i) row[4 + i] = i < std::min(nsize, nval) ? eg[i] : 0.0;
    }
    if (ipr > 2)
      printf("  ditsp_c16_ritz ic = %d  nconv = %d  niter = %d  nsize = %d  ndeg = %d  xmax = %.6e  e1 = %.12f\n", ic,
             nconv, niter, nsize, ndeg, xmax, eg[0]);
    lconv = xmax < epspsi * epspsi;
    if (lconv) break;
    nitold = niter;
    lortho = true;
    lsafe = true;
    if (xmax < C0P01) mcref = std::min(mcref + 2, 8);
  }
  if (!lconv) {
    *ifail = 1 + (int)(-log10(xmax));
    if (*ifail == 0) *ifail = 1;
  }
  for (int i = 0; i < neig; ++i) ei[i] = eg[i];
  *neig_io = neig;
  *ihkpsum = S.ihk;
  if (packed) {
    if ((s = S.ck(cudaMemcpy2DAsync(psi, ldp * sizeof(Z), PP, mtxd * sizeof(Z), mtxd * sizeof(Z), mxdbnd,
                                    cudaMemcpyDeviceToDevice, st),
                  "unpack")))
      return s;
    if ((s = S.ck(cudaMemcpy2DAsync(hpsi, ldp * sizeof(Z), HPP, mtxd * sizeof(Z), mtxd * sizeof(Z), mxdbnd,
                                    cudaMemcpyDeviceToDevice, st),
                  "unpack")))
      return s;
  }
  if (ipr > 1) {
    const double tot = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    printf("  ditsp_c16: %lld H|psi> band products, total %.4f s: H|psi> %.4f s, Gram-Schmidt %.4f s, "
           "subspace eigensolve %.4f s, other %.4f s\n",
           S.ihk, tot, S.tphase[0], S.tphase[1], S.tphase[2], tot - S.tphase[0] - S.tphase[1] - S.tphase[2]);
    printf("  ditsp_c16: Gram-Schmidt %lld calls, %lld vectors: passes against converged %.4f s, "
           "in-block %.4f s (%lld modified Gram-Schmidt leaves, %lld Cholesky QR dropping %lld vectors, %lld shifted, "
           "%lld fallbacks: %lld factorisation, %lld drop rule, %lld conditioning)\n",
           S.n_gs, S.n_gs_vec, S.tphase[4], S.tphase[3], S.n_leaf, S.n_chol, S.n_chol_dropped, S.n_chol_shifted,
           S.n_chol_fallback, S.n_fb_info, S.n_fb_drop, S.n_fb_cond);
    printf("  ditsp_c16: outside: residual norms %.4f s, span test %.4f s, relaxation %.4f s, Ritz subspace "
           "Hamiltonian %.4f s (%lld reused leading blocks, %lld full), Ritz rotations + residual check %.4f s\n",
           S.tphase[5], S.tphase[6], S.tphase[7], S.tphase[8], S.ham_reused, S.ham_full, S.tphase[9]);
    printf("  ditsp_c16: Cholesky QR parts: Gram %.4f s, factorisation %.4f s, triangular solves %.4f s; "
           "partial subspace eigensolves redone in full: %lld; basis products: %lld int8 tensor-core (%d slices), "
           "%lld cuBLAS\n",
           S.tphase[10], S.tphase[11], S.tphase[12], S.n_eig_full_again, S.n_i8, S.oz_slices, S.n_cublas);
    fflush(stdout);
  }
  if ((s = S.ck(cudaStreamSynchronize(st), "ditsp"))) return s;
  if (S.basis_i8 && (s = oz_read_error(c->ozs))) return s;
  return lconv ? kOk : kNotConverged;
}

void ditsp_release(cpw_b200_ctx* c) {
  if (c->ditsp_sol) cusolverDnDestroy((cusolverDnHandle_t)c->ditsp_sol);
  c->ditsp_sol = nullptr;
}

}  // namespace cpwb
