// Adjoint of H|psi> for fixed wavefunctions (Hellmann-Feynman):
//
//  * density      rho(r) = sum_n f_n |psi_n(r)|^2 on the FFT box, with psi_n(r) the
//                 unscaled backward transform -- what Src/omp/charge_by_fft.f90
//                 (:185-199) accumulates; rho/N is dE/dV(r) for E = sum_n f_n <psi_n|H|psi_n>.
//  * local term   dE/dtau_aj = sum_r g(r) dV(r)/dtau_aj for V(r) = sum_G V(G) e^{iG.r},
//                 V(G) = sum_a e^{-2 pi i m.tau_a} v_t(G); with FG = sum_r g e^{-iG.r}:
//                 dE/dtau_aj = Re sum_G (-2 pi i m_j) e^{-2 pi i m.tau_a} v_t(G) conj(FG(G))
//                 (the structure-factor derivative of Src/ALFA/for_str_local_force.f90:102-145).
//  * KB term      P = X^H psi, Q_j = X^H (G_j psi); dE/dtau_aj = -4 pi sum_n f_n
//                 sum_{projectors of a} xnlkb Im(conj(P) Q_j) -- the dhd(1..4) products of
//                 Src/ALFA/for_str_nl_kb.f90:289-362 written with the projectors of
//                 proj_nl_kb_c16 (d/dtau of e^{-2 pi i G.tau} is -2 pi i G).
// Positions tau are lattice coordinates; derivatives are covariant (per lattice
// coordinate). Band-block recomputation: the density recomputes psi(r) chunk by
// chunk through the slab, nothing real-space is kept between calls.
#include <cufft.h>
#include <math.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/cpw_b200.h"
#include "context.hpp"

namespace cpwb {
namespace {

using Z = cuDoubleComplex;
constexpr int kDensThreads = 256;
constexpr int kDensCB = 32;

// inverse z of the kept planes of every band of the chunk, |.|^2 accumulated with
// the band weights; one CTA per 32 xy-columns; rho += the chunk's contribution
__global__ void __launch_bounds__(kDensThreads)
k_dens_z(LocalPlan p, int nbc, const double* __restrict__ occ, const C2<double>* __restrict__ twz,
         const C2<double>* __restrict__ W, double* __restrict__ rho) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int cb = kDensCB, n3 = p.n3, r1 = p.dz.r1, r2 = p.dz.r2;
  C2<double>* Cs = reinterpret_cast<C2<double>*>(smem_raw);
  double* acc = reinterpret_cast<double*>(Cs + (size_t)n3 * cb);
  C2<double>* sz = reinterpret_cast<C2<double>*>(acc + (size_t)n3 * cb);
  const long long c0 = (long long)blockIdx.x * cb;
  const int ncol = (int)min((long long)cb, p.plane - c0);
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < n3; i += nt) sz[i] = twz[i];
  for (int i = tid; i < n3 * cb; i += nt) acc[i] = 0.0;
  for (int b = 0; b < nbc; ++b) {
    const C2<double>* Wb = W + (size_t)b * p.nz * (size_t)p.plane + c0;
    const double f = occ[b];
    __syncthreads();
    for (int it = tid; it < cb * p.nz; it += nt) {
      const int cl = it % cb, zi = it / cb;
      if (cl < ncol) Cs[(size_t)kept_to_idx(zi, p.kd3, n3, p.nz) * cb + cl] = Wb[(size_t)zi * p.plane + cl];
    }
    __syncthreads();
    for (int it = tid; it < cb * r2; it += nt) {
      const int cl = it % cb, n2i = it / cb;
      if (cl < ncol) {
        radix_dispatch(r1, [&](auto rc_) {
          constexpr int RR = decltype(rc_)::value;
          C2<double> v[RR];
#pragma unroll
          for (int a = 0; a < RR; ++a) {
            const int z = r2 * a + n2i;
            v[a] = idx_to_kept(z, p.kd3, n3, p.nz) >= 0 ? Cs[(size_t)z * cb + cl] : mk<double>(0.0, 0.0);
          }
          DFT<RR, +1, double>::run(v);
#pragma unroll
          for (int a = 0; a < RR; ++a)
            Cs[(size_t)(r2 * a + n2i) * cb + cl] = a == 0 ? v[0] : cmulc<double>(v[a], sz[n2i * a]);
        });
      }
    }
    __syncthreads();
    for (int it = tid; it < cb * r1; it += nt) {
      const int cl = it % cb, k1 = it / cb;
      if (cl < ncol) {
        radix_dispatch(r2, [&](auto rc_) {
          constexpr int RR = decltype(rc_)::value;
          C2<double> v[RR];
#pragma unroll
          for (int a = 0; a < RR; ++a) v[a] = Cs[(size_t)(r2 * k1 + a) * cb + cl];
          DFT<RR, +1, double>::run(v);
#pragma unroll
          for (int a = 0; a < RR; ++a) acc[(size_t)(k1 + r1 * a) * cb + cl] += f * (v[a].x * v[a].x + v[a].y * v[a].y);
        });
      }
    }
  }
  __syncthreads();
  for (int it = tid; it < cb * n3; it += nt) {
    const int cl = it % cb, z = it / cb;
    if (cl < ncol) rho[(size_t)z * p.plane + c0 + cl] += acc[(size_t)z * cb + cl];
  }
}

__device__ __forceinline__ double block_sum3(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;   // valid in thread 0
}

__device__ __forceinline__ int freq(int i, int n) { return i <= (n - 1) / 2 ? i : i - n; }

// one CTA per atom: dE/dtau_aj = Re sum_G (-2 pi i m_j) e^{-2 pi i m.tau_a} v_t(G) conj(FG(G))
__global__ void __launch_bounds__(256)
k_structure_grad(int n1, int n2, int n3, const Z* __restrict__ FG, const double* __restrict__ vgt,
                 const int* __restrict__ atom_type, const double* __restrict__ tau, double* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Z* px = reinterpret_cast<Z*>(smem_raw);
  Z* py = px + n1;
  Z* pz = py + n2;
  __shared__ double sh[32];
  const int a = blockIdx.x;
  const double tx = tau[3 * a], ty = tau[3 * a + 1], tz = tau[3 * a + 2];
  for (int i = threadIdx.x; i < n1; i += blockDim.x) {
    double s, c;
    sincospi(-2.0 * freq(i, n1) * tx, &s, &c);
    px[i] = make_cuDoubleComplex(c, s);
  }
  for (int i = threadIdx.x; i < n2; i += blockDim.x) {
    double s, c;
    sincospi(-2.0 * freq(i, n2) * ty, &s, &c);
    py[i] = make_cuDoubleComplex(c, s);
  }
  for (int i = threadIdx.x; i < n3; i += blockDim.x) {
    double s, c;
    sincospi(-2.0 * freq(i, n3) * tz, &s, &c);
    pz[i] = make_cuDoubleComplex(c, s);
  }
  __syncthreads();
  const double* v = vgt + (size_t)atom_type[a] * n1 * n2 * n3;
  double g0 = 0, g1 = 0, g2 = 0;
  const long long ntot = (long long)n1 * n2 * n3;
  for (long long t = threadIdx.x; t < ntot; t += blockDim.x) {
    const int x = (int)(t % n1);
    const long long r = t / n1;
    const int y = (int)(r % n2), z = (int)(r / n2);
    const double vt = v[t];
    if (vt == 0.0) continue;
    const Z ph = cuCmul(cuCmul(px[x], py[y]), pz[z]);
    const Z fg = FG[t];
    // w = e^{-2 pi i m.tau} v_t conj(FG); the term is Re(-2 pi i m_j w) = 2 pi m_j Im(w)
    const double wim = vt * (ph.y * fg.x - ph.x * fg.y);
    g0 += freq(x, n1) * wim;
    g1 += freq(y, n2) * wim;
    g2 += freq(z, n3) * wim;
  }
  const double tp = 6.283185307179586476925286766559005768;
  const double s0 = block_sum3(g0, sh);
  const double s1 = block_sum3(g1, sh);
  const double s2 = block_sum3(g2, sh);
  if (threadIdx.x == 0) {
    out[3 * a] = tp * s0;
    out[3 * a + 1] = tp * s1;
    out[3 * a + 2] = tp * s2;
  }
}

// y_j = G_j o psi for j = 0..2 (G lattice components of the basis), bands [0, nb)
__global__ void k_scale_by_g(int m, int nb, const int* __restrict__ kgvb, const Z* __restrict__ psi, long long ld,
                             Z* __restrict__ y) {
  const long long n = (long long)m * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long b = t / m;
    const int i = (int)(t - b * m);
    const Z v = psi[b * ld + i];
    for (int j = 0; j < 3; ++j) {
      const double g = (double)kgvb[3 * i + j];
      y[((size_t)j * nb + b) * m + i] = make_cuDoubleComplex(g * v.x, g * v.y);
    }
  }
}

// c[a][j] = sum_n f_n Im(conj(P_an) Q_jan), P (nanl x nb), Q_j (nanl x nb) stacked in j
__global__ void k_nl_contract(int nanl, int nb, const Z* __restrict__ P, const Z* __restrict__ Q,
                              const double* __restrict__ occ, double* __restrict__ c) {
  const int a = blockIdx.x;
  __shared__ double sh[32];
  double s[3] = {0, 0, 0};
  for (int n = threadIdx.x; n < nb; n += blockDim.x) {
    const Z p = P[(size_t)n * nanl + a];
    for (int j = 0; j < 3; ++j) {
      const Z q = Q[((size_t)j * nb + n) * nanl + a];
      s[j] += occ[n] * (p.x * q.y - p.y * q.x);
    }
  }
  for (int j = 0; j < 3; ++j) {
    const double t = block_sum3(s[j], sh);
    if (threadIdx.x == 0) c[3 * a + j] = t;
  }
}

// w(i) = sum_n f_n |c_n(i)|^2 (the kinetic stress weight of plane wave i)
__global__ void k_band_weights(int m, int nb, const Z* __restrict__ psi, long long ld, const double* __restrict__ f,
                               double* __restrict__ w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int n = 0; n < nb; ++n) {
      const Z c = psi[(size_t)n * ld + i];
      s += f[n] * (c.x * c.x + c.y * c.y);
    }
    w[i] = s;
  }
}

// M(n, a) = f_n conj(P(a, n)) xnlkb(a), M (nb x nanl) column-major
__global__ void k_stress_m(int nanl, int nb, const Z* __restrict__ P, const double* __restrict__ f,
                           const double* __restrict__ xnl, Z* __restrict__ M) {
  const long long n = (long long)nanl * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(t / nb), b = (int)(t - (long long)a * nb);
    const Z p = P[(size_t)b * nanl + a];
    const double s = f[b] * xnl[a];
    M[(size_t)a * nb + b] = make_cuDoubleComplex(s * p.x, -s * p.y);
  }
}

}  // namespace

// The two blocks the strain derivative of E = sum_n f_n <psi_n|H|psi_n> needs besides the
// density: w(i) = sum_n f_n |c_n(i)|^2 (kinetic) and Y = psi diag(f) P^H diag(xnlkb)
// (mtxd x nanl, KB term: dE = 2 Re sum conj(dX) Y for a change dX of the projectors).
int stress_inputs_device(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, const double* occ, double* w,
                         void* y, cudaStream_t st) {
  if (!c->have_basis) return fail(kNotReady, "stress inputs: basis must be set");
  const int na = c->nanl, m = c->mtxd;
  if (nb < 0 || ldpsi < m) return fail(kBadArg, "stress inputs: invalid block");
  if (m == 0) return kOk;
  int s;
  DevBuf P, M, docc, dxnl;
  if ((s = docc.ensure(sizeof(double) * std::max(nb, 1)))) return s;
  cudaError_t e;
  if (nb > 0 && (e = cudaMemcpyAsync(docc.p, occ, sizeof(double) * nb, cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return cuda_fail(e, "stress inputs occ");
  if (nb == 0) {
    if ((e = cudaMemsetAsync(w, 0, sizeof(double) * m, st)) != cudaSuccess) return cuda_fail(e, "stress inputs");
  } else {
    k_band_weights<<<std::min(1184, (m + 255) / 256), 256, 0, st>>>(m, nb, (const Z*)psi, ldpsi,
                                                                   (const double*)docc.p, w);
  }
  if (na > 0) {
    if (nb == 0) {
      if ((e = cudaMemsetAsync(y, 0, sizeof(Z) * (size_t)m * na, st)) != cudaSuccess) return cuda_fail(e, "stress");
    } else {
      if ((s = P.ensure(sizeof(Z) * (size_t)na * nb)) || (s = M.ensure(sizeof(Z) * (size_t)na * nb)) ||
          (s = dxnl.ensure(sizeof(double) * na)))
        return s;
      if ((e = cudaMemcpyAsync(dxnl.p, c->xnl_h.data(), sizeof(double) * na, cudaMemcpyHostToDevice, st)) !=
          cudaSuccess)
        return cuda_fail(e, "stress inputs xnlkb");
      cublasSetStream(c->blas, st);
      const Z one = make_cuDoubleComplex(1, 0), zero = make_cuDoubleComplex(0, 0);
      cublasStatus_t bs = cublasZgemm(c->blas, CUBLAS_OP_C, CUBLAS_OP_N, na, nb, m, &one, (const Z*)c->anl.p, m,
                                      (const Z*)psi, (int)ldpsi, &zero, (Z*)P.p, na);
      if (bs != CUBLAS_STATUS_SUCCESS) return fail(kCublas, "stress inputs zgemm P");
      k_stress_m<<<std::max(1, std::min(1184, (na * nb + 255) / 256)), 256, 0, st>>>(
          na, nb, (const Z*)P.p, (const double*)docc.p, (const double*)dxnl.p, (Z*)M.p);
      bs = cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, m, na, nb, &one, (const Z*)psi, (int)ldpsi, (const Z*)M.p,
                       nb, &zero, (Z*)y, m);
      if (bs != CUBLAS_STATUS_SUCCESS) return fail(kCublas, "stress inputs zgemm Y");
    }
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "stress inputs");
  return kOk;
}

int density_device(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, const double* occ, void* rho,
                   cudaStream_t st) {
  if (!c->have_basis) return fail(kNotReady, "density: basis must be set");
  if (nb < 0 || ldpsi < c->mtxd) return fail(kBadArg, "density: bad neig or leading dimension");
  const LocalPlan& p = c->plan;
  cudaError_t e = cudaMemsetAsync(rho, 0, sizeof(double) * (size_t)p.plane * p.n3, st);
  if (e != cudaSuccess) return cuda_fail(e, "density memset");
  if (nb == 0 || c->mtxd == 0) return kOk;
  const size_t per_band = sizeof(C2<double>) * (size_t)p.nz * (size_t)p.plane;
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)nb, c->slab_budget / per_band));
  int s;
  if ((s = c->slab.ensure(per_band * (size_t)chunk))) return s;
  DevBuf docc;
  if ((s = docc.ensure(sizeof(double) * nb))) return s;
  if ((e = cudaMemcpyAsync(docc.p, occ, sizeof(double) * nb, cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return cuda_fail(e, "density occ");
  const size_t sm = (sizeof(C2<double>) + sizeof(double)) * (size_t)p.n3 * kDensCB + sizeof(C2<double>) * p.n3;
  if ((e = smem_limit((const void*)k_dens_z, (size_t)sm)) != cudaSuccess)
    return cuda_fail(e, "density attribute");
  for (int b0 = 0; b0 < nb; b0 += chunk) {
    const int nbc = std::min(chunk, nb - b0);
    e = launch_inverse_xy<double>(p, nbc, b0, (const C2<double>*)psi, ldpsi, (const int*)c->plane_start.p,
                                  (const int*)c->pw_idx.p, (const int*)c->pw_pos.p, (const C2<double>*)c->tw64[0].p,
                                  (const C2<double>*)c->tw64[1].p, (C2<double>*)c->slab.p, st);
    if (e != cudaSuccess) return cuda_fail(e, "density inverse xy");
    const unsigned grid = (unsigned)((p.plane + kDensCB - 1) / kDensCB);
    k_dens_z<<<grid, kDensThreads, sm, st>>>(p, nbc, (const double*)docc.p + b0, (const C2<double>*)c->tw64[2].p,
                                             (const C2<double>*)c->slab.p, (double*)rho);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "density z");
  }
  e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? kOk : cuda_fail(e, "density");
}

int structure_grad_device(cpw_b200_ctx* c, const void* g, int natom, const int* atom_type, const double* tau,
                          int ntype, const void* vgt, double* dedtau, cudaStream_t st) {
  if (!c->have_basis) return fail(kNotReady, "structure gradient: basis (box) must be set");
  const LocalPlan& p = c->plan;
  const long long ntot = (long long)p.n1 * p.n2 * p.n3;
  int s;
  DevBuf fg, dtype, dtau, dout;
  if ((s = fg.ensure(sizeof(Z) * (size_t)ntot)) || (s = dtype.ensure(sizeof(int) * std::max(natom, 1))) ||
      (s = dtau.ensure(sizeof(double) * 3 * std::max(natom, 1))) || (s = dout.ensure(sizeof(double) * 3 * std::max(natom, 1))))
    return s;
  for (int a = 0; a < natom; ++a)
    if (atom_type[a] < 0 || atom_type[a] >= ntype) return fail(kBadArg, "structure gradient: atom type out of range");
  cudaError_t e = cudaMemcpy2DAsync(fg.p, sizeof(Z), g, sizeof(double), sizeof(double), (size_t)ntot,
                                    cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "structure gradient copy");
  e = cudaMemset2DAsync((char*)fg.p + sizeof(double), sizeof(Z), 0, sizeof(double), (size_t)ntot, st);
  if (e != cudaSuccess) return cuda_fail(e, "structure gradient copy");
  cufftHandle plan;
  if (cufftPlan3d(&plan, p.n3, p.n2, p.n1, CUFFT_Z2Z) != CUFFT_SUCCESS) return fail(kCuda, "cufftPlan3d failed");
  cufftSetStream(plan, st);
  const cufftResult fr = cufftExecZ2Z(plan, (cufftDoubleComplex*)fg.p, (cufftDoubleComplex*)fg.p, CUFFT_FORWARD);
  if (fr != CUFFT_SUCCESS) {
    cufftDestroy(plan);
    return fail(kCuda, "cufftExecZ2Z failed");
  }
  if ((e = cudaMemcpyAsync(dtype.p, atom_type, sizeof(int) * natom, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(dtau.p, tau, sizeof(double) * 3 * natom, cudaMemcpyHostToDevice, st)) != cudaSuccess) {
    cufftDestroy(plan);
    return cuda_fail(e, "structure gradient upload");
  }
  const size_t sm = sizeof(Z) * ((size_t)p.n1 + p.n2 + p.n3);
  if (natom > 0) {
    smem_limit((const void*)k_structure_grad, (size_t)sm);
    k_structure_grad<<<natom, 256, sm, st>>>(p.n1, p.n2, p.n3, (const Z*)fg.p, (const double*)vgt,
                                             (const int*)dtype.p, (const double*)dtau.p, (double*)dout.p);
    e = cudaMemcpyAsync(dedtau, dout.p, sizeof(double) * 3 * natom, cudaMemcpyDeviceToHost, st);
  }
  cudaError_t e2 = cudaStreamSynchronize(st);
  cufftDestroy(plan);
  if (e != cudaSuccess) return cuda_fail(e, "structure gradient");
  return e2 == cudaSuccess ? kOk : cuda_fail(e2, "structure gradient");
}

int nl_grad_device(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, const double* occ,
                   const int* proj_atom, int natom, double* dedtau, cudaStream_t st) {
  if (!c->have_basis) return fail(kNotReady, "projector gradient: basis must be set");
  for (int a = 0; a < 3 * natom; ++a) dedtau[a] = 0.0;
  const int na = c->nanl, m = c->mtxd;
  if (na == 0 || nb == 0 || m == 0) return kOk;
  for (int a = 0; a < na; ++a)
    if (proj_atom[a] < 0 || proj_atom[a] >= natom) return fail(kBadArg, "projector gradient: proj_atom out of range");
  int s;
  DevBuf P, Q, Y, docc, dc;
  if ((s = P.ensure(sizeof(Z) * (size_t)na * nb)) || (s = Q.ensure(sizeof(Z) * 3 * (size_t)na * nb)) ||
      (s = Y.ensure(sizeof(Z) * 3 * (size_t)m * nb)) || (s = docc.ensure(sizeof(double) * nb)) ||
      (s = dc.ensure(sizeof(double) * 3 * na)))
    return s;
  cudaError_t e = cudaMemcpyAsync(docc.p, occ, sizeof(double) * nb, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "projector gradient occ");
  k_scale_by_g<<<1184, 256, 0, st>>>(m, nb, (const int*)c->kgvb.p, (const Z*)psi, ldpsi, (Z*)Y.p);
  cublasSetStream(c->blas, st);
  const Z one = make_cuDoubleComplex(1, 0), zero = make_cuDoubleComplex(0, 0);
  cublasStatus_t bs = cublasZgemm(c->blas, CUBLAS_OP_C, CUBLAS_OP_N, na, nb, m, &one, (const Z*)c->anl.p, m,
                                  (const Z*)psi, (int)ldpsi, &zero, (Z*)P.p, na);
  if (bs != CUBLAS_STATUS_SUCCESS) return fail(kCublas, "projector gradient zgemm P");
  bs = cublasZgemm(c->blas, CUBLAS_OP_C, CUBLAS_OP_N, na, 3 * nb, m, &one, (const Z*)c->anl.p, m, (const Z*)Y.p, m,
                   &zero, (Z*)Q.p, na);
  if (bs != CUBLAS_STATUS_SUCCESS) return fail(kCublas, "projector gradient zgemm Q");
  k_nl_contract<<<na, 128, 0, st>>>(na, nb, (const Z*)P.p, (const Z*)Q.p, (const double*)docc.p, (double*)dc.p);
  std::vector<double> ch(3 * (size_t)na);
  e = cudaMemcpyAsync(ch.data(), dc.p, sizeof(double) * 3 * na, cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return cuda_fail(e, "projector gradient copy");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "projector gradient");
  const double fpi = 12.566370614359172953850573533118011537;
  for (int a = 0; a < na; ++a)
    for (int j = 0; j < 3; ++j) dedtau[3 * proj_atom[a] + j] += -fpi * c->xnl_h[a] * ch[3 * (size_t)a + j];
  return kOk;
}

}  // namespace cpwb
