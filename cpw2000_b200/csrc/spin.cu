// H|psi> of two-component spinors, Src/hk_psi/reference/hk_psi_spin_c16.f90: psi_sp holds the
// up component of plane wave i at row 2i and the down component at row 2i+1 (0-based), the
// screened potential has nsp = 1, 2 or 4 components (1, sigma_z, sigma_x, sigma_y), and the
// KB projectors act on the interleaved 2 mtxd rows (the spin-orbit projectors anlsp).
//
// Each component is a stride-2 view of the spinor block: the plane lists are reused with doubled
// indices (plane wave i -> row 2i) and a doubled kinetic diagonal, so the same local kernels read
// and write the spinor rows in place. nsp = 1 and 2 run the fused local kernels once per
// component with its own potential (V, or V1 +- V2). nsp = 4 couples the components point by
// point: kernel A brings both components of a chunk of spinors to the kept-plane slab, a spinor
// z stage (below) transforms both columns, applies [[V1+V2, V3-iV4], [V3+iV4, V1-V2]] and
// transforms back, and kernel C gathers both.
#include <math.h>
#include <stdio.h>

#include <string>
#include <vector>

#include "context.hpp"
#include "hkpsi_kernels.cuh"

namespace cpwb {

namespace {

constexpr int kSpCols = 8;       // columns per CTA of the spinor z stage
constexpr int kSpThreads = 256;

__global__ void k_double_index(int m, const int* __restrict__ idx, const double* __restrict__ ek,
                               int* __restrict__ idx2, double* __restrict__ ek2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    idx2[i] = 2 * idx[i];
    ek2[2 * i] = ek[i];
    ek2[2 * i + 1] = ek[i];
  }
}

// z stage of the nsp = 4 form for one tile of kSpCols xy columns of one spinor: up slab of
// spinor b at W[b], down slab at W[nbc + b]. Potentials pre-scaled by 1/N in [z][y][x] order:
// vu = V1+V2, vd = V1-V2, and the off-diagonal V3 - iV4 = vr + i vi.
template <typename T>
__global__ void __launch_bounds__(kSpThreads)
k_z_spinor(LocalPlan p, int nbc, const T* __restrict__ vu, const T* __restrict__ vd, const T* __restrict__ vr,
           const T* __restrict__ vi, const C2<T>* __restrict__ twz, C2<T>* __restrict__ W) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n3 = p.n3, nz = p.nz, r1 = p.dz.r1, r2 = p.dz.r2;
  C2<T>* Cs = reinterpret_cast<C2<T>*>(smem_raw);             // [component][z][column]
  C2<T>* sz = Cs + 2 * (size_t)n3 * kSpCols;
  const long long c0 = (long long)blockIdx.x * kSpCols;
  const int ncol = (int)min((long long)kSpCols, p.plane - c0);
  const int b = blockIdx.y;
  const int tid = threadIdx.x, nt = blockDim.x;
  C2<T>* Wc[2] = {W + (size_t)b * nz * (size_t)p.plane + c0, W + (size_t)(nbc + b) * nz * (size_t)p.plane + c0};
  for (int i = tid; i < n3; i += nt) sz[i] = twz[i];
  for (int i = tid; i < 2 * n3 * kSpCols; i += nt) Cs[i] = mk<T>(T(0), T(0));
  __syncthreads();
  for (int it = tid; it < 2 * nz * kSpCols; it += nt) {
    const int cl = it % kSpCols, zi = (it / kSpCols) % nz, s = it / (kSpCols * nz);
    if (cl < ncol) Cs[((size_t)s * n3 + kept_to_idx(zi, p.kd3, n3, nz)) * kSpCols + cl] = Wc[s][(size_t)zi * p.plane + cl];
  }
  __syncthreads();
  // inverse pass 1 on both components
  for (int it = tid; it < 2 * kSpCols * r2; it += nt) {
    const int cl = it % kSpCols, n2i = (it / kSpCols) % r2, s = it / (kSpCols * r2);
    if (cl < ncol) {
      C2<T>* C = Cs + (size_t)s * n3 * kSpCols;
      with_radix<0>(r1, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<T> v[RR];
#pragma unroll
        for (int a = 0; a < RR; ++a) v[a] = C[(size_t)(r2 * a + n2i) * kSpCols + cl];
        DFT<RR, +1, T>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a)
          C[(size_t)(r2 * a + n2i) * kSpCols + cl] = a == 0 ? v[0] : cmulc<T>(v[a], sz[n2i * a]);
      });
    }
  }
  __syncthreads();
  // inverse pass 2 of both components -> 2x2 potential -> forward pass 1 of both
  for (int it = tid; it < kSpCols * r1; it += nt) {
    const int cl = it % kSpCols, k1 = it / kSpCols;
    if (cl < ncol) {
      with_radix<0>(r2, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<T> u[RR], d[RR];
        C2<T>* Cu = Cs;
        C2<T>* Cd = Cs + (size_t)n3 * kSpCols;
#pragma unroll
        for (int a = 0; a < RR; ++a) {
          u[a] = Cu[(size_t)(r2 * k1 + a) * kSpCols + cl];
          d[a] = Cd[(size_t)(r2 * k1 + a) * kSpCols + cl];
        }
        DFT<RR, +1, T>::run(u);
        DFT<RR, +1, T>::run(d);
#pragma unroll
        for (int a = 0; a < RR; ++a) {
          const size_t o = (size_t)(k1 + r1 * a) * p.plane + c0 + cl;
          const T a11 = vu[o], a22 = vd[o], xr = vr[o], xi = vi[o];
          const C2<T> pu = u[a], pd = d[a];
          // up' = (V1+V2) up + (V3 - i V4) down ; down' = (V1-V2) down + (V3 + i V4) up
          u[a] = mk<T>(a11 * pu.x + xr * pd.x - xi * pd.y, a11 * pu.y + xr * pd.y + xi * pd.x);
          d[a] = mk<T>(a22 * pd.x + xr * pu.x + xi * pu.y, a22 * pd.y + xr * pu.y - xi * pu.x);
        }
        DFT<RR, -1, T>::run(u);
        DFT<RR, -1, T>::run(d);
#pragma unroll
        for (int a = 0; a < RR; ++a) {
          Cu[(size_t)(r2 * k1 + a) * kSpCols + cl] = a == 0 ? u[0] : cmul<T>(u[a], sz[k1 * a]);
          Cd[(size_t)(r2 * k1 + a) * kSpCols + cl] = a == 0 ? d[0] : cmul<T>(d[a], sz[k1 * a]);
        }
      });
    }
  }
  __syncthreads();
  // forward pass 2, kept planes back to the slabs
  for (int it = tid; it < 2 * kSpCols * r2; it += nt) {
    const int cl = it % kSpCols, m2 = (it / kSpCols) % r2, s = it / (kSpCols * r2);
    if (cl < ncol) {
      const C2<T>* C = Cs + (size_t)s * n3 * kSpCols;
      with_radix<0>(r1, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<T> v[RR];
#pragma unroll
        for (int a = 0; a < RR; ++a) v[a] = C[(size_t)(r2 * a + m2) * kSpCols + cl];
        DFT<RR, -1, T>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a) {
          const int zi = idx_to_kept(m2 + r2 * a, p.kd3, n3, nz);
          if (zi >= 0) Wc[s][(size_t)zi * p.plane + cl] = v[a];
        }
      });
    }
  }
}

// X diag(xnlkb) of the spinor projectors (columns of 2 mtxd rows)
__global__ void k_scale_spin_cols(const C2<double>* __restrict__ a, C2<double>* __restrict__ b,
                                  const double* __restrict__ x, long long rows, int cols) {
  const long long n = rows * cols;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const double f = x[t / rows];
    b[t] = mk<double>(a[t].x * f, a[t].y * f);
  }
}

// Plane-wave kinetic term hpsi (+)= ekpg psi, one or two components per plane wave
// (Src/omp/hk_psi_kin_c16.f90).
__global__ void k_kinetic(int m, int nb, int nspin, const double* __restrict__ ek, const C2<double>* __restrict__ psi,
                          long long ldpsi, C2<double>* __restrict__ hpsi, long long ldh, int ladd) {
  const long long rows = (long long)nspin * m, n = rows * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long b = t / rows, r = t - b * rows;
    const double e = ek[r / nspin];
    const C2<double> x = psi[b * ldpsi + r];
    C2<double> y = mk<double>(e * x.x, e * x.y);
    if (ladd) {
      const C2<double> h0 = hpsi[b * ldh + r];
      y.x += h0.x;
      y.y += h0.y;
    }
    hpsi[b * ldh + r] = y;
  }
}

template <typename T>
int spin_local(cpw_b200_ctx* c, int nb, const C2<double>* psi, long long ldpsi, C2<double>* hpsi, long long ldh,
               cudaStream_t st, bool kinetic = true, int accum = 0) {
  LocalPlan p = c->plan;
  p.accum = accum;
  const bool f32 = sizeof(T) == 4;
  const int* ps = (const int*)c->plane_start.p;
  const int* idx2 = (const int*)c->sp_idx2.p;
  const int* pos = (const int*)c->pw_pos.p;
  const double* ek2 = kinetic ? (const double*)c->sp_ek2.p : nullptr;
  const C2<T>* tw[3];
  for (int a = 0; a < 3; ++a) tw[a] = (const C2<T>*)(f32 ? c->tw32[a].p : c->tw64[a].p);
  const DevBuf* v = f32 ? c->sp_v32 : c->sp_v64;
  const size_t per_band = sizeof(C2<T>) * (size_t)p.nz * (size_t)p.plane;
  C2<T>* W = (C2<T>*)c->slab.p;
  cudaError_t e;
  if (c->nsp != 4) {
    // V (nsp 1) or V1 +- V2 (nsp 2) per component, the fused kernels on stride-2 views
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)nb, c->slab_budget / per_band));
    if (int s = c->slab.ensure(per_band * (size_t)chunk)) return s;
    W = (C2<T>*)c->slab.p;
    for (int b0 = 0; b0 < nb; b0 += chunk) {
      const int nbc = std::min(chunk, nb - b0);
      for (int comp = 0; comp < 2; ++comp) {
        const T* vr = (const T*)v[c->nsp == 1 ? 0 : comp].p;
        e = launch_local<T>(p, nbc, b0, psi + comp, ldpsi, hpsi + comp, ldh, ps, idx2, pos, ek2, vr, tw[0], tw[1],
                            tw[2], W, st, nullptr);
        if (e != cudaSuccess) return cuda_fail(e, "hk_psi_spin local kernels");
      }
    }
    return kOk;
  }
  // nsp = 4: both components of a chunk of spinors in the slab, coupled in the z stage
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)nb, c->slab_budget / (2 * per_band)));
  if (int s = c->slab.ensure(2 * per_band * (size_t)chunk)) return s;
  W = (C2<T>*)c->slab.p;
  const size_t sm_pl = smem_planes<T>(p);
  auto* kc = kern::k_fwd_xy<T, 0, 0, 0, 0, 0>;
  if ((e = smem_limit((const void*)kc, (size_t)sm_pl)) != cudaSuccess)
    return cuda_fail(e, "hk_psi_spin attribute");
  const size_t sm_z = sizeof(C2<T>) * (2 * (size_t)p.n3 * kSpCols + p.n3);
  if ((e = smem_limit((const void*)k_z_spinor<T>, (size_t)sm_z)) != cudaSuccess)
    return cuda_fail(e, "hk_psi_spin attribute");
  const unsigned tiles = (unsigned)((p.plane + kSpCols - 1) / kSpCols);
  for (int b0 = 0; b0 < nb; b0 += chunk) {
    const int nbc = std::min(chunk, nb - b0);
    for (int comp = 0; comp < 2; ++comp) {
      e = launch_inverse_xy<T>(p, nbc, b0, psi + comp, ldpsi, ps, idx2, pos, tw[0], tw[1],
                               W + (size_t)comp * nbc * p.nz * p.plane, st);
      if (e != cudaSuccess) return cuda_fail(e, "hk_psi_spin inverse xy");
    }
    k_z_spinor<T><<<dim3(tiles, nbc), kSpThreads, sm_z, st>>>(p, nbc, (const T*)v[0].p, (const T*)v[1].p,
                                                               (const T*)v[2].p, (const T*)v[3].p, tw[2], W);
    for (int comp = 0; comp < 2; ++comp)
      kc<<<dim3(p.nz, nbc), kern::kThreadsPlanes, sm_pl, st>>>(p, b0, psi + comp, ldpsi, hpsi + comp, ldh, ps, idx2,
                                                               pos, ek2, tw[0], tw[1],
                                                               W + (size_t)comp * nbc * p.nz * p.plane);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "hk_psi_spin kernels");
  }
  return kOk;
}

}  // namespace

int ctx_set_potential_spin(cpw_b200_ctx* c, const double* vscr_sp, long long mxdscr, int nsp) {
  if (!c->have_basis) return fail(kNotReady, "set_potential_spin: call set_basis first (box size)");
  if (nsp != 1 && nsp != 2 && nsp != 4) return fail(kBadArg, "hk_psi_spin_c16: nsp is an incorrect value, should be 1,2,4");
  const LocalPlan& p = c->plan;
  const int n1 = p.n1, n2 = p.n2, n3 = p.n3;
  const long long id = c->ident;
  if (mxdscr < id * n2 * (long long)n3) return fail(kBadArg, "set_potential_spin: vscr smaller than id*n2*n3");
  const double inv = 1.0 / ((double)n1 * n2 * n3);
  const size_t N = (size_t)n1 * n2 * n3;
  const int ncomb = nsp;
  std::vector<double> v(N);
  std::vector<float> vf(N);
  for (int k = 0; k < ncomb; ++k) {
    for (int z = 0; z < n3; ++z)
      for (int y = 0; y < n2; ++y)
        for (int x = 0; x < n1; ++x) {
          const size_t r = ((size_t)z * n2 + y) * id + x, o = ((size_t)z * n2 + y) * n1 + x;
          auto col = [&](int j) { return vscr_sp[r + (size_t)j * mxdscr]; };
          double val;
          if (nsp == 1) val = col(0);
          else if (k == 0) val = col(0) + col(1);          // up: V1 + V2
          else if (k == 1) val = col(0) - col(1);          // down: V1 - V2
          else if (k == 2) val = col(2);                   // off-diagonal V3 - i V4: real part
          else val = -col(3);                              //                        imaginary part
          v[o] = val * inv;
          vf[o] = (float)v[o];
        }
    int s;
    if ((s = upload(c->sp_v64[k], v.data(), N * sizeof(double)))) return s;
    if ((s = upload(c->sp_v32[k], vf.data(), N * sizeof(float)))) return s;
  }
  c->nsp = nsp;
  return kOk;
}

int ctx_set_projectors_spin(cpw_b200_ctx* c, int nanl, const double* anlsp, long long ld, const double* xnlkb) {
  if (!c->have_basis) return fail(kNotReady, "set_projectors_spin: call set_basis first");
  if (nanl < 0) return fail(kBadArg, "set_projectors_spin: nanl < 0");
  const long long m2 = 2LL * c->mtxd;
  if (nanl > 0 && ld < m2) return fail(kBadArg, "set_projectors_spin: leading dimension smaller than 2*mtxd");
  c->nanl_sp = nanl;
  if (nanl == 0 || m2 == 0) return kOk;
  int s;
  const size_t bytes = (size_t)m2 * nanl * sizeof(C2<double>);
  if ((s = c->anl_sp.ensure(bytes)) || (s = c->anld_sp.ensure(bytes))) return s;
  cudaError_t e = cudaMemcpy2D(c->anl_sp.p, m2 * sizeof(C2<double>), anlsp, (size_t)ld * sizeof(C2<double>),
                               m2 * sizeof(C2<double>), nanl, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);   // landed before the context stream reads it
  if (e != cudaSuccess) return cuda_fail(e, "set_projectors_spin copy");
  DevBuf dx;
  if ((s = upload(dx, xnlkb, (size_t)nanl * sizeof(double)))) return s;
  k_scale_spin_cols<<<1184, 256, 0, c->stream>>>((const C2<double>*)c->anl_sp.p, (C2<double>*)c->anld_sp.p,
                                                 (const double*)dx.p, m2, nanl);
  e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? kOk : cuda_fail(e, "set_projectors_spin");
}

int ctx_hkpsi_kin_device(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, void* hpsi, long long ldh,
                         bool ladd, int nspin, cudaStream_t st) {
  if (!c->have_basis) return fail(kNotReady, "hk_psi_kin: basis must be set");
  if (nspin != 1 && nspin != 2) return fail(kBadArg, "hk_psi_kin_c16: nspin should be 1 or 2");
  if (nb < 0) return fail(kBadArg, "hk_psi_kin: neig < 0");
  const long long m = c->mtxd;
  if (nb == 0 || m == 0) return kOk;
  if (ldpsi < nspin * m || ldh < nspin * m) return fail(kBadArg, "hk_psi_kin: leading dimension smaller than nspin*mtxd");
  k_kinetic<<<1184, 256, 0, st>>>((int)m, nb, nspin, (const double*)c->ekpg.p, (const C2<double>*)psi, ldpsi,
                                  (C2<double>*)hpsi, ldh, ladd ? 1 : 0);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? kOk : cuda_fail(e, "hk_psi_kin");
}

int ctx_hkpsi_loc_general(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, void* hpsi, long long ldh,
                          bool ladd, int nspin, cudaStream_t st) {
  if (nspin != 1 && nspin != 2) return fail(kBadArg, "hk_psi_loc_c16: nspin should be 1 or 2");
  if (!c->have_basis) return fail(kNotReady, "hk_psi_loc: basis must be set");
  if (nb < 0) return fail(kBadArg, "hk_psi_loc: neig < 0");
  const long long m = c->mtxd;
  if (nb == 0 || m == 0) return kOk;
  if (ldpsi < nspin * m || ldh < nspin * m) return fail(kBadArg, "hk_psi_loc: leading dimension smaller than nspin*mtxd");
  const C2<double>* x = (const C2<double>*)psi;
  C2<double>* y = (C2<double>*)hpsi;
  if (nspin == 2) {
    if (c->nsp == 0) return fail(kNotReady, "hk_psi_loc: spin potential must be set (cpw_b200_set_potential_spin)");
    int s;
    if ((s = c->sp_idx2.ensure((size_t)m * sizeof(int))) || (s = c->sp_ek2.ensure((size_t)2 * m * sizeof(double))))
      return s;
    k_double_index<<<592, 256, 0, st>>>((int)m, (const int*)c->pw_idx.p, (const double*)c->ekpg.p,
                                        (int*)c->sp_idx2.p, (double*)c->sp_ek2.p);
    return c->precision ? spin_local<float>(c, nb, x, ldpsi, y, ldh, st, false, ladd)
                        : spin_local<double>(c, nb, x, ldpsi, y, ldh, st, false, ladd);
  }
  if (!c->have_pot) return fail(kNotReady, "hk_psi_loc: potential must be set");
  LocalPlan p = c->plan;
  p.accum = ladd ? 1 : 0;
  const bool f32 = c->precision != 0;
  const size_t per_band = (f32 ? sizeof(C2<float>) : sizeof(C2<double>)) * (size_t)p.nz * (size_t)p.plane;
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)nb, c->slab_budget / per_band));
  if (int s = c->slab.ensure(per_band * (size_t)chunk)) return s;
  for (int b0 = 0; b0 < nb; b0 += chunk) {
    const int nbc = std::min(chunk, nb - b0);
    cudaError_t e;
    if (f32)
      e = launch_local<float>(p, nbc, b0, x, ldpsi, y, ldh, (const int*)c->plane_start.p, (const int*)c->pw_idx.p,
                              (const int*)c->pw_pos.p, nullptr, (const float*)c->v32.p, (const C2<float>*)c->tw32[0].p,
                              (const C2<float>*)c->tw32[1].p, (const C2<float>*)c->tw32[2].p, (C2<float>*)c->slab.p,
                              st, nullptr);
    else
      e = launch_local<double>(p, nbc, b0, x, ldpsi, y, ldh, (const int*)c->plane_start.p, (const int*)c->pw_idx.p,
                               (const int*)c->pw_pos.p, nullptr, (const double*)c->v64.p,
                               (const C2<double>*)c->tw64[0].p, (const C2<double>*)c->tw64[1].p,
                               (const C2<double>*)c->tw64[2].p, (C2<double>*)c->slab.p, st, nullptr);
    if (e != cudaSuccess) return cuda_fail(e, "hk_psi_loc local kernels");
  }
  return kOk;
}

int ctx_hkpsi_spin_device(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, void* hpsi, long long ldh,
                          cudaStream_t st) {
  if (!c->have_basis || c->nsp == 0) return fail(kNotReady, "hk_psi_spin: basis and spin potential must be set");
  if (nb < 0) return fail(kBadArg, "hk_psi_spin: neig < 0");
  const long long m = c->mtxd;
  if (nb == 0 || m == 0) return kOk;
  if (ldpsi < 2 * m || ldh < 2 * m) return fail(kBadArg, "hk_psi_spin: leading dimension smaller than 2*mtxd");
  int s;
  // component views of the current basis: plane wave i -> spinor rows 2i (+1), kinetic doubled
  if ((s = c->sp_idx2.ensure((size_t)m * sizeof(int))) || (s = c->sp_ek2.ensure((size_t)2 * m * sizeof(double))))
    return s;
  k_double_index<<<592, 256, 0, st>>>((int)m, (const int*)c->pw_idx.p, (const double*)c->ekpg.p, (int*)c->sp_idx2.p,
                                      (double*)c->sp_ek2.p);
  const C2<double>* x = (const C2<double>*)psi;
  C2<double>* y = (C2<double>*)hpsi;
  s = c->precision ? spin_local<float>(c, nb, x, ldpsi, y, ldh, st) : spin_local<double>(c, nb, x, ldpsi, y, ldh, st);
  if (s) return s;
  if (c->nanl_sp > 0) {
    // KB term on the interleaved 2 mtxd rows (hk_psi_spin_c16.f90: hk_psi_nl_c16 with 2*mtxd)
    if ((s = c->proj.ensure((size_t)c->nanl_sp * nb * sizeof(C2<double>)))) return s;
    cublasSetStream(c->blas, st);
    const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
    const int m2 = (int)(2 * m);
    if (cublasZgemm(c->blas, CUBLAS_OP_C, CUBLAS_OP_N, c->nanl_sp, nb, m2, &one, (const cuDoubleComplex*)c->anl_sp.p,
                    m2, (const cuDoubleComplex*)psi, (int)ldpsi, &zero, (cuDoubleComplex*)c->proj.p,
                    c->nanl_sp) != CUBLAS_STATUS_SUCCESS)
      return fail(kCublas, "hk_psi_spin: zgemm X^H psi");
    if (cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, m2, nb, c->nanl_sp, &one, (const cuDoubleComplex*)c->anld_sp.p,
                    m2, (const cuDoubleComplex*)c->proj.p, c->nanl_sp, &one, (cuDoubleComplex*)hpsi,
                    (int)ldh) != CUBLAS_STATUS_SUCCESS)
      return fail(kCublas, "hk_psi_spin: zgemm X D P");
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? kOk : cuda_fail(e, "hk_psi_spin");
}

}  // namespace cpwb
