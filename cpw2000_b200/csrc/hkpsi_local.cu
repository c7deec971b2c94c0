// Kernels A, B, C of the local H|psi> (see hkpsi_local.cuh for the design).
#include "hkpsi_local.cuh"

namespace cpwb {

namespace {

constexpr int kThreadsPlanes = 256;
constexpr int kThreadsCols = 256;

template <typename T> __device__ __forceinline__ C2<T> czero() { return mk<T>(T(0), T(0)); }

// ---------------------------------------------------------------------------
// A: scatter + inverse x + inverse y, one CTA per (band, kept z-plane)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreadsPlanes, 1)
k_inv_xy(LocalPlan p, int band0, const C2<double>* __restrict__ psi, long long ldpsi,
         const int* __restrict__ plane_start, const int* __restrict__ pw_idx,
         const int* __restrict__ pw_pos, const C2<T>* __restrict__ twx,
         const C2<T>* __restrict__ twy, C2<T>* __restrict__ W) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2<T>* R = reinterpret_cast<C2<T>*>(smem_raw);
  C2<T>* Tb = R + (size_t)p.ny * p.rowp;
  C2<T>* sx = Tb + (size_t)p.n2 * p.tcol;
  C2<T>* sy = sx + p.n1;
  const int zi = blockIdx.x, b = blockIdx.y;
  const int tid = threadIdx.x, nt = blockDim.x;

  for (int i = tid; i < p.n1; i += nt) sx[i] = twx[i];
  for (int i = tid; i < p.n2; i += nt) sy[i] = twy[i];
  for (int i = tid; i < p.ny * p.rowp; i += nt) R[i] = czero<T>();
  __syncthreads();

  const C2<double>* ps = psi + (size_t)(band0 + b) * ldpsi;
  const int e0 = plane_start[zi], e1 = plane_start[zi + 1];
  for (int e = e0 + tid; e < e1; e += nt) {
    const int pos = pw_pos[e];
    const C2<double> v = ps[pw_idx[e]];
    R[(pos >> 16) * p.rowp + (pos & 0xffff)] = mk<T>(T(v.x), T(v.y));
  }
  __syncthreads();

  // inverse x, pass 1: lines (row, n2), DFT_r1 over stride r2, twiddle
  {
    const int r1 = p.dx.r1, r2 = p.dx.r2;
    for (int it = tid; it < p.ny * r2; it += nt) {
      const int row = it / r2, n2 = it - row * r2;
      C2<T>* line = R + (size_t)row * p.rowp;
      radix_dispatch(r1, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<T> v[RR];
#pragma unroll
        for (int a = 0; a < RR; ++a) v[a] = line[r2 * a + n2];
        DFT<RR, +1, T>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a) line[r2 * a + n2] = cmulc<T>(v[a], sx[n2 * a]);
      });
    }
  }
  __syncthreads();
  // inverse x, pass 2: lines (row, k1), DFT_r2 over contiguous block, permuted in place
  {
    const int r1 = p.dx.r1, r2 = p.dx.r2;
    for (int it = tid; it < p.ny * r1; it += nt) {
      const int row = it / r1, k1 = it - row * r1;
      C2<T>* line = R + (size_t)row * p.rowp + r2 * k1;
      radix_dispatch(r2, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<T> v[RR];
#pragma unroll
        for (int a = 0; a < RR; ++a) v[a] = line[a];
        DFT<RR, +1, T>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a) line[a] = v[a];
      });
    }
  }
  __syncthreads();

  // inverse y on every column, in batches of tcol storage positions
  const int r1y = p.dy.r1, r2y = p.dy.r2, tc = p.tcol;
  C2<T>* Wp = W + ((size_t)b * p.nz + zi) * (size_t)p.plane;
  for (int pb = 0; pb < p.n1; pb += tc) {
    const int ncol = min(tc, p.n1 - pb);
    for (int it = tid; it < tc * r2y; it += nt) {
      const int pl = it % tc, n2 = it / tc;
      if (pl < ncol) {
        radix_dispatch(r1y, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
          C2<T> v[RR];
#pragma unroll
          for (int a = 0; a < RR; ++a) {
            const int y = r2y * a + n2;
            const int yi = idx_to_kept(y, p.kd2, p.n2, p.ny);
            v[a] = yi >= 0 ? R[(size_t)yi * p.rowp + pb + pl] : czero<T>();
          }
          DFT<RR, +1, T>::run(v);
#pragma unroll
          for (int a = 0; a < RR; ++a) Tb[(size_t)(r2y * a + n2) * tc + pl] = cmulc<T>(v[a], sy[n2 * a]);
        });
      }
    }
    __syncthreads();
    for (int it = tid; it < tc * r1y; it += nt) {
      const int pl = it % tc, k1 = it / tc;
      if (pl < ncol) {
        const int pp = pb + pl;
        const int xk1 = pp / p.dx.r2, xk2 = pp - xk1 * p.dx.r2;
        const int x = xk1 + p.dx.r1 * xk2;
        radix_dispatch(r2y, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
          C2<T> v[RR];
#pragma unroll
          for (int a = 0; a < RR; ++a) v[a] = Tb[(size_t)(r2y * k1 + a) * tc + pl];
          DFT<RR, +1, T>::run(v);
#pragma unroll
          for (int a = 0; a < RR; ++a) Wp[(size_t)(k1 + r1y * a) * p.n1 + x] = v[a];
        });
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// B: inverse z, V(r)/N, forward z, one CTA per (band, cb xy-columns)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreadsCols, 1)
k_z_vloc(LocalPlan p, const T* __restrict__ vr, const C2<T>* __restrict__ twz, C2<T>* __restrict__ W) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int cb = p.cb;
  C2<T>* Cs = reinterpret_cast<C2<T>*>(smem_raw);
  C2<T>* sz = Cs + (size_t)p.n3 * cb;
  const long long c0 = (long long)blockIdx.x * cb;
  const int b = blockIdx.y;
  const int ncol = (int)min((long long)cb, p.plane - c0);
  const int tid = threadIdx.x, nt = blockDim.x;
  const int r1 = p.dz.r1, r2 = p.dz.r2;
  C2<T>* Wb = W + (size_t)b * p.nz * (size_t)p.plane + c0;

  for (int i = tid; i < p.n3; i += nt) sz[i] = twz[i];
  for (int it = tid; it < cb * p.nz; it += nt) {
    const int cl = it % cb, zi = it / cb;
    if (cl < ncol) Cs[(size_t)kept_to_idx(zi, p.kd3, p.n3, p.nz) * cb + cl] = Wb[(size_t)zi * p.plane + cl];
  }
  __syncthreads();
  // inverse pass 1 (reads only kept planes; others are zero)
  for (int it = tid; it < cb * r2; it += nt) {
    const int cl = it % cb, n2 = it / cb;
    if (cl < ncol) {
      radix_dispatch(r1, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<T> v[RR];
#pragma unroll
        for (int a = 0; a < RR; ++a) {
          const int z = r2 * a + n2;
          v[a] = idx_to_kept(z, p.kd3, p.n3, p.nz) >= 0 ? Cs[(size_t)z * cb + cl] : czero<T>();
        }
        DFT<RR, +1, T>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a) Cs[(size_t)(r2 * a + n2) * cb + cl] = cmulc<T>(v[a], sz[n2 * a]);
      });
    }
  }
  __syncthreads();
  // inverse pass 2 -> multiply V(r)/N -> forward pass 1, in registers
  for (int it = tid; it < cb * r1; it += nt) {
    const int cl = it % cb, k1 = it / cb;
    if (cl < ncol) {
      radix_dispatch(r2, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<T> v[RR];
#pragma unroll
        for (int a = 0; a < RR; ++a) v[a] = Cs[(size_t)(r2 * k1 + a) * cb + cl];
        DFT<RR, +1, T>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a) {
          const int z = k1 + r1 * a;
          v[a] = scal<T>(v[a], vr[(size_t)z * p.plane + c0 + cl]);
        }
        DFT<RR, -1, T>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a) Cs[(size_t)(r2 * k1 + a) * cb + cl] = cmul<T>(v[a], sz[k1 * a]);
      });
    }
  }
  __syncthreads();
  // forward pass 2, keep the kept planes
  for (int it = tid; it < cb * r2; it += nt) {
    const int cl = it % cb, m2 = it / cb;
    if (cl < ncol) {
      radix_dispatch(r1, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<T> v[RR];
#pragma unroll
        for (int a = 0; a < RR; ++a) v[a] = Cs[(size_t)(r2 * a + m2) * cb + cl];
        DFT<RR, -1, T>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a) {
          const int m = m2 + r2 * a;
          const int zi = idx_to_kept(m, p.kd3, p.n3, p.nz);
          if (zi >= 0) Wb[(size_t)zi * p.plane + cl] = v[a];
        }
      });
    }
  }
}

// ---------------------------------------------------------------------------
// C: forward y + forward x + gather + kinetic, one CTA per (band, kept z-plane)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreadsPlanes, 1)
k_fwd_xy(LocalPlan p, int band0, const C2<double>* __restrict__ psi, long long ldpsi,
         C2<double>* __restrict__ hpsi, long long ldh, const int* __restrict__ plane_start,
         const int* __restrict__ pw_idx, const int* __restrict__ pw_pos,
         const double* __restrict__ ekpg, const C2<T>* __restrict__ twx,
         const C2<T>* __restrict__ twy, const C2<T>* __restrict__ W) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2<T>* R = reinterpret_cast<C2<T>*>(smem_raw);
  C2<T>* Tb = R + (size_t)p.ny * p.rowp;
  C2<T>* sx = Tb + (size_t)p.n2 * p.tcol;
  C2<T>* sy = sx + p.n1;
  const int zi = blockIdx.x, b = blockIdx.y;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < p.n1; i += nt) sx[i] = twx[i];
  for (int i = tid; i < p.n2; i += nt) sy[i] = twy[i];

  const int r1y = p.dy.r1, r2y = p.dy.r2, tc = p.tcol;
  const C2<T>* Wp = W + ((size_t)b * p.nz + zi) * (size_t)p.plane;
  for (int xb = 0; xb < p.n1; xb += tc) {
    const int ncol = min(tc, p.n1 - xb);
    for (int it = tid; it < tc * p.n2; it += nt) {
      const int xl = it % tc, y = it / tc;
      if (xl < ncol) Tb[(size_t)y * tc + xl] = Wp[(size_t)y * p.n1 + xb + xl];
    }
    __syncthreads();
    for (int it = tid; it < tc * r2y; it += nt) {
      const int xl = it % tc, n2 = it / tc;
      if (xl < ncol) {
        radix_dispatch(r1y, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
          C2<T> v[RR];
#pragma unroll
          for (int a = 0; a < RR; ++a) v[a] = Tb[(size_t)(r2y * a + n2) * tc + xl];
          DFT<RR, -1, T>::run(v);
#pragma unroll
          for (int a = 0; a < RR; ++a) Tb[(size_t)(r2y * a + n2) * tc + xl] = cmul<T>(v[a], sy[n2 * a]);
        });
      }
    }
    __syncthreads();
    for (int it = tid; it < tc * r1y; it += nt) {
      const int xl = it % tc, k1 = it / tc;
      if (xl < ncol) {
        radix_dispatch(r2y, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
          C2<T> v[RR];
#pragma unroll
          for (int a = 0; a < RR; ++a) v[a] = Tb[(size_t)(r2y * k1 + a) * tc + xl];
          DFT<RR, -1, T>::run(v);
#pragma unroll
          for (int a = 0; a < RR; ++a) {
            const int yi = idx_to_kept(k1 + r1y * a, p.kd2, p.n2, p.ny);
            if (yi >= 0) R[(size_t)yi * p.rowp + xb + xl] = v[a];
          }
        });
      }
    }
    __syncthreads();
  }

  // forward x on the kept rows
  {
    const int r1 = p.dx.r1, r2 = p.dx.r2;
    for (int it = tid; it < p.ny * r2; it += nt) {
      const int row = it / r2, n2 = it - row * r2;
      C2<T>* line = R + (size_t)row * p.rowp;
      radix_dispatch(r1, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<T> v[RR];
#pragma unroll
        for (int a = 0; a < RR; ++a) v[a] = line[r2 * a + n2];
        DFT<RR, -1, T>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a) line[r2 * a + n2] = cmul<T>(v[a], sx[n2 * a]);
      });
    }
    __syncthreads();
    for (int it = tid; it < p.ny * r1; it += nt) {
      const int row = it / r1, k1 = it - row * r1;
      C2<T>* line = R + (size_t)row * p.rowp + r2 * k1;
      radix_dispatch(r2, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<T> v[RR];
#pragma unroll
        for (int a = 0; a < RR; ++a) v[a] = line[a];
        DFT<RR, -1, T>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a) line[a] = v[a];
      });
    }
    __syncthreads();
  }

  // gather the sphere (permuted x storage) and add the kinetic diagonal
  const C2<double>* ps = psi + (size_t)(band0 + b) * ldpsi;
  C2<double>* hp = hpsi + (size_t)(band0 + b) * ldh;
  const int e0 = plane_start[zi], e1 = plane_start[zi + 1];
  const int r1x = p.dx.r1, r2x = p.dx.r2;
  for (int e = e0 + tid; e < e1; e += nt) {
    const int pos = pw_pos[e];
    const int x = pos & 0xffff, yi = pos >> 16;
    const int q = x / r1x;
    const int pp = r2x * (x - q * r1x) + q;
    const C2<T> v = R[(size_t)yi * p.rowp + pp];
    const int i = pw_idx[e];
    C2<double> out = mk<double>(double(v.x), double(v.y));
    if (ekpg) {
      const C2<double> s = ps[i];
      const double ek = ekpg[i];
      out.x += ek * s.x;
      out.y += ek * s.y;
    }
    hp[i] = out;
  }
}

}  // namespace

template <typename T>
cudaError_t launch_local(const LocalPlan& p, int nbc, int band0, const C2<double>* psi, long long ldpsi,
                         C2<double>* hpsi, long long ldh, const int* plane_start, const int* pw_idx,
                         const int* pw_pos, const double* ekpg, const T* vr, const C2<T>* twx,
                         const C2<T>* twy, const C2<T>* twz, C2<T>* W, cudaStream_t st, cudaEvent_t* ev) {
  const size_t sm_pl = smem_planes<T>(p);
  const size_t sm_co = smem_columns<T>(p);
  cudaError_t e;
  e = cudaFuncSetAttribute(k_inv_xy<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_pl);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_fwd_xy<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_pl);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_z_vloc<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_co);
  if (e != cudaSuccess) return e;
  dim3 gA(p.nz, nbc);
  if (ev) cudaEventRecord(ev[0], st);
  k_inv_xy<T><<<gA, kThreadsPlanes, sm_pl, st>>>(p, band0, psi, ldpsi, plane_start, pw_idx, pw_pos, twx, twy, W);
  if (ev) cudaEventRecord(ev[1], st);
  dim3 gB((unsigned)((p.plane + p.cb - 1) / p.cb), nbc);
  k_z_vloc<T><<<gB, kThreadsCols, sm_co, st>>>(p, vr, twz, W);
  if (ev) cudaEventRecord(ev[2], st);
  k_fwd_xy<T><<<gA, kThreadsPlanes, sm_pl, st>>>(p, band0, psi, ldpsi, hpsi, ldh, plane_start, pw_idx, pw_pos,
                                                  ekpg, twx, twy, W);
  if (ev) cudaEventRecord(ev[3], st);
  return cudaGetLastError();
}

template cudaError_t launch_local<double>(const LocalPlan&, int, int, const C2<double>*, long long, C2<double>*,
                                          long long, const int*, const int*, const int*, const double*,
                                          const double*, const C2<double>*, const C2<double>*,
                                          const C2<double>*, C2<double>*, cudaStream_t, cudaEvent_t*);
template cudaError_t launch_local<float>(const LocalPlan&, int, int, const C2<double>*, long long, C2<double>*,
                                         long long, const int*, const int*, const int*, const double*,
                                         const float*, const C2<float>*, const C2<float>*, const C2<float>*,
                                         C2<float>*, cudaStream_t, cudaEvent_t*);

}  // namespace cpwb
