// Kernel templates A, B, C of the local H|psi> (design in hkpsi_local.cuh).
//
// Template parameters fix the radix pair of each dimension (RX1*RX2 = n1,
// RY1*RY2 = n2, RZ1*RZ2 = n3) and the column batch widths TC (A/C) and CB
// (B) at compile time; 0 means "taken from the LocalPlan at run time". The
// compile-time forms get constant index arithmetic and register allocation
// sized for their own radices; the all-zero form serves any supported box.
#pragma once
#include <algorithm>

#include "hkpsi_local.cuh"

namespace cpwb {
namespace kern {

constexpr int kThreadsPlanes = 256;
constexpr int kThreadsCols = 256;
// Threads of a CTA of a two-pass (four-step) transform stage: one per line of the larger pass
// when that is 192 or 384 lines (96- and 144-point lines in 32- or 16-column tiles), so that
// no pass leaves part of the CTA idle before the barrier; else 256.
constexpr int pass_threads(int lines_a, int lines_b) {
  return (lines_a > lines_b ? lines_a : lines_b) == 384 ? 384
         : (lines_a > lines_b ? lines_a : lines_b) == 192 ? 192 : 256;
}
// CTAs per SM asked of the register allocator: two CTAs of 384 threads fit in 80 registers.
constexpr int pass_min_blocks(int nt) { return nt == 384 ? 2 : 1; }
// Kernels A and C: FP64 planes of 128 points or more take over 200 KB of shared memory (one CTA
// per SM whatever the registers), so they get no register cap.
template <typename T> constexpr int plane_min_blocks(int nt, int n1) {
  return sizeof(T) == 8 && n1 >= 128 ? 1 : pass_min_blocks(nt);
}

template <typename T> __device__ __forceinline__ C2<T> czero() { return mk<T>(T(0), T(0)); }

// ---------------------------------------------------------------------------
// A: scatter + inverse x + inverse y, one CTA per (band, kept z-plane)
// ---------------------------------------------------------------------------
template <typename T, int RX1, int RX2, int RY1, int RY2, int TC, int NT = kThreadsPlanes>
__global__ void __launch_bounds__(NT, plane_min_blocks<T>(NT, RX1 * RX2))
k_inv_xy(LocalPlan p, int band0, const C2<double>* __restrict__ psi, long long ldpsi,
         const int* __restrict__ plane_start, const int* __restrict__ pw_idx,
         const int* __restrict__ pw_pos, const C2<T>* __restrict__ twx,
         const C2<T>* __restrict__ twy, C2<T>* __restrict__ W) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tc = TC ? TC : p.tcol;
  const int r1x = RX1 ? RX1 : p.dx.r1, r2x = RX2 ? RX2 : p.dx.r2;
  const int r1y = RY1 ? RY1 : p.dy.r1, r2y = RY2 ? RY2 : p.dy.r2;
  const int n1 = RX1 ? RX1 * RX2 : p.n1, n2 = RY1 ? RY1 * RY2 : p.n2;
  const int ny = p.ny, rowp = p.rowp;
  C2<T>* R = reinterpret_cast<C2<T>*>(smem_raw);
  C2<T>* Tb = R + (size_t)ny * rowp;
  C2<T>* sx = Tb + (size_t)n2 * tc;
  C2<T>* sy = sx + n1;
  const int zi = blockIdx.x, b = blockIdx.y;
  const int tid = threadIdx.x, nt = NT;     // every launch uses NT threads

  const C2<double>* ps = psi + (size_t)(band0 + b) * ldpsi;
  if (p.kdesc) {      // batch of k-points: this band's own basis and block
    const int2 r = p.bref[band0 + b];
    const KDesc& D = p.kdesc[r.x];
    ps = D.psi + (size_t)r.y * D.ldpsi;
    plane_start = D.plane_start;
    pw_idx = D.pw_idx;
    pw_pos = D.pw_pos;
  }
  const int e0 = plane_start[zi], e1 = plane_start[zi + 1];
  // the first kPre sphere points of this thread are loaded before the plane is cleared, so
  // that their gather latency overlaps the clearing
  constexpr int kPre = 2;
  int pre_pos[kPre];
  C2<double> pre_v[kPre];
#pragma unroll
  for (int j = 0; j < kPre; ++j) {
    const int e = e0 + tid + j * nt;
    pre_pos[j] = -1;
    if (e < e1) {
      pre_pos[j] = pw_pos[e];
      pre_v[j] = ps[pw_idx[e]];
    }
  }
  for (int i = tid; i < n1; i += nt) sx[i] = twx[i];
  for (int i = tid; i < n2; i += nt) sy[i] = twy[i];
  for (int i = tid; i < ny * rowp; i += nt) R[i] = czero<T>();
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kPre; ++j)
    if (pre_pos[j] >= 0)
      R[(pre_pos[j] >> 16) * rowp + (pre_pos[j] & 0xffff)] = mk<T>(T(pre_v[j].x), T(pre_v[j].y));
  for (int e = e0 + tid + kPre * nt; e < e1; e += nt) {
    const int pos = pw_pos[e];
    const C2<double> v = ps[pw_idx[e]];
    R[(pos >> 16) * rowp + (pos & 0xffff)] = mk<T>(T(v.x), T(v.y));
  }
  __syncthreads();

  // inverse x, pass 1: lines (row, n2) with the row index fastest across lanes
  for (int it = tid; it < ny * r2x; it += nt) {
    const int row = it % ny, n2i = it / ny;
    C2<T>* line = R + (size_t)row * rowp + n2i;
    with_radix<RX1>(r1x, [&](auto rc_) {
      constexpr int RR = decltype(rc_)::value;
      C2<T> v[RR];
#pragma unroll
      for (int a = 0; a < RR; ++a) v[a] = line[r2x * a];
      DFT<RR, +1, T>::run(v);
#pragma unroll
      for (int a = 0; a < RR; ++a) line[r2x * a] = a == 0 ? v[0] : cmulc<T>(v[a], sx[n2i * a]);
    });
  }
  __syncthreads();
  // inverse x, pass 2: lines (row, k1), contiguous block of r2x, permuted in place
  for (int it = tid; it < ny * r1x; it += nt) {
    const int row = it % ny, k1 = it / ny;
    C2<T>* line = R + (size_t)row * rowp + r2x * k1;
    with_radix<RX2>(r2x, [&](auto rc_) {
      constexpr int RR = decltype(rc_)::value;
      C2<T> v[RR];
#pragma unroll
      for (int a = 0; a < RR; ++a) v[a] = line[a];
      DFT<RR, +1, T>::run(v);
#pragma unroll
      for (int a = 0; a < RR; ++a) line[a] = v[a];
    });
  }
  __syncthreads();

  // inverse y on every column, in batches of tc storage positions
  C2<T>* Wp = W + ((size_t)b * p.nz + zi) * (size_t)p.plane;
  for (int pb = 0; pb < n1; pb += tc) {
    const int ncol = min(tc, n1 - pb);
    for (int it = tid; it < tc * r2y; it += nt) {
      const int pl = it % tc, n2i = it / tc;
      if (pl < ncol) {
        with_radix<RY1>(r1y, [&](auto rc_) {
          constexpr int RR = decltype(rc_)::value;
          C2<T> v[RR];
#pragma unroll
          for (int a = 0; a < RR; ++a) {
            const int y = r2y * a + n2i;
            const int yi = idx_to_kept(y, p.kd2, n2, ny);
            v[a] = yi >= 0 ? R[(size_t)yi * rowp + pb + pl] : czero<T>();
          }
          DFT<RR, +1, T>::run(v);
#pragma unroll
          for (int a = 0; a < RR; ++a)
            Tb[(size_t)(r2y * a + n2i) * tc + pl] = a == 0 ? v[0] : cmulc<T>(v[a], sy[n2i * a]);
        });
      }
    }
    __syncthreads();
    for (int it = tid; it < tc * r1y; it += nt) {
      const int pl = it % tc, k1 = it / tc;
      if (pl < ncol) {
        const int pp = pb + pl;
        const int xk1 = pp / r2x, xk2 = pp - xk1 * r2x;
        const int x = xk1 + r1x * xk2;
        with_radix<RY2>(r2y, [&](auto rc_) {
          constexpr int RR = decltype(rc_)::value;
          C2<T> v[RR];
#pragma unroll
          for (int a = 0; a < RR; ++a) v[a] = Tb[(size_t)(r2y * k1 + a) * tc + pl];
          DFT<RR, +1, T>::run(v);
#pragma unroll
          for (int a = 0; a < RR; ++a) Wp[(size_t)(k1 + r1y * a) * n1 + x] = v[a];
        });
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// B: inverse z, V(r)/N, forward z, one CTA per (band, CB xy-columns)
// ---------------------------------------------------------------------------
template <typename T, int RZ1, int RZ2, int CB>
__global__ void __launch_bounds__(kThreadsCols, 1)
k_z_vloc(LocalPlan p, const T* __restrict__ vr, const C2<T>* __restrict__ twz, C2<T>* __restrict__ W) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int cb = CB ? CB : p.cb;
  const int r1 = RZ1 ? RZ1 : p.dz.r1, r2 = RZ2 ? RZ2 : p.dz.r2;
  const int n3 = RZ1 ? RZ1 * RZ2 : p.n3;
  C2<T>* Cs = reinterpret_cast<C2<T>*>(smem_raw);
  C2<T>* sz = Cs + (size_t)n3 * cb;
  const long long c0 = (long long)blockIdx.x * cb;
  const int b = blockIdx.y;
  const int ncol = (int)min((long long)cb, p.plane - c0);
  const int tid = threadIdx.x, nt = blockDim.x;
  C2<T>* Wb = W + (size_t)b * p.nz * (size_t)p.plane + c0;

  for (int i = tid; i < n3; i += nt) sz[i] = twz[i];
  for (int it = tid; it < cb * p.nz; it += nt) {
    const int cl = it % cb, zi = it / cb;
    if (cl < ncol) Cs[(size_t)kept_to_idx(zi, p.kd3, n3, p.nz) * cb + cl] = Wb[(size_t)zi * p.plane + cl];
  }
  __syncthreads();
  // inverse pass 1 (reads only kept planes; the others are zero)
  for (int it = tid; it < cb * r2; it += nt) {
    const int cl = it % cb, n2i = it / cb;
    if (cl < ncol) {
      with_radix<RZ1>(r1, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<T> v[RR];
#pragma unroll
        for (int a = 0; a < RR; ++a) {
          const int z = r2 * a + n2i;
          v[a] = idx_to_kept(z, p.kd3, n3, p.nz) >= 0 ? Cs[(size_t)z * cb + cl] : czero<T>();
        }
        DFT<RR, +1, T>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a)
          Cs[(size_t)(r2 * a + n2i) * cb + cl] = a == 0 ? v[0] : cmulc<T>(v[a], sz[n2i * a]);
      });
    }
  }
  __syncthreads();
  // inverse pass 2 -> multiply V(r)/N -> forward pass 1, in registers
  for (int it = tid; it < cb * r1; it += nt) {
    const int cl = it % cb, k1 = it / cb;
    if (cl < ncol) {
      with_radix<RZ2>(r2, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<T> v[RR];
        T vz[RR];
#pragma unroll
        for (int a = 0; a < RR; ++a) vz[a] = vr[(size_t)(k1 + r1 * a) * p.plane + c0 + cl];
#pragma unroll
        for (int a = 0; a < RR; ++a) v[a] = Cs[(size_t)(r2 * k1 + a) * cb + cl];
        DFT<RR, +1, T>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a) v[a] = scal<T>(v[a], vz[a]);
        DFT<RR, -1, T>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a)
          Cs[(size_t)(r2 * k1 + a) * cb + cl] = a == 0 ? v[0] : cmul<T>(v[a], sz[k1 * a]);
      });
    }
  }
  __syncthreads();
  // forward pass 2, keep the kept planes
  for (int it = tid; it < cb * r2; it += nt) {
    const int cl = it % cb, m2 = it / cb;
    if (cl < ncol) {
      with_radix<RZ1>(r1, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<T> v[RR];
#pragma unroll
        for (int a = 0; a < RR; ++a) v[a] = Cs[(size_t)(r2 * a + m2) * cb + cl];
        DFT<RR, -1, T>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a) {
          const int zi = idx_to_kept(m2 + r2 * a, p.kd3, n3, p.nz);
          if (zi >= 0) Wb[(size_t)zi * p.plane + cl] = v[a];
        }
      });
    }
  }
}


// ---------------------------------------------------------------------------
// B (pipelined): one CTA per (CB xy-columns, band group). The V(r)/N tile of
// the columns is loaded into shared memory once; the kept planes of band b+1
// stream in with cp.async while band b is transformed, so global latency
// overlaps the butterflies. Same arithmetic as k_z_vloc.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async_bytes(void* smem, const void* gmem, int bytes) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  if (bytes == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
  else if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// shared memory of k_z_vloc_pipe: work columns, two staging buffers of kept planes, twiddles, V tile
template <typename T> inline size_t smem_columns_pipe(const LocalPlan& p, int cb, int nstage = 2) {
  return smem_columns_pipe_bytes(sizeof(C2<T>), p, cb, nstage);
}

// NSTAGE: kept-plane staging buffers (2: band b+1 streams in during band b; 1: it streams in
// during the second and third pass of band b, which frees shared memory for a third CTA per SM).
// MINB: CTAs per SM asked of the register allocator (0: the pass-size default).
// TWREG: each thread keeps the z-twiddles of its own line in registers; it needs RZ1 == RZ2 and
// NT == CB * RZ1, so that every thread owns the same line index in all three passes.
// VG: V(r)/N read from global memory (L2) in the middle pass instead of a shared-memory tile.
template <typename T, int RZ1, int RZ2, int CB, int NT = kThreadsCols, int NSTAGE = 2, int MINB = 0,
          bool TWREG = false, bool VG = false>
__global__ void __launch_bounds__(NT, MINB ? MINB : pass_min_blocks(NT))
k_z_vloc_pipe(LocalPlan p, int nbc, int bands_per_group, const T* __restrict__ vr, const C2<T>* __restrict__ twz,
              C2<T>* __restrict__ W) {
  static_assert(NSTAGE == 1 || NSTAGE == 2, "one or two staging buffers");
  static_assert(!TWREG || (RZ1 == RZ2 && RZ1 > 0 && CB > 0 && NT == CB * RZ1), "register twiddles need one line per thread");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int cb = CB ? CB : p.cb;
  const int r1 = RZ1 ? RZ1 : p.dz.r1, r2 = RZ2 ? RZ2 : p.dz.r2;
  const int n3 = RZ1 ? RZ1 * RZ2 : p.n3;
  const int nz = p.nz;
  C2<T>* Cs = reinterpret_cast<C2<T>*>(smem_raw);
  C2<T>* Ws = Cs + (size_t)n3 * cb;
  C2<T>* sz = Ws + NSTAGE * (size_t)nz * cb;
  T* Vs = reinterpret_cast<T*>(sz + n3);
  const long long c0 = (long long)blockIdx.x * cb;
  const int ncol = (int)min((long long)cb, p.plane - c0);
  const int b_lo = blockIdx.y * bands_per_group;
  const int b_hi = min(nbc, b_lo + bands_per_group);
  if (b_lo >= b_hi) return;
  const int tid = threadIdx.x, nt = NT;     // every launch uses NT threads

  auto stage = [&](int b, int buf) {
    const C2<T>* Wb = W + (size_t)b * nz * (size_t)p.plane + c0;
    C2<T>* dst = Ws + (size_t)buf * nz * cb;
    for (int it = tid; it < cb * nz; it += nt) {
      const int cl = it % cb, zi = it / cb;
      if (cl < ncol) cp_async_bytes(dst + (size_t)zi * cb + cl, Wb + (size_t)zi * p.plane + cl, (int)sizeof(C2<T>));
    }
  };
  for (int i = tid; i < n3; i += nt) sz[i] = twz[i];
  if (!VG) {
    for (int it = tid; it < cb * n3; it += nt) {
      const int cl = it % cb, z = it / cb;
      if (cl < ncol) cp_async_bytes(Vs + (size_t)z * cb + cl, vr + (size_t)z * p.plane + c0 + cl, (int)sizeof(T));
    }
  }
  stage(b_lo, 0);
  cp_async_commit();
  if (NSTAGE == 2) {
    if (b_lo + 1 < b_hi) stage(b_lo + 1, 1);
    cp_async_commit();
  }
  // register twiddles: the thread's line index is tid / CB in every pass (n2i of pass 1, k1 of
  // pass 2); W^(j a) for a = 1 .. R-1 (read once the twiddle table has been written)
  C2<T> twr[TWREG ? RZ1 : 1];
  bool tw_loaded = !TWREG;
  // one pass-1 / pass-3 line per thread (line index j = tid / CB in both): the kept-plane index
  // of each of its points z = RZ2 a + j, fixed for all bands, is computed once (FP32: the FP64
  // form has no registers to spare for it under its 3-CTA bound)
  constexpr bool kOneLine = sizeof(T) == 4 && CB > 0 && RZ1 > 0 && RZ2 > 0 && NT == CB * RZ2;
  int zk[kOneLine ? RZ1 : 1];
  if constexpr (kOneLine) {
#pragma unroll
    for (int a = 0; a < RZ1; ++a) zk[a] = idx_to_kept(RZ2 * a + tid / CB, p.kd3, n3, nz);
  }

  for (int b = b_lo; b < b_hi; ++b) {
    const int buf = NSTAGE == 2 ? (b - b_lo) & 1 : 0;
    if (NSTAGE == 2)
      cp_async_wait<1>();     // every group but the newest (band b+1) has landed
    else
      cp_async_wait<0>();     // band b has landed
    __syncthreads();
    if (TWREG && !tw_loaded) {
      const int j = tid / (CB ? CB : 1);
#pragma unroll
      for (int a = 0; a < (TWREG ? RZ1 : 1); ++a) twr[a] = sz[(j * a) % n3];
      tw_loaded = true;
    }
    const C2<T>* Wsb = Ws + (size_t)buf * nz * cb;
    // inverse pass 1 straight from the staged kept planes
    for (int it = tid; it < cb * r2; it += nt) {
      const int cl = it % cb, n2i = it / cb;
      if (cl < ncol) {
        with_radix<RZ1>(r1, [&](auto rc_) {
          constexpr int RR = decltype(rc_)::value;
          C2<T> v[RR];
#pragma unroll
          for (int a = 0; a < RR; ++a) {
            int zi;
            if constexpr (kOneLine)
              zi = zk[a];
            else
              zi = idx_to_kept(r2 * a + n2i, p.kd3, n3, nz);
            v[a] = zi >= 0 ? Wsb[(size_t)zi * cb + cl] : czero<T>();
          }
          DFT<RR, +1, T>::run(v);
#pragma unroll
          for (int a = 0; a < RR; ++a) {
            if constexpr (TWREG)
              Cs[(size_t)(r2 * a + n2i) * cb + cl] = a == 0 ? v[0] : cmulc<T>(v[a], twr[a]);
            else
              Cs[(size_t)(r2 * a + n2i) * cb + cl] = a == 0 ? v[0] : cmulc<T>(v[a], sz[n2i * a]);
          }
        });
      }
    }
    __syncthreads();
    // the staging buffer of band b is free: prefetch band b+2 (two buffers) or b+1 (one) into it
    if (b + NSTAGE < b_hi) stage(b + NSTAGE, buf);
    cp_async_commit();
    // inverse pass 2 -> V/N -> forward pass 1, in registers
    for (int it = tid; it < cb * r1; it += nt) {
      const int cl = it % cb, k1 = it / cb;
      if (cl < ncol) {
        with_radix<RZ2>(r2, [&](auto rc_) {
          constexpr int RR = decltype(rc_)::value;
          C2<T> v[RR];
          T vz[VG ? RR : 1];
          if constexpr (VG) {
#pragma unroll
            for (int a = 0; a < RR; ++a) vz[a] = __ldg(vr + (size_t)(k1 + r1 * a) * p.plane + c0 + cl);
          }
#pragma unroll
          for (int a = 0; a < RR; ++a) v[a] = Cs[(size_t)(r2 * k1 + a) * cb + cl];
          DFT<RR, +1, T>::run(v);
#pragma unroll
          for (int a = 0; a < RR; ++a) {
            if constexpr (VG)
              v[a] = scal<T>(v[a], vz[a]);
            else
              v[a] = scal<T>(v[a], Vs[(size_t)(k1 + r1 * a) * cb + cl]);
          }
          DFT<RR, -1, T>::run(v);
#pragma unroll
          for (int a = 0; a < RR; ++a) {
            if constexpr (TWREG)
              Cs[(size_t)(r2 * k1 + a) * cb + cl] = a == 0 ? v[0] : cmul<T>(v[a], twr[a]);
            else
              Cs[(size_t)(r2 * k1 + a) * cb + cl] = a == 0 ? v[0] : cmul<T>(v[a], sz[k1 * a]);
          }
        });
      }
    }
    __syncthreads();
    // forward pass 2, kept planes back to the slab
    C2<T>* Wb = W + (size_t)b * nz * (size_t)p.plane + c0;
    for (int it = tid; it < cb * r2; it += nt) {
      const int cl = it % cb, m2 = it / cb;
      if (cl < ncol) {
        with_radix<RZ1>(r1, [&](auto rc_) {
          constexpr int RR = decltype(rc_)::value;
          C2<T> v[RR];
#pragma unroll
          for (int a = 0; a < RR; ++a) v[a] = Cs[(size_t)(r2 * a + m2) * cb + cl];
          DFT<RR, -1, T>::run(v);
#pragma unroll
          for (int a = 0; a < RR; ++a) {
            int zi;
            if constexpr (kOneLine)
              zi = zk[a];
            else
              zi = idx_to_kept(m2 + r2 * a, p.kd3, n3, nz);
            if (zi >= 0) Wb[(size_t)zi * p.plane + cl] = v[a];
          }
        });
      }
    }
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// C: forward y + forward x + gather + kinetic, one CTA per (band, kept z-plane)
// ---------------------------------------------------------------------------
template <typename T, int RX1, int RX2, int RY1, int RY2, int TC, int NT = kThreadsPlanes>
__global__ void __launch_bounds__(NT, plane_min_blocks<T>(NT, RX1 * RX2))
k_fwd_xy(LocalPlan p, int band0, const C2<double>* __restrict__ psi, long long ldpsi,
         C2<double>* __restrict__ hpsi, long long ldh, const int* __restrict__ plane_start,
         const int* __restrict__ pw_idx, const int* __restrict__ pw_pos,
         const double* __restrict__ ekpg, const C2<T>* __restrict__ twx,
         const C2<T>* __restrict__ twy, const C2<T>* __restrict__ W) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tc = TC ? TC : p.tcol;
  const int r1x = RX1 ? RX1 : p.dx.r1, r2x = RX2 ? RX2 : p.dx.r2;
  const int r1y = RY1 ? RY1 : p.dy.r1, r2y = RY2 ? RY2 : p.dy.r2;
  const int n1 = RX1 ? RX1 * RX2 : p.n1, n2 = RY1 ? RY1 * RY2 : p.n2;
  const int ny = p.ny, rowp = p.rowp;
  C2<T>* R = reinterpret_cast<C2<T>*>(smem_raw);
  C2<T>* Tb = R + (size_t)ny * rowp;
  C2<T>* sx = Tb + (size_t)n2 * tc;
  C2<T>* sy = sx + n1;
  const int zi = blockIdx.x, b = blockIdx.y;
  const int tid = threadIdx.x, nt = NT;     // every launch uses NT threads
  for (int i = tid; i < n1; i += nt) sx[i] = twx[i];
  for (int i = tid; i < n2; i += nt) sy[i] = twy[i];
  const C2<double>* ps = psi + (size_t)(band0 + b) * ldpsi;
  C2<double>* hp = hpsi + (size_t)(band0 + b) * ldh;
  if (p.kdesc) {      // batch of k-points: this band's own basis and block
    const int2 r = p.bref[band0 + b];
    const KDesc& D = p.kdesc[r.x];
    ps = D.psi + (size_t)r.y * D.ldpsi;
    hp = D.hpsi + (size_t)r.y * D.ldh;
    plane_start = D.plane_start;
    pw_idx = D.pw_idx;
    pw_pos = D.pw_pos;
    ekpg = D.ekpg;
  }
  const int e0 = plane_start[zi], e1 = plane_start[zi + 1];

  const C2<T>* Wp = W + ((size_t)b * p.nz + zi) * (size_t)p.plane;
  for (int xb = 0; xb < n1; xb += tc) {
    const int ncol = min(tc, n1 - xb);
    // the tile's columns of every y row, all copies in flight at once
    for (int it = tid; it < tc * n2; it += nt) {
      const int xl = it % tc, y = it / tc;
      if (xl < ncol) cp_async_bytes(Tb + (size_t)y * tc + xl, Wp + (size_t)y * n1 + xb + xl, (int)sizeof(C2<T>));
    }
    cp_async_commit();
    if (sizeof(T) == 8 && xb == 0 && ekpg) {
      // while the first tile lands: bring the psi values and kinetic terms of the final gather
      // into L2, so that its dependent loads do not wait on HBM at the end of the CTA (FP64
      // only: in FP32 the extra registers cost a CTA per SM on 96-point lines)
      for (int e = e0 + tid; e < e1; e += nt) {
        const int i = pw_idx[e];
        asm volatile("prefetch.global.L2 [%0];" ::"l"(ps + i));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(ekpg + i));
      }
    }
    cp_async_wait<0>();
    __syncthreads();
    for (int it = tid; it < tc * r2y; it += nt) {
      const int xl = it % tc, n2i = it / tc;
      if (xl < ncol) {
        with_radix<RY1>(r1y, [&](auto rc_) {
          constexpr int RR = decltype(rc_)::value;
          C2<T> v[RR];
#pragma unroll
          for (int a = 0; a < RR; ++a) v[a] = Tb[(size_t)(r2y * a + n2i) * tc + xl];
          DFT<RR, -1, T>::run(v);
#pragma unroll
          for (int a = 0; a < RR; ++a)
            Tb[(size_t)(r2y * a + n2i) * tc + xl] = a == 0 ? v[0] : cmul<T>(v[a], sy[n2i * a]);
        });
      }
    }
    __syncthreads();
    for (int it = tid; it < tc * r1y; it += nt) {
      const int xl = it % tc, k1 = it / tc;
      if (xl < ncol) {
        with_radix<RY2>(r2y, [&](auto rc_) {
          constexpr int RR = decltype(rc_)::value;
          C2<T> v[RR];
#pragma unroll
          for (int a = 0; a < RR; ++a) v[a] = Tb[(size_t)(r2y * k1 + a) * tc + xl];
          DFT<RR, -1, T>::run(v);
#pragma unroll
          for (int a = 0; a < RR; ++a) {
            const int yi = idx_to_kept(k1 + r1y * a, p.kd2, n2, ny);
            if (yi >= 0) R[(size_t)yi * rowp + xb + xl] = v[a];
          }
        });
      }
    }
    __syncthreads();
  }

  // forward x on the kept rows (row index fastest across lanes)
  for (int it = tid; it < ny * r2x; it += nt) {
    const int row = it % ny, n2i = it / ny;
    C2<T>* line = R + (size_t)row * rowp + n2i;
    with_radix<RX1>(r1x, [&](auto rc_) {
      constexpr int RR = decltype(rc_)::value;
      C2<T> v[RR];
#pragma unroll
      for (int a = 0; a < RR; ++a) v[a] = line[r2x * a];
      DFT<RR, -1, T>::run(v);
#pragma unroll
      for (int a = 0; a < RR; ++a) line[r2x * a] = a == 0 ? v[0] : cmul<T>(v[a], sx[n2i * a]);
    });
  }
  __syncthreads();
  for (int it = tid; it < ny * r1x; it += nt) {
    const int row = it % ny, k1 = it / ny;
    C2<T>* line = R + (size_t)row * rowp + r2x * k1;
    with_radix<RX2>(r2x, [&](auto rc_) {
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

  // gather the sphere (permuted x storage) and add the kinetic diagonal
  for (int e = e0 + tid; e < e1; e += nt) {
    const int pos = pw_pos[e];
    const int x = pos & 0xffff, yi = pos >> 16;
    const int q = x / r1x;
    const int pp = r2x * (x - q * r1x) + q;
    const C2<T> v = R[(size_t)yi * rowp + pp];
    const int i = pw_idx[e];
    C2<double> out = mk<double>(double(v.x), double(v.y));
    if (ekpg) {
      const C2<double> s = ps[i];
      const double ek = ekpg[i];
      out.x += ek * s.x;
      out.y += ek * s.y;
    }
    if (p.accum) {
      const C2<double> h0 = hp[i];
      out.x += h0.x;
      out.y += h0.y;
    }
    hp[i] = out;
  }
}

// Launch A, B, C for one band chunk with one compile-time configuration.
template <typename T, int RX1, int RX2, int RY1, int RY2, int RZ1, int RZ2, int TC, int CB>
cudaError_t launch_impl(const LocalPlan& p, int nbc, int band0, const C2<double>* psi, long long ldpsi,
                        C2<double>* hpsi, long long ldh, const int* plane_start, const int* pw_idx,
                        const int* pw_pos, const double* ekpg, const T* vr, const C2<T>* twx, const C2<T>* twy,
                        const C2<T>* twz, C2<T>* W, cudaStream_t st, cudaEvent_t* ev) {
  constexpr int NTP = TC && RY1 ? pass_threads(TC * RY2, TC * RY1) : kThreadsPlanes;
  constexpr int NTZ = CB && RZ1 ? pass_threads(CB * RZ2, CB * RZ1) : kThreadsCols;
  // C keeps 256 threads where 384 measured slower: FP32 on 96-point lines.
  constexpr bool c_wide = sizeof(T) == 8 || RY1 * RY2 >= 128;
  constexpr int NTC = NTP == 384 && c_wide ? 384 : kThreadsPlanes;
  const size_t sm_pl = smem_planes<T>(p);
  auto* ka = k_inv_xy<T, RX1, RX2, RY1, RY2, TC, NTP>;
  auto* kc = k_fwd_xy<T, RX1, RX2, RY1, RY2, TC, NTC>;
  cudaError_t e;
  if ((e = smem_limit((const void*)ka, (size_t)sm_pl)) != cudaSuccess) return e;
  if ((e = smem_limit((const void*)kc, (size_t)sm_pl)) != cudaSuccess) return e;
  int nsm = 148, dev = 0, smax = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  dim3 gA(p.nz, nbc);
  if (ev) cudaEventRecord(ev[0], st);
  ka<<<gA, NTP, sm_pl, st>>>(p, band0, psi, ldpsi, plane_start, pw_idx, pw_pos, twx, twy, W);
  if (ev) cudaEventRecord(ev[1], st);
  // kernel B form on boxes whose z split is square (one line per thread in every pass):
  // CPW_B200_ZB_VARIANT 1 = one staging buffer + 3 CTAs per SM (the default there: on the 144^3
  // box, 480 bands, FP64 B 8.58 -> 7.17 ms, FP32 5.38 -> 5.32 ms, identical results),
  // 2 = register twiddles (FP32 6.49 ms), 3 = both, 4 = one staging buffer, V(r)/N from L2 and 4
  // CTAs per SM, 5 = the same with 3 CTAs; 0 = two staging buffers, twiddles in shared memory (the
  // only form elsewhere)
  int zv = 0;
  if constexpr (RZ1 == RZ2 && RZ1 > 0 && CB > 0 && NTZ == CB * RZ1) {
    zv = 1;
    if (const char* v = getenv("CPW_B200_ZB_VARIANT")) zv = std::max(0, std::min(5, atoi(v)));
  }
  size_t sm_pipe = smem_columns_pipe<T>(p, p.cb, zv == 1 || zv >= 3 ? 1 : 2);
  if (zv >= 4) sm_pipe -= sizeof(T) * (size_t)p.n3 * p.cb;     // no V tile
  const long long tiles = (p.plane + p.cb - 1) / p.cb;
  if (sm_pipe > (size_t)smax) {
    // the staged form does not fit: one CTA per (band, column tile)
    const size_t sm_co = smem_columns<T>(p);
    auto* kb = k_z_vloc<T, RZ1, RZ2, CB>;
    if ((e = smem_limit((const void*)kb, (size_t)sm_co)) != cudaSuccess) return e;
    kb<<<dim3((unsigned)tiles, nbc), kThreadsCols, sm_co, st>>>(p, vr, twz, W);
  } else {
    // column tiles x band groups: enough CTAs for two per SM on small boxes
    const long long per_sm = p.bgroups > 0 ? p.bgroups : 2;
    long long groups = std::max(1LL, std::min((long long)nbc, (per_sm * nsm + tiles - 1) / tiles));
    const int per = (int)((nbc + groups - 1) / groups);
    groups = (nbc + per - 1) / per;
    auto* kbp = k_z_vloc_pipe<T, RZ1, RZ2, CB, NTZ>;
    if constexpr (RZ1 == RZ2 && RZ1 > 0 && CB > 0 && NTZ == CB * RZ1) {
      if (zv == 1) kbp = k_z_vloc_pipe<T, RZ1, RZ2, CB, NTZ, 1, 3, false>;
      if (zv == 2) kbp = k_z_vloc_pipe<T, RZ1, RZ2, CB, NTZ, 2, 0, true>;
      if (zv == 3) kbp = k_z_vloc_pipe<T, RZ1, RZ2, CB, NTZ, 1, 3, true>;
      if (zv == 4) kbp = k_z_vloc_pipe<T, RZ1, RZ2, CB, NTZ, 1, 4, false, true>;
      if (zv == 5) kbp = k_z_vloc_pipe<T, RZ1, RZ2, CB, NTZ, 1, 3, false, true>;
    }
    if ((e = smem_limit((const void*)kbp, (size_t)sm_pipe)) != cudaSuccess)
      return e;
    kbp<<<dim3((unsigned)tiles, (unsigned)groups), NTZ, sm_pipe, st>>>(p, nbc, per, vr, twz, W);
  }
  if (ev) cudaEventRecord(ev[2], st);
  kc<<<gA, NTC, sm_pl, st>>>(p, band0, psi, ldpsi, hpsi, ldh, plane_start, pw_idx, pw_pos, ekpg, twx, twy, W);
  if (ev) cudaEventRecord(ev[3], st);
  return cudaGetLastError();
}

// Launch kernel A alone (scatter + inverse x + inverse y into the slab W).
template <typename T, int RX1, int RX2, int RY1, int RY2, int TC>
cudaError_t launch_inv_impl(const LocalPlan& p, int nbc, int band0, const C2<double>* psi, long long ldpsi,
                            const int* plane_start, const int* pw_idx, const int* pw_pos, const C2<T>* twx,
                            const C2<T>* twy, C2<T>* W, cudaStream_t st) {
  constexpr int NTP = TC && RY1 ? pass_threads(TC * RY2, TC * RY1) : kThreadsPlanes;
  const size_t sm_pl = smem_planes<T>(p);
  auto* ka = k_inv_xy<T, RX1, RX2, RY1, RY2, TC, NTP>;
  cudaError_t e = smem_limit((const void*)ka, (size_t)sm_pl);
  if (e != cudaSuccess) return e;
  ka<<<dim3(p.nz, nbc), NTP, sm_pl, st>>>(p, band0, psi, ldpsi, plane_start, pw_idx, pw_pos, twx, twy, W);
  return cudaGetLastError();
}

}  // namespace kern

#define CPWB_INV_ARGS(T)                                                                                     \
  const LocalPlan &p, int nbc, int band0, const C2<double>*psi, long long ldpsi, const int *plane_start,     \
      const int *pw_idx, const int *pw_pos, const C2<T>*twx, const C2<T>*twy, C2<T>*W, cudaStream_t st

#define CPWB_LAUNCH_ARGS(T)                                                                                  \
  const LocalPlan &p, int nbc, int band0, const C2<double>*psi, long long ldpsi, C2<double>*hpsi,            \
      long long ldh, const int *plane_start, const int *pw_idx, const int *pw_pos, const double *ekpg,       \
      const T *vr, const C2<T>*twx, const C2<T>*twy, const C2<T>*twz, C2<T>*W, cudaStream_t st,             \
      cudaEvent_t *ev

#define CPWB_INSTANTIATE(T, RX1, RX2, RY1, RY2, RZ1, RZ2, TC, CB)                                        \
  template cudaError_t kern::launch_impl<T, RX1, RX2, RY1, RY2, RZ1, RZ2, TC, CB>(CPWB_LAUNCH_ARGS(T)); \
  template cudaError_t kern::launch_inv_impl<T, RX1, RX2, RY1, RY2, TC>(CPWB_INV_ARGS(T));

}  // namespace cpwb
