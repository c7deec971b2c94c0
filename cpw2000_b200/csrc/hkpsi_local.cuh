// Local part of H|psi>: G-sphere scatter, pruned inverse 3D FFT, V_loc(r)
// multiply, pruned forward 3D FFT, gather and kinetic diagonal, for a chunk
// of bands. Restates the per-band loop of Src/hk_psi/reference/hk_psi_c16.f90
// (:176-223) with the Goedecker pruning of Src/fft/_cfft/cfft_wf_c16.f
// (:110-410), re-organised for the GPU as three kernels per band chunk:
//
//   A  one CTA per (band, kept z-plane): scatter the plane's coefficients
//      into shared memory, inverse FFT along x on the 2kd2+1 kept rows,
//      inverse FFT along y on every column, write the plane to the slab W.
//   B  one CTA per (band, run of xy columns): inverse FFT along z of the
//      2kd3+1 kept planes, multiply by V(r)/N, forward FFT along z, keep the
//      2kd3+1 planes. The inverse's second pass, the multiply and the
//      forward's first pass share registers.
//   C  one CTA per (band, kept z-plane): forward FFT along y keeping the kept
//      rows, forward FFT along x, gather the sphere, add ekpg*psi.
//
// Slab W layout: [band][zi][y][x] (x fastest), zi = compact index of the
// kept z planes. Every 1D transform of length n = r1*r2 is two register
// passes with one shared-memory exchange (four-step), twiddles W_n^k from a
// table in shared memory.
#pragma once
#include <stdlib.h>

#include <map>
#include <mutex>
#include <utility>

#include "cplx.cuh"

namespace cpwb {

// Raise, never lower, the dynamic shared memory a kernel may take. Function attributes are
// process-wide: host threads that launch one kernel with different sizes (contexts of different
// k-points in flight) must not lower each other's limit between the setting and the launch.
inline cudaError_t smem_limit(const void* f, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> cur;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  size_t& v = cur[{dev, f}];
  if (bytes <= v) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) v = bytes;
  return e;
}

struct FftDim {
  int n, r1, r2;
};

// One k-point of a batch: its wavefunction blocks, its plane lists (relative to the
// batch's common kept planes and rows) and its kinetic diagonal.
struct KDesc {
  const C2<double>* psi;
  C2<double>* hpsi;
  long long ldpsi, ldh;
  const int* plane_start;
  const int* pw_idx;
  const int* pw_pos;
  const double* ekpg;     // null: no kinetic term
};

struct LocalPlan {
  // batch mode (null for one k-point): global band b of a launch is band bref[b].y of
  // k-point bref[b].x, described by kdesc[bref[b].x]; the per-call pointer arguments
  // of kernels A and C are then ignored
  const KDesc* kdesc;
  const int2* bref;
  int bgroups;            // kernel B band grouping: 0 = heuristic, else target CTAs per SM
  int n1, n2, n3;         // FFT box
  int kd1, kd2, kd3;      // sphere half-widths (largest |k_j| of the basis)
  int nx, ny, nz;         // 2*kd+1
  FftDim dx, dy, dz;
  int rowp;               // shared-memory row stride (complex elements) in A/C
  int tcol;               // columns per batch in the y passes of A/C
  int cb;                 // columns per CTA in B
  long long plane;        // n1*n2
  int accum;              // kernel C adds its result to hpsi instead of storing it (ladd)
};

__host__ __device__ __forceinline__ int kept_to_idx(int i, int kd, int n, int nk) {
  return i <= kd ? i : n - nk + i;
}
__host__ __device__ __forceinline__ int idx_to_kept(int z, int kd, int n, int nk) {
  return z <= kd ? z : (z >= n - kd ? z - (n - nk) : -1);
}

// Shared-memory footprint in bytes of kernels A/C and B.
template <typename T> inline size_t smem_planes(const LocalPlan& p) {
  return sizeof(C2<T>) * ((size_t)p.ny * p.rowp + (size_t)p.n2 * p.tcol + p.n1 + p.n2);
}
template <typename T> inline size_t smem_columns(const LocalPlan& p) {
  return sizeof(C2<T>) * ((size_t)p.n3 * p.cb + p.n3);
}
// Staged (pipelined) form of kernel B: a column tile, two kept-plane buffers, the z-twiddles
// and the potential columns; esz is the size of one complex element.
inline size_t smem_columns_pipe_bytes(size_t esz, const LocalPlan& p, int cb, int nstage = 2) {
  return esz * ((size_t)p.n3 * cb + (size_t)nstage * p.nz * cb + p.n3) + esz / 2 * (size_t)p.n3 * cb;
}
// Column tile of kernel B: 32 columns on short columns, 16 on columns of 128 points or more
// and wherever the staged form would leave room for only one CTA per SM. Measured on a
// 144^3 box (480 bands): FP64 13.7 -> 9.4 ms, FP32 8.0 -> 6.3 ms; on a 96^3 box the 16-column
// form is 13-18 % slower. CPW_B200_ZCOLS=16|32 forces the first choice. The tile is then
// halved while even the plain form does not fit.
inline int column_tile(size_t esz, const LocalPlan& p, size_t smem_block, size_t smem_sm) {
  int cb = 32;
  if (p.n3 >= 128 || 2 * (smem_columns_pipe_bytes(esz, p, cb) + 1024) > smem_sm) cb = 16;
  if (const char* v = getenv("CPW_B200_ZCOLS")) cb = atoi(v) == 16 ? 16 : 32;
  while (cb > 4 && esz * ((size_t)p.n3 * cb + p.n3) > smem_block) cb /= 2;
  return cb;
}

// Launch the three kernels for bands [band0, band0+nbc). psi/hpsi are
// complex128 column-major with leading dimensions ldpsi/ldh. W holds nbc
// slabs. ekpg may be null (no kinetic term). If ev is not null, ev[0..3] are
// recorded before A, after A, after B and after C (stage timers). Returns a
// cudaError_t.
template <typename T>
cudaError_t launch_local(const LocalPlan& p, int nbc, int band0, const C2<double>* psi, long long ldpsi,
                         C2<double>* hpsi, long long ldh, const int* plane_start, const int* pw_idx,
                         const int* pw_pos, const double* ekpg, const T* vr, const C2<T>* twx,
                         const C2<T>* twy, const C2<T>* twz, C2<T>* W, cudaStream_t st,
                         cudaEvent_t* ev = nullptr);

// Kernel A alone for bands [band0, band0+nbc): the kept z-planes of every band,
// inverse-transformed in x and y, into W (density / adjoint path).
template <typename T>
cudaError_t launch_inverse_xy(const LocalPlan& p, int nbc, int band0, const C2<double>* psi, long long ldpsi,
                              const int* plane_start, const int* pw_idx, const int* pw_pos, const C2<T>* twx,
                              const C2<T>* twy, C2<T>* W, cudaStream_t st);

}  // namespace cpwb
