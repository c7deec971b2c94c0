// Allocation-free variant of the local H|psi> (V_loc psi [+ ekpg psi]).
//
// Who needs it: callers that cannot call cudaMalloc -- code that runs under a
// caller-owned memory pool or a fixed device-memory budget, and host codes that
// hand this library device buffers they already own and forbid it to grow the
// device heap. Every buffer such a caller passes is its own; the work space
// this operation needs (the FFT slab of a band chunk, the plane lists of the
// basis, the twiddle tables and the repacked potential) lives in one
// file-scope __device__ array of fixed size, so this entry point calls no
// cudaMalloc, cudaFree or allocating library routine.
//
// Each call reads the sphere extent of the basis back to the host (12 bytes)
// before it sizes the FFT planes, so it returns only after the work queued
// earlier on its stream and that reduction have finished.
//
// The array costs kNoAllocScratchBytes of device memory on every GPU that
// loads this library, for the life of the process. Every call shares it and
// it keeps the previous call's contents: the parts that must start at zero
// (plane counters) are cleared by each call, everything else is written before
// it is read. Calls that overlap on the GPU (different streams, or several
// host threads) race on the array and must be serialised by the caller.
//
// The first call on a device resolves the array's device address with
// cudaGetSymbolAddress while that device is current; make that first call
// before any stream capture. The address is kept for the life of the process:
// do not use this entry point on a device after cudaDeviceReset.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/cpw_b200.h"
#include "context.hpp"

namespace cpwb {
namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)CPW_B200_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;
constexpr int kMaxN = 4096;  // largest FFT length this entry point accepts per direction

// The scratch array. In host code `g_noalloc_scratch` is only a host-side stand-in
// for the symbol; its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_sym_mu;
void* g_sym_addr[kMaxDevices] = {nullptr};

int scratch_address(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) return fail(kBadArg, "hk_psi_loc_noalloc: device index out of range");
  std::lock_guard<std::mutex> lk(g_sym_mu);
  if (!g_sym_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return cuda_fail(e, "hk_psi_loc_noalloc: cudaGetSymbolAddress");
    g_sym_addr[dev] = p;
  }
  *out = (unsigned char*)g_sym_addr[dev];
  return kOk;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

bool split2(int n, FftDim& d) {
  int best = -1;
  for (int r1 = 1; r1 <= 16; ++r1) {
    if (n % r1) continue;
    const int r2 = n / r1;
    if (radix_ok(r1) && radix_ok(r2) && r1 <= r2) best = r1;
  }
  if (best < 0) return false;
  d.n = n;
  d.r1 = best;
  d.r2 = n / best;
  return true;
}

// ---- set-up kernels, all writing into the scratch array ----

__global__ void k_na_extent(int mtxd, const int* __restrict__ kgvb, int* __restrict__ kd) {
  int m0 = 0, m1 = 0, m2 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < mtxd; i += gridDim.x * blockDim.x) {
    m0 = max(m0, abs(kgvb[3 * i]));
    m1 = max(m1, abs(kgvb[3 * i + 1]));
    m2 = max(m2, abs(kgvb[3 * i + 2]));
  }
  atomicMax(&kd[0], m0);
  atomicMax(&kd[1], m1);
  atomicMax(&kd[2], m2);
}

__device__ __forceinline__ int wrap(int k, int n) { return k < 0 ? k + n : k; }

__global__ void k_na_count(LocalPlan p, int mtxd, const int* __restrict__ kgvb, int* __restrict__ counts) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < mtxd; i += gridDim.x * blockDim.x) {
    const int zi = idx_to_kept(wrap(kgvb[3 * i + 2], p.n3), p.kd3, p.n3, p.nz);
    atomicAdd(&counts[zi], 1);
  }
}

// one block: exclusive scan of counts[nz] into start[nz+1], cursor = start
__global__ void k_na_scan(int nz, const int* __restrict__ counts, int* __restrict__ start, int* __restrict__ cursor) {
  if (threadIdx.x == 0) {
    int s = 0;
    for (int z = 0; z < nz; ++z) {
      start[z] = s;
      cursor[z] = s;
      s += counts[z];
    }
    start[nz] = s;
  }
}

__global__ void k_na_fill(LocalPlan p, int mtxd, const int* __restrict__ kgvb, int* __restrict__ cursor,
                          int* __restrict__ pw_idx, int* __restrict__ pw_pos) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < mtxd; i += gridDim.x * blockDim.x) {
    const int k1 = wrap(kgvb[3 * i], p.n1), k2 = wrap(kgvb[3 * i + 1], p.n2), k3 = wrap(kgvb[3 * i + 2], p.n3);
    const int zi = idx_to_kept(k3, p.kd3, p.n3, p.nz);
    const int yi = idx_to_kept(k2, p.kd2, p.n2, p.ny);
    const int e = atomicAdd(&cursor[zi], 1);
    pw_idx[e] = i;
    pw_pos[e] = (yi << 16) | k1;
  }
}

// W_n^k = exp(-2 pi i k / n)
__global__ void k_na_twiddles(int n, C2<double>* __restrict__ tw) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)k / (double)n, &s, &c);
    tw[k] = mk<double>(c, -s);
  }
}

// vscr(id, n2, n3) -> [z][y][x] scaled by 1/(n1 n2 n3)
__global__ void k_na_potential(LocalPlan p, int ident, const double* __restrict__ vscr, double* __restrict__ v) {
  const long long n = (long long)p.n1 * p.n2 * p.n3;
  const double inv = 1.0 / (double)n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long x = t % p.n1, r = t / p.n1;
    const long long y = r % p.n2, z = r / p.n2;
    v[t] = vscr[(z * p.n2 + y) * ident + x] * inv;
  }
}

}  // namespace
}  // namespace cpwb

using namespace cpwb;

extern "C" int cpw_b200_hk_psi_loc_noalloc(int mtxd, int neig, const void* psi, long long ldpsi, void* hpsi,
                                           long long ldhpsi, const int* kgvb, const double* ekpg,
                                           const double* vscr, const int* kmscr, void* stream) {
  if (mtxd < 1 || neig < 0) return fail(kBadArg, "hk_psi_loc_noalloc: mtxd must be >= 1 and neig >= 0");
  if (ldpsi < mtxd || ldhpsi < mtxd) return fail(kBadArg, "hk_psi_loc_noalloc: leading dimension smaller than mtxd");
  if (!psi || !hpsi || !kgvb || !vscr || !kmscr) return fail(kBadArg, "hk_psi_loc_noalloc: null pointer argument");
  if (neig == 0) return kOk;
  const int n1 = kmscr[3], n2 = kmscr[4], n3 = kmscr[5], ident = kmscr[6];
  if (n1 < 2 || n2 < 2 || n3 < 2 || ident < n1) return fail(kBadArg, "hk_psi_loc_noalloc: bad FFT box in kmscr(4:7)");
  if (n1 > kMaxN || n2 > kMaxN || n3 > kMaxN)
    return fail(kUnsupported, "hk_psi_loc_noalloc: FFT dimension above 4096");
  LocalPlan p{};
  p.n1 = n1; p.n2 = n2; p.n3 = n3;
  if (!split2(n1, p.dx) || !split2(n2, p.dy) || !split2(n3, p.dz))
    return fail(kUnsupported, "hk_psi_loc_noalloc: FFT length is not a product of two supported radices");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "hk_psi_loc_noalloc: cudaGetDevice");
  unsigned char* base = nullptr;
  if (int s = scratch_address(dev, &base)) return s;
  cudaStream_t st = (cudaStream_t)stream;

  // scratch layout: [ints: kd(3) | counts(n3) | cursor(n3) | start(n3+1)] [pw_idx] [pw_pos] [twiddles] [V] [slab]
  const size_t off_int = 0;
  const size_t int_bytes = align256(sizeof(int) * (3 + 3 * (size_t)n3 + 1));
  const size_t off_idx = off_int + int_bytes;
  const size_t off_pos = off_idx + align256(sizeof(int) * (size_t)mtxd);
  const size_t off_tw = off_pos + align256(sizeof(int) * (size_t)mtxd);
  const size_t off_v = off_tw + align256(sizeof(C2<double>) * ((size_t)n1 + n2 + n3));
  const size_t off_slab = off_v + align256(sizeof(double) * (size_t)n1 * n2 * n3);
  if (off_slab > kNoAllocScratchBytes) {
    char buf[200];
    snprintf(buf, sizeof buf,
             "hk_psi_loc_noalloc: basis %d and box %dx%dx%d need %zu bytes of set-up scratch, above the %zu-byte maximum",
             mtxd, n1, n2, n3, off_slab, kNoAllocScratchBytes);
    return fail(kBadArg, buf);
  }
  int* kd = (int*)(base + off_int);
  int* counts = kd + 3;
  int* cursor = counts + n3;
  int* start = cursor + n3;
  int* pw_idx = (int*)(base + off_idx);
  int* pw_pos = (int*)(base + off_pos);
  C2<double>* tw = (C2<double>*)(base + off_tw);
  double* v = (double*)(base + off_v);
  C2<double>* slab = (C2<double>*)(base + off_slab);

  // sphere extent (hk_psi_c16.f90:145-158) and wraparound check (:161-172)
  if ((e = cudaMemsetAsync(kd, 0, int_bytes, st)) != cudaSuccess) return cuda_fail(e, "hk_psi_loc_noalloc: memset");
  const int nblk = (int)std::min<long long>(1184, (mtxd + 255) / 256);
  k_na_extent<<<nblk, 256, 0, st>>>(mtxd, kgvb, kd);
  int kdh[3] = {0, 0, 0};
  if ((e = cudaMemcpyAsync(kdh, kd, sizeof kdh, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return cuda_fail(e, "hk_psi_loc_noalloc: extent copy");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "hk_psi_loc_noalloc: extent");
  if (kdh[0] > (n1 - 1) / 2 || kdh[1] > (n2 - 1) / 2 || kdh[2] > (n3 - 1) / 2) {
    char buf[200];
    snprintf(buf, sizeof buf, "hk_psi_loc_noalloc: dimension of k index= %d %d %d exceeds %d %d %d", kdh[0], kdh[1],
             kdh[2], (n1 - 1) / 2, (n2 - 1) / 2, (n3 - 1) / 2);
    return fail(kWrap, buf);
  }
  p.kd1 = kdh[0]; p.kd2 = kdh[1]; p.kd3 = kdh[2];
  p.nx = 2 * kdh[0] + 1; p.ny = 2 * kdh[1] + 1; p.nz = 2 * kdh[2] + 1;
  p.plane = (long long)n1 * n2;
  p.rowp = n1 + 1;
  int smax = 0;
  cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const size_t es = sizeof(C2<double>);
  p.tcol = 32;
  while (p.tcol > 4 && es * ((size_t)p.ny * p.rowp + (size_t)n2 * p.tcol + n1 + n2) > (size_t)smax) p.tcol /= 2;
  if (es * ((size_t)p.ny * p.rowp + (size_t)n2 * p.tcol + n1 + n2) > (size_t)smax)
    return fail(kUnsupported, "hk_psi_loc_noalloc: plane does not fit in shared memory");
  int smsm = 0;
  cudaDeviceGetAttribute(&smsm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  p.cb = column_tile(es, p, (size_t)smax, (size_t)smsm);

  const size_t per_band = es * (size_t)p.nz * (size_t)p.plane;
  const size_t room = kNoAllocScratchBytes - off_slab;
  if (room < per_band) {
    char buf[200];
    snprintf(buf, sizeof buf,
             "hk_psi_loc_noalloc: one band needs %zu bytes of FFT slab, only %zu of the %zu-byte scratch are left",
             per_band, room, kNoAllocScratchBytes);
    return fail(kBadArg, buf);
  }
  // bands per chunk: what fits in the rest of the array, and at most the 65535 blocks a grid's y
  // dimension takes (kernels A and C launch one block row per band)
  const int chunk = (int)std::min<size_t>(std::min<size_t>((size_t)neig, room / per_band), 65535);

  // plane lists, twiddles and the repacked potential, all in the scratch array
  k_na_count<<<nblk, 256, 0, st>>>(p, mtxd, kgvb, counts);
  k_na_scan<<<1, 32, 0, st>>>(p.nz, counts, start, cursor);
  k_na_fill<<<nblk, 256, 0, st>>>(p, mtxd, kgvb, cursor, pw_idx, pw_pos);
  k_na_twiddles<<<1, 256, 0, st>>>(n1, tw);
  k_na_twiddles<<<1, 256, 0, st>>>(n2, tw + n1);
  k_na_twiddles<<<1, 256, 0, st>>>(n3, tw + n1 + n2);
  k_na_potential<<<1184, 256, 0, st>>>(p, ident, vscr, v);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "hk_psi_loc_noalloc: set-up kernels");

  for (int b0 = 0; b0 < neig; b0 += chunk) {
    const int nbc = std::min(chunk, neig - b0);
    e = launch_local<double>(p, nbc, b0, (const C2<double>*)psi, ldpsi, (C2<double>*)hpsi, ldhpsi, start, pw_idx,
                             pw_pos, ekpg, v, tw, tw + n1, tw + n1 + n2, slab, st, nullptr);
    if (e != cudaSuccess) return cuda_fail(e, "hk_psi_loc_noalloc: local kernels");
  }
  return kOk;
}
