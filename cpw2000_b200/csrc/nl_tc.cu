// Mixed-precision KB projector products on the 5th-generation tensor cores.
//
// The complex products of Src/cpw_lib/hk_psi_nl_c16.f90:82-97 written as real
// GEMMs in split TF32 (x = hi + lo, both TF32; a.b ~ hi.hi + hi.lo + lo.hi with
// FP32 accumulation in tensor memory, ~2^-21 relative per product):
//
//   1. P = X^H psi:  [Re P; Im P] (2 nanl x nb) = A1 (2 nanl x 2 mtxd) . psi_interleaved
//      A1 row a      = (xr_1, xi_1, xr_2, xi_2, ...) of projector a
//      A1 row nanl+a = (-xi_1, xr_1, ...)
//      psi is read in FP64 and split while it is staged into shared memory.
//      Split over K across CTAs, FP32 partials summed in FP64 by k_reduce_p.
//   2. hpsi += (X D) P: [Re | Im] (mtxd x 2 nb) = A2 (mtxd x 2 nanl) . B2^T with
//      A2 row i = (xd_r(i, :), xd_i(i, :)), B2 row n = (Pr(:,n), -Pi(:,n)),
//      B2 row nb+n = (Pi(:,n), Pr(:,n)); the epilogue adds into the FP64 hpsi.
//
// Kernel: one CTA of 4 warps per 128 x 128 output tile (and K range); 32-wide
// K blocks staged (global -> registers -> shared, 128-byte swizzle) into two
// buffers; thread 0 issues tcgen05.mma kind::tf32 (M 128, N 128, K 8) and
// commits each block to an mbarrier; the other buffer is refilled meanwhile.
// The accumulator lives in 128 TMEM columns and is read back with
// tcgen05.ld 32x32b. Every mbarrier wait is bounded: on timeout the kernel sets
// an error flag, skips its epilogue, frees its TMEM and returns.
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>
#include <string>

#include "context.hpp"

namespace cpwb {
namespace tc {

constexpr int BM = 128, BN = 128, BK = 32;
constexpr int kThreads = 128;
constexpr int kTileBytes = BM * BK * 4;            // 16 KB per operand tile
constexpr int kStageBytes = 4 * kTileBytes;        // A hi/lo + B hi/lo
constexpr int kSmemBytes = 2 * kStageBytes + 1024 + 64;
constexpr long long kWaitLimit = 1LL << 22;
constexpr int kMainAcc = 3;                        // hi.hi accumulators; + 1 for the corrections
constexpr int kTmemCols = (kMainAcc + 1) * BN;     // 512 columns

struct GemmArgs {
  int M, N, K;                 // output rows / cols, reduction length
  int kb_per_split;            // 32-wide K blocks per CTA (blockIdx.z)
  const float* a_hi;           // M x lda, row-major, zero beyond K
  const float* a_lo;
  long long lda;
  const float* b_hi;           // N x ldb row-major (B source 0)
  const float* b_lo;
  long long ldb;
  const double* b64;           // B source 1: row n = doubles b64[n*ldb64 ...], K reals per row
  long long ldb64;
  float* part;                 // mode 0: part[z][n][mpad]
  long long mpad;
  double* hpsi;                // mode 1: complex128 (interleaved), ld ldh complex elements
  long long ldh;
  int nbh;                     // mode 1: columns < nbh are real parts, >= nbh imaginary parts
  int terms;                   // 3: hi.hi + hi.lo + lo.hi; 4: also lo.lo
  int* err;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ float tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// K-major, 128-byte swizzled tile of rows x 32 fp32: row r, 16-byte chunk c
__device__ __forceinline__ int sw_off(int r, int c) { return r * 128 + ((c ^ (r & 7)) << 4); }

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);               // start address
  d |= (uint64_t)1 << 16;                               // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)((1024 >> 4) & 0x3FFF) << 32;          // stride byte offset: 8 rows x 128 B
  d |= (uint64_t)1 << 46;                               // descriptor version
  d |= (uint64_t)2 << 61;                               // 128-byte swizzle
  return d;
}

__device__ __forceinline__ uint32_t instr_desc() {
  return (1u << 4)                  // D format F32
         | (2u << 7)                // A TF32
         | (2u << 10)               // B TF32
         | ((uint32_t)(BN >> 3) << 17)
         | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t"
      "}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (long long it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// stage rows [r0, r0+128) x K block kb of a row-major FP32 hi/lo pair
__device__ __forceinline__ void load_split(unsigned char* hi_t, unsigned char* lo_t, const float* hi, const float* lo,
                                          long long ld, int rows, int r0, int k0) {
  for (int idx = threadIdx.x; idx < BM * 8; idx += kThreads) {
    const int r = idx >> 3, c = idx & 7;
    float4 vh = make_float4(0.f, 0.f, 0.f, 0.f), vl = vh;
    if (r0 + r < rows) {
      const size_t o = (size_t)(r0 + r) * ld + k0 + 4 * c;
      vh = *reinterpret_cast<const float4*>(hi + o);
      vl = *reinterpret_cast<const float4*>(lo + o);
    }
    *reinterpret_cast<float4*>(hi_t + sw_off(r, c)) = vh;
    *reinterpret_cast<float4*>(lo_t + sw_off(r, c)) = vl;
  }
}

// stage rows of an FP64 source, splitting into TF32 hi/lo on the way
__device__ __forceinline__ void load_fp64(unsigned char* hi_t, unsigned char* lo_t, const double* src, long long ld,
                                         int rows, int K, int r0, int k0) {
  for (int idx = threadIdx.x; idx < BN * 8; idx += kThreads) {
    const int r = idx >> 3, c = idx & 7;
    float h[4] = {0.f, 0.f, 0.f, 0.f}, l[4] = {0.f, 0.f, 0.f, 0.f};
    if (r0 + r < rows) {
      const double* row = src + (size_t)(r0 + r) * ld;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = k0 + 4 * c + j;
        if (k < K) {
          const double x = row[k];
          const float xh = tf32((float)x);
          h[j] = xh;
          l[j] = tf32((float)(x - (double)xh));
        }
      }
    }
    *reinterpret_cast<float4*>(hi_t + sw_off(r, c)) = make_float4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<float4*>(lo_t + sw_off(r, c)) = make_float4(l[0], l[1], l[2], l[3]);
  }
}

template <int BSRC, int MODE>
__global__ void __launch_bounds__(kThreads, 1) k_gemm_tf32x3(GemmArgs g) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* tiles = base;                                     // 2 stages x (A hi, A lo, B hi, B lo)
  uint64_t* mbar = reinterpret_cast<uint64_t*>(base + 2 * kStageBytes);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(base + 2 * kStageBytes + 16);
  __shared__ int failed;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int nkb_total = (g.K + BK - 1) / BK;
  const int kb0 = blockIdx.z * g.kb_per_split;
  const int kb1 = min(nkb_total, kb0 + g.kb_per_split);

  if (threadIdx.x == 0) {
    failed = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n");
  const uint32_t tmem = *tslot;
  const uint32_t idesc = instr_desc();

  const int nblk = kb1 - kb0;
  for (int i = 0; i < nblk; ++i) {
    const int s = i & 1;
    unsigned char* st = tiles + s * kStageBytes;
    if (i >= 2) {
      // the MMAs that read this stage two blocks ago must be finished
      if (!mbar_wait(smem_u32(&mbar[s]), (uint32_t)(((i - 2) >> 1) & 1))) {
        if (threadIdx.x == 0) atomicExch(g.err, 1);
        failed = 1;
      }
      __syncthreads();
      if (failed) break;
    }
    const int k0 = (kb0 + i) * BK;
    load_split(st, st + kTileBytes, g.a_hi, g.a_lo, g.lda, g.M, m0, k0);
    if (BSRC == 0)
      load_split(st + 2 * kTileBytes, st + 3 * kTileBytes, g.b_hi, g.b_lo, g.ldb, g.N, n0, k0);
    else
      load_fp64(st + 2 * kTileBytes, st + 3 * kTileBytes, g.b64, g.ldb64, g.N, g.K, n0, k0);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n");
      const uint32_t ah = smem_u32(st), al = smem_u32(st + kTileBytes);
      const uint32_t bh = smem_u32(st + 2 * kTileBytes), bl = smem_u32(st + 3 * kTileBytes);
      // hi.hi into main accumulator i % 3 (round-robin keeps each FP32 chain short),
      // the small correction products into the fourth accumulator
      const uint32_t tmain = tmem + (uint32_t)((i % kMainAcc) * BN);
      const uint32_t tcorr = tmem + (uint32_t)(kMainAcc * BN);
#pragma unroll
      for (int ks = 0; ks < BK / 8; ++ks) {
        const uint32_t off = ks * 32;       // 8 tf32 = 32 bytes along K inside the swizzled row
        mma_tf32(tmain, smem_desc(ah + off), smem_desc(bh + off), idesc, (i < kMainAcc && ks == 0) ? 0u : 1u);
        mma_tf32(tcorr, smem_desc(ah + off), smem_desc(bl + off), idesc, (i == 0 && ks == 0) ? 0u : 1u);
        mma_tf32(tcorr, smem_desc(al + off), smem_desc(bh + off), idesc, 1u);
        if (g.terms > 3) mma_tf32(tcorr, smem_desc(al + off), smem_desc(bl + off), idesc, 1u);
      }
      mma_commit(smem_u32(&mbar[s]));
    }
  }
  // wait for the last block's MMAs (they complete after all earlier ones)
  if (nblk > 0 && !failed) {
    const int last = nblk - 1;
    if (!mbar_wait(smem_u32(&mbar[last & 1]), (uint32_t)((last >> 1) & 1))) {
      if (threadIdx.x == 0) atomicExch(g.err, 1);
      failed = 1;
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n");
  if (!failed && nblk > 0) {
    const int m = m0 + warp * 32 + lane;
    const int nacc = min(nblk, kMainAcc);
    for (int c0 = 0; c0 < BN; c0 += 16) {
      double acc[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) acc[j] = 0.0;
      for (int a = 0; a <= kMainAcc; ++a) {
        if (a < kMainAcc && a >= nacc) continue;      // main accumulators that never received a block
        uint32_t r[16];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(a * BN + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[j] += (double)__uint_as_float(r[j]);
      }
      if (m < g.M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = n0 + c0 + j;
          if (n >= g.N) continue;
          const double v = acc[j];
          if (MODE == 0) {
            g.part[((size_t)blockIdx.z * g.N + n) * g.mpad + m] = (float)v;
          } else {
            const int col = n < g.nbh ? n : n - g.nbh;
            double* dst = g.hpsi + 2 * ((size_t)col * g.ldh + m) + (n < g.nbh ? 0 : 1);
            *dst += v;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols));
}

// A1 (2 nanl x k1p) and A2 (mtxd x k2p) TF32 hi/lo from X (anl) and X D (anld), complex128 ld mtxd
__global__ void k_prep_a1(int mtxd, int nanl, long long k1p, const C2<double>* __restrict__ x, float* __restrict__ hi,
                          float* __restrict__ lo) {
  const long long n = 2LL * nanl * k1p;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long row = t / k1p, k = t - row * k1p;
    const int a = (int)(row % nanl);
    const bool rot = row >= nanl;
    const long long i = k >> 1;
    double v = 0.0;
    if (i < mtxd) {
      const C2<double> z = x[(size_t)a * mtxd + i];
      v = (k & 1) ? (rot ? z.x : z.y) : (rot ? -z.y : z.x);
    }
    const float h = tf32((float)v);
    hi[t] = h;
    lo[t] = tf32((float)(v - (double)h));
  }
}

__global__ void k_prep_a2(int mtxd, int nanl, long long k2p, const C2<double>* __restrict__ xd, float* __restrict__ hi,
                          float* __restrict__ lo) {
  const long long n = (long long)mtxd * k2p;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / k2p, k = t - i * k2p;
    double v = 0.0;
    if (k < 2 * nanl) {
      const int a = (int)(k % nanl);
      const C2<double> z = xd[(size_t)a * mtxd + i];
      v = k < nanl ? z.x : z.y;
    }
    const float h = tf32((float)v);
    hi[t] = h;
    lo[t] = tf32((float)(v - (double)h));
  }
}

// P from the split-K partials, and B2 (2 nb x k2p) TF32 hi/lo for the expansion GEMM
__global__ void k_reduce_p(int nanl, int nb, int nsplit, long long mpad, long long k2p, const float* __restrict__ part,
                           float* __restrict__ b2hi, float* __restrict__ b2lo) {
  const long long n = (long long)nanl * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(t % nanl), b = (int)(t / nanl);
    double pr = 0.0, pi = 0.0;
    for (int z = 0; z < nsplit; ++z) {
      const float* pz = part + ((size_t)z * nb + b) * mpad;
      pr += pz[a];
      pi += pz[nanl + a];
    }
    auto put = [&](long long row, long long k, double v) {
      const float h = tf32((float)v);
      b2hi[row * k2p + k] = h;
      b2lo[row * k2p + k] = tf32((float)(v - (double)h));
    };
    put(b, a, pr);
    put(b, nanl + a, -pi);
    put(nb + b, a, pi);
    put(nb + b, nanl + a, pr);
  }
}

}  // namespace tc

int tc_prepare_projectors(cpw_b200_ctx* c) {
  const int m = c->mtxd, na = c->nanl;
  if (na == 0 || m == 0) return kOk;
  const long long k1p = ((2LL * m + tc::BK - 1) / tc::BK) * tc::BK;
  const long long k2p = ((2LL * na + tc::BK - 1) / tc::BK) * tc::BK;
  int s;
  if ((s = c->tc_a1.ensure(sizeof(float) * 2 * (size_t)(2 * na) * k1p)) ||
      (s = c->tc_a2.ensure(sizeof(float) * 2 * (size_t)m * k2p)))
    return s;
  float* a1 = (float*)c->tc_a1.p;
  float* a2 = (float*)c->tc_a2.p;
  tc::k_prep_a1<<<1184, 256, 0, c->stream>>>(m, na, k1p, (const C2<double>*)c->anl.p, a1, a1 + (size_t)2 * na * k1p);
  tc::k_prep_a2<<<1184, 256, 0, c->stream>>>(m, na, k2p, (const C2<double>*)c->anld.p, a2, a2 + (size_t)m * k2p);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "tensor-core projector preparation");
  c->tc_k1p = k1p;
  c->tc_k2p = k2p;
  c->tc_ready = true;
  return kOk;
}

// hpsi += X D X^H psi in split TF32 on the tensor cores (hpsi already holds the local part)
int tc_nl_apply(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, void* hpsi, long long ldh, cudaStream_t st,
                cudaEvent_t t0, cudaEvent_t t1, cudaEvent_t t2) {
  if (!c->tc_ready) return fail(kNotReady, "tensor-core projectors not prepared");
  const int m = c->mtxd, na = c->nanl;
  const long long k1p = c->tc_k1p, k2p = c->tc_k2p;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  // GEMM 1: (2 nanl) x nb, K = 2 mtxd, split over K
  const int mt1 = (2 * na + tc::BM - 1) / tc::BM, nt1 = (nb + tc::BN - 1) / tc::BN;
  const int nkb = (int)(k1p / tc::BK);
  // K blocks per CTA of the projection: at most 16 (three main accumulators of <= 6 blocks each keep the
  // FP32 accumulation bias of the tensor cores near 5e-7 relative), fewer when the grid is too small
  int nsplit = std::max(1, std::min(nkb, (2 * nsm) / std::max(1, mt1 * nt1)));
  int kbps = std::min(16, (nkb + nsplit - 1) / nsplit);
  // tuning: K blocks per CTA (shorter chains are more accurate, longer ones write fewer partials)
  if (const char* ev = getenv("CPW_B200_TC_KBLOCKS")) kbps = std::max(1, std::min(nkb, atoi(ev)));
  nsplit = (nkb + kbps - 1) / kbps;
  const long long mpad = (long long)mt1 * tc::BM;
  int s;
  if ((s = c->tc_part.ensure(sizeof(float) * (size_t)nsplit * nb * mpad)) ||
      (s = c->tc_b2.ensure(sizeof(float) * 2 * (size_t)(2 * nb) * k2p)) || (s = c->tc_err.ensure(sizeof(int))))
    return s;
  cudaError_t e = cudaMemsetAsync(c->tc_err.p, 0, sizeof(int), st);
  if (e != cudaSuccess) return cuda_fail(e, "tc nl");
  // B2 rows beyond 2 nanl in K must be zero: clear once per call (small)
  e = cudaMemsetAsync(c->tc_b2.p, 0, sizeof(float) * 2 * (size_t)(2 * nb) * k2p, st);
  if (e != cudaSuccess) return cuda_fail(e, "tc nl");
  if ((e = cudaFuncSetAttribute(tc::k_gemm_tf32x3<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                tc::kSmemBytes)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(tc::k_gemm_tf32x3<0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                tc::kSmemBytes)) != cudaSuccess)
    return cuda_fail(e, "tensor-core GEMM attribute");
  tc::GemmArgs g1{};
  g1.M = 2 * na;
  g1.N = nb;
  g1.K = 2 * m;
  g1.kb_per_split = kbps;
  g1.a_hi = (const float*)c->tc_a1.p;
  g1.a_lo = g1.a_hi + (size_t)2 * na * k1p;
  g1.lda = k1p;
  g1.b64 = (const double*)psi;
  g1.ldb64 = 2 * ldpsi;
  g1.part = (float*)c->tc_part.p;
  g1.mpad = mpad;
  g1.err = (int*)c->tc_err.p;
  int terms = 3;
  if (const char* ev = getenv("CPW_B200_TC_TERMS")) terms = atoi(ev) == 4 ? 4 : 3;
  g1.terms = terms;
  if (t0) cudaEventRecord(t0, st);
  tc::k_gemm_tf32x3<1, 0><<<dim3(mt1, nt1, nsplit), tc::kThreads, tc::kSmemBytes, st>>>(g1);
  float* b2 = (float*)c->tc_b2.p;
  tc::k_reduce_p<<<std::max(1, std::min(1184, (na * nb + 255) / 256)), 256, 0, st>>>(
      na, nb, nsplit, mpad, k2p, (const float*)c->tc_part.p, b2, b2 + (size_t)(2 * nb) * k2p);
  if (t1) cudaEventRecord(t1, st);
  // GEMM 2: mtxd x (2 nb), K = 2 nanl, accumulate into hpsi
  tc::GemmArgs g2{};
  g2.M = m;
  g2.N = 2 * nb;
  g2.K = (int)k2p;
  g2.kb_per_split = (int)(k2p / tc::BK);
  g2.a_hi = (const float*)c->tc_a2.p;
  g2.a_lo = g2.a_hi + (size_t)m * k2p;
  g2.lda = k2p;
  g2.b_hi = b2;
  g2.b_lo = b2 + (size_t)(2 * nb) * k2p;
  g2.ldb = k2p;
  g2.hpsi = (double*)hpsi;
  g2.ldh = ldh;
  g2.nbh = nb;
  g2.err = (int*)c->tc_err.p;
  g2.terms = terms;
  tc::k_gemm_tf32x3<0, 1><<<dim3((m + tc::BM - 1) / tc::BM, (2 * nb + tc::BN - 1) / tc::BN, 1), tc::kThreads,
                            tc::kSmemBytes, st>>>(g2);
  if (t2) cudaEventRecord(t2, st);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "tensor-core projector GEMMs");
  return kOk;
}

int tc_check_error(cpw_b200_ctx* c) {
  if (!c->tc_err.p) return kOk;
  int h = 0;
  cudaError_t e = cudaMemcpy(&h, c->tc_err.p, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "tc error flag");
  return h ? fail(kTimeout, "tensor-core GEMM: an mbarrier wait gave up") : kOk;
}

}  // namespace cpwb
