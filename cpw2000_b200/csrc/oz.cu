// FP64-accurate complex GEMMs on the 5th-generation tensor cores, int8 x int8 -> int32
// (the Ozaki splitting scheme: Ozaki, Ogita, Oishi, Rump 2012; int8 form after Ootomo, Ozaki,
// Yokota 2024, "DGEMM on integer matrix multiplication unit").
//
//   C (M x N) = alpha * op(A) * B (+ C),  op(A) = A (M x K) or A^H (A is K x M), all complex128
//   column-major, B K x N.
//
// Real embedding: the complex product is one real GEMM D = A' B'^T with K' = 2K, A' (M x K')
// holding each complex row of op(A) as interleaved (re, im), and B' (2N x K') holding two real
// rows per column j of B chosen so that D(i, 2j) = Re C(i, j) and D(i, 2j + 1) = Im C(i, j):
//   op(A) = A  : B' rows (Re b, -Im b) and (Im b, Re b)
//   op(A) = A^H: B' rows (Re b,  Im b) and (Im b, -Re b)
// Splitting: every real row r of A' (and every column j of B, for both of its real rows) gets
// a power-of-two scale 2^e with max |x| < 2^e over the row; y = x 2^-e in (-1, 1) is written
// as y 2^6 = d_1 + d_2 2^-7 + ... + d_s 2^-7(s-1) + rest with integer digits |d_p| <= 64
// (round to nearest at every step, all steps exact in FP64). Then
//   D(i, j) = 2^(eA_i + eB_j - 12) sum_{g = 0}^{s-1} 2^(-7 g) G_g(i, j),
//   G_g = sum_{p + q = g} A_p B_q^T  (p, q = 0-based slice indices),
// with the pairs p + q >= s left out (their terms are below 2^(-7 s) of the leading one).
// Each G_g is an exact integer sum: a work item accumulates at most kMaxKbPerItem K blocks
// (57,344 products of |d| <= 64 digits, at most 8 pairs per group) in an int32 TMEM accumulator; longer K is
// split over work items whose FP64 partials are summed in a fixed order. With s = 7 slices the
// product carries 6 + 7 * 6 = 48 bits of every operand relative to its row maximum: the error
// of an entry is below ~2^-48 K max|a| max|b|, the FP64 range for these products.
//
// Operand layout ("tiled", written by the splitting kernels): slice p of A' as 128-row x
// 128-byte tiles, slice p of B' as 64-row x 128-byte tiles, each tile in the 128-byte-swizzled
// K-major order the tensor cores read (row r at r * 128 bytes, 16-byte chunk c at
// (c ^ (r & 7)) * 16): tile (p, row block, K block) at ((p * RB + rb) * NKB + kb) * tile bytes.
//
// Kernel (persistent; work item = 128 x 64 output tile x K range; 10 warps):
//   warp 0      producer: per K block the s B' slice tiles (one stage of a 2-deep ring), then
//               the s A' slice tiles one by one (3-deep ring of 16 KB stages); bulk copies
//               (cp.async.bulk, no tensor map, no multicast) completing on mbarriers;
//   warp 1      allocates 512 TMEM columns (s groups x 64 columns of int32) and issues
//               tcgen05.mma.cta_group::1.kind::i8 (M 128, N 64, K 32): for A' slice p, the B'
//               slices q = 0 .. s-1-p into accumulator group p + q;
//   warps 2-9   drain: each reads its 32 TMEM lanes x 32 columns of every group (tcgen05.ld),
//               converts exactly to FP64 and sums the groups with their 2^(-12-7g) weights,
//               releases TMEM to the next work item, then scales by 2^(eA + eB) and alpha and
//               writes C (or an FP64 partial of a K split).
// Every mbarrier wait is bounded in time; on timeout the kernel sets an error flag, skips its
// stores, waits (bounded) for its copies and MMAs in flight, frees its TMEM and returns.
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>

#include "context.hpp"

namespace cpwb {
namespace oz {

constexpr int BM = 128;                 // rows of D per tile
constexpr int BN = 64;                  // real columns of D per tile (32 complex columns)
constexpr int KBYTES = 128;             // int8 K elements per K block
constexpr int kMaxSlices = 8;
constexpr int kAStages = 3;
constexpr int kBStages = 2;
constexpr int kATile = BM * KBYTES;     // 16 KB
constexpr int kBTile = BN * KBYTES;     // 8 KB
constexpr int kMaxKbPerItem = 448;      // K blocks per int32 accumulation: 8 pairs x 57,344 x 64^2 < 2^31
constexpr int kDrainWarps = 8;          // 4 lane quarters x 2 column halves
constexpr int kThreads = 32 * (2 + kDrainWarps);
constexpr int kTmemCols = 512;
constexpr int kBarBytes = 256;
constexpr unsigned long long kWaitNs = 2000000000ull;

inline size_t smem_bytes(int s) {
  return 1024 + (size_t)kAStages * kATile + (size_t)kBStages * s * kBTile + kBarBytes;
}

struct Args {
  const int8_t* a;             // tiled A' slices: s x RBM x NKB tiles
  const int8_t* b;             // tiled B' slices: s x RBN x NKB tiles
  const double* sa;            // 2^eA per row of A' (M)
  const double* sb;            // 2^eB per column of B (N)
  int M, N;                    // complex output dimensions (A' has M rows, B' has 2N rows)
  int s;                       // slices
  int nkb;                     // K blocks of K'
  int kb_per_split, nsplit;
  int tiles_m, tiles_n;        // tiles of 128 rows / 64 real columns
  double alpha;
  int accumulate;              // C += (nsplit == 1)
  double2* c;
  long long ldc;
  double2* part;               // nsplit > 1: partials [split][N][M]
  int* err;
  unsigned long long wait_ns;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major operand tile, 128-byte swizzle: 8-row groups 1024 bytes apart
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)((1024 >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// kind::i8 instruction descriptor: D S32, A and B signed 8-bit, both K-major, N = BN, M = BM
__device__ __forceinline__ uint32_t instr_desc_i8() {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t"
      "}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(mbar), "r"(parity)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// wait bounded in time (limit_ns); gives up early once another role has recorded a failure
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, const volatile int* failed,
                                          unsigned long long limit_ns = kWaitNs) {
  const unsigned long long t0 = globaltimer_ns();
  for (unsigned it = 0;; ++it) {
    if (mbar_try(mbar, parity)) return true;
    if ((it & 63) == 63) {
      if (failed && *failed) return false;
      if (globaltimer_ns() - t0 > limit_ns) return false;
    }
  }
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mbar), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar), "r"(bytes) : "memory");
}
// contiguous global -> shared bulk copy (16-byte aligned, size a multiple of 16), no multicast
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}

struct Item {
  int m0, n0, mt, nt, split, kb0, nblk, rows_a, rows_b;
};

__device__ __forceinline__ Item item_of(const Args& g, int it) {
  Item w;
  const int tiles = g.tiles_m * g.tiles_n;
  w.split = it / tiles;
  const int tile = it - w.split * tiles;
  w.nt = tile % g.tiles_n;         // consecutive items share an A' row block
  w.mt = tile / g.tiles_n;
  w.m0 = w.mt * BM;
  w.n0 = w.nt * BN;
  w.kb0 = w.split * g.kb_per_split;
  w.nblk = max(0, min(g.nkb, w.kb0 + g.kb_per_split) - w.kb0);
  w.rows_a = min(BM, g.M - w.m0);
  w.rows_b = min(BN, 2 * g.N - w.n0);
  return w;
}

__global__ void __launch_bounds__(kThreads, 1) k_oz_gemm(const Args g) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* aring = base;                                  // kAStages x 16 KB
  unsigned char* bring = base + kAStages * kATile;              // kBStages x s x 8 KB
  const int s = g.s;
  const size_t bslot = (size_t)s * kBTile;
  uint64_t* bars = reinterpret_cast<uint64_t*>(bring + kBStages * bslot);
  uint64_t* a_full = bars;
  uint64_t* a_empty = bars + kAStages;
  uint64_t* b_full = bars + 2 * kAStages;
  uint64_t* b_empty = b_full + kBStages;
  uint64_t* accf = b_empty + kBStages;        // accumulators complete (MMA -> drain)
  uint64_t* acce = accf + 1;                  // accumulators read (drain -> MMA)
  uint64_t* done = acce + 1;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  __shared__ volatile int failed;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nitems = g.tiles_m * g.tiles_n * g.nsplit;
  const size_t nkb = (size_t)g.nkb;

  if (threadIdx.x == 0) {
    failed = 0;
    for (int i = 0; i < kAStages; ++i) {
      mbar_init(smem_u32(&a_full[i]), 1);
      mbar_init(smem_u32(&a_empty[i]), 1);
    }
    for (int i = 0; i < kBStages; ++i) {
      mbar_init(smem_u32(&b_full[i]), 1);
      mbar_init(smem_u32(&b_empty[i]), 1);
    }
    mbar_init(smem_u32(accf), 1);
    mbar_init(smem_u32(acce), kDrainWarps);
    mbar_init(smem_u32(done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n");
  const uint32_t tmem = *tslot;

  if (warp == 0) {
    if (lane == 0) {
      long long ga = 0, gb = 0;            // A' and B' stages issued (ring positions)
      for (int it = blockIdx.x; it < nitems && !failed; it += gridDim.x) {
        const Item w = item_of(g, it);
        const uint32_t bytes_a = (uint32_t)w.rows_a * KBYTES, bytes_b = (uint32_t)w.rows_b * KBYTES;
        for (int i = 0; i < w.nblk && !failed; ++i) {
          const size_t kb = (size_t)(w.kb0 + i);
          // the s B' slice tiles of this K block
          {
            const int sb = (int)(gb % kBStages);
            const long long r = gb / kBStages;
            if (r > 0 && !mbar_wait(smem_u32(&b_empty[sb]), (uint32_t)((r - 1) & 1), &failed, g.wait_ns)) {
              failed = 1;
              atomicExch(g.err, 1);
              break;
            }
            const uint32_t fb = smem_u32(&b_full[sb]);
            mbar_expect_tx(fb, (uint32_t)s * bytes_b);
            for (int q = 0; q < s; ++q) {
              const int8_t* src = g.b + (((size_t)q * g.tiles_n + w.nt) * nkb + kb) * kBTile;
              bulk_load(smem_u32(bring + sb * bslot + (size_t)q * kBTile), src, bytes_b, fb);
            }
            ++gb;
          }
          // then the A' slice tiles one by one
          for (int p = 0; p < s; ++p) {
            const int sa = (int)(ga % kAStages);
            const long long r = ga / kAStages;
            if (r > 0 && !mbar_wait(smem_u32(&a_empty[sa]), (uint32_t)((r - 1) & 1), &failed, g.wait_ns)) {
              failed = 1;
              atomicExch(g.err, 1);
              break;
            }
            const uint32_t fa = smem_u32(&a_full[sa]);
            mbar_expect_tx(fa, bytes_a);
            const int8_t* src = g.a + (((size_t)p * g.tiles_m + w.mt) * nkb + kb) * kATile;
            bulk_load(smem_u32(aring + (size_t)sa * kATile), src, bytes_a, fa);
            ++ga;
          }
        }
      }
      // copies still in flight land before the CTA may exit
      for (long long i = (ga > kAStages ? ga - kAStages : 0); i < ga; ++i)
        if (!mbar_wait(smem_u32(&a_full[i % kAStages]), (uint32_t)((i / kAStages) & 1), nullptr))
          atomicExch(g.err, 1);
      for (long long i = (gb > kBStages ? gb - kBStages : 0); i < gb; ++i)
        if (!mbar_wait(smem_u32(&b_full[i % kBStages]), (uint32_t)((i / kBStages) & 1), nullptr))
          atomicExch(g.err, 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = instr_desc_i8();
      long long ga = 0, gb = 0;
      int nit = 0;
      for (int it = blockIdx.x; it < nitems && !failed; it += gridDim.x, ++nit) {
        const Item w = item_of(g, it);
        // the previous work item's accumulators must have been read
        if (nit > 0 && !mbar_wait(smem_u32(acce), (uint32_t)((nit - 1) & 1), &failed, g.wait_ns)) {
          failed = 1;
          atomicExch(g.err, 1);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n");
        bool ok = true;
        for (int i = 0; i < w.nblk && ok; ++i) {
          const int sb = (int)(gb % kBStages);
          if (!mbar_wait(smem_u32(&b_full[sb]), (uint32_t)((gb / kBStages) & 1), &failed, g.wait_ns)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;\n");
          const uint32_t bbase = smem_u32(bring + sb * bslot);
          for (int p = 0; p < s; ++p) {
            const int sa = (int)(ga % kAStages);
            if (!mbar_wait(smem_u32(&a_full[sa]), (uint32_t)((ga / kAStages) & 1), &failed, g.wait_ns)) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n");
            const uint32_t abase = smem_u32(aring + (size_t)sa * kATile);
            for (int q = 0; q + p < s; ++q) {
              const uint32_t tacc = tmem + (uint32_t)((p + q) * BN);
#pragma unroll
              for (int ks = 0; ks < KBYTES / 32; ++ks) {
                // the first product of group p + q in this work item starts the accumulator
                const uint32_t acc = (i == 0 && p == 0 && ks == 0) ? 0u : 1u;
                mma_i8(tacc, smem_desc(abase + ks * 32), smem_desc(bbase + q * kBTile + ks * 32), idesc, acc);
              }
            }
            mma_commit(smem_u32(&a_empty[sa]));
            ++ga;
          }
          if (!ok) break;
          mma_commit(smem_u32(&b_empty[sb]));
          ++gb;
        }
        if (!ok) {
          failed = 1;
          atomicExch(g.err, 1);
          break;
        }
        mma_commit(smem_u32(accf));
      }
      // every MMA of this thread completes before TMEM is freed
      mma_commit(smem_u32(done));
      if (!mbar_wait(smem_u32(done), 0u, nullptr)) atomicExch(g.err, 1);
    }
  } else {
    const int quarter = warp & 3, half = (warp - 2) >> 2;
    const uint32_t lane_base = tmem + ((uint32_t)(32 * quarter) << 16);
    int nit = 0;
    for (int it = blockIdx.x; it < nitems && !failed; it += gridDim.x, ++nit) {
      const Item w = item_of(g, it);
      if (!mbar_wait(smem_u32(accf), (uint32_t)(nit & 1), &failed, g.wait_ns)) {
        failed = 1;
        atomicExch(g.err, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n");
      double acc[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) acc[j] = 0.0;
      if (w.nblk > 0) {
        for (int grp = 0; grp < s; ++grp) {
          const double wgt = ldexp(1.0, -12 - 7 * grp);
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            uint32_t r[8];
            tmem_ld8(lane_base + (uint32_t)(grp * BN + 32 * half + 8 * j), r);
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
            for (int t = 0; t < 8; ++t) acc[8 * j + t] += (double)(int)r[t] * wgt;
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(acce));
      // rows of this lane, 16 complex columns of this half
      const int i = w.m0 + 32 * quarter + lane;
      if (i < g.M) {
        const double si = g.sa[i];
        const int j0 = (w.n0 + 32 * half) >> 1;
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          const int j = j0 + c;
          if (j < g.N) {
            const double sc = si * g.sb[j];
            double re = acc[2 * c] * sc, im = acc[2 * c + 1] * sc;
            if (g.nsplit > 1) {
              g.part[((size_t)w.split * g.N + j) * g.M + i] = make_double2(re, im);
            } else {
              double2* cp = g.c + (size_t)j * g.ldc + i;
              re *= g.alpha;
              im *= g.alpha;
              if (g.accumulate) {
                const double2 o = *cp;
                re += o.x;
                im += o.y;
              }
              *cp = make_double2(re, im);
            }
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n");
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols));
}

// C = alpha * sum_split part (+ C), fixed order of the splits
__global__ void k_oz_reduce(int M, int N, int nsplit, const double2* __restrict__ part, double alpha, int accumulate,
                            double2* __restrict__ c, long long ldc) {
  const long long n = (long long)M * N;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % M), j = (int)(t / M);
    double re = 0.0, im = 0.0;
    for (int sp = 0; sp < nsplit; ++sp) {
      const double2 v = part[((size_t)sp * N + j) * M + i];
      re += v.x;
      im += v.y;
    }
    re *= alpha;
    im *= alpha;
    double2* cp = c + (size_t)j * ldc + i;
    if (accumulate) {
      const double2 o = *cp;
      re += o.x;
      im += o.y;
    }
    *cp = make_double2(re, im);
  }
}

// ---- splitting ----

// 2^e with max |x| < 2^e (0 for an all-zero row)
__device__ __forceinline__ int exp_of_max(double mx) {
  int e = 0;
  if (mx > 0.0) frexp(mx, &e);
  return e;
}

// per column of a complex block (rows K, ld): scale 2^e of max(|re|, |im|); one warp per column
__global__ void k_oz_scale_cols(int K, int ncol, const double2* __restrict__ x, long long ldx, int* __restrict__ e,
                                double* __restrict__ sc) {
  const int wpb = blockDim.x >> 5;
  const int col = blockIdx.x * wpb + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (col >= ncol) return;
  const double2* p = x + (size_t)col * ldx;
  double mx = 0.0;
  for (int k = lane; k < K; k += 32) mx = fmax(mx, fmax(fabs(p[k].x), fabs(p[k].y)));
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) {
    const int ee = exp_of_max(mx);
    e[col] = ee;
    sc[col] = ldexp(1.0, ee);
  }
}

// per row of a complex block (M rows, K columns, ld): one thread per row (coalesced across rows)
__global__ void k_oz_scale_rows(int M, int K, const double2* __restrict__ x, long long ldx, int* __restrict__ e,
                                double* __restrict__ sc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  double mx = 0.0;
  for (int k = 0; k < K; ++k) {
    const double2 v = x[(size_t)k * ldx + i];
    mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
  }
  const int ee = exp_of_max(mx);
  e[i] = ee;
  sc[i] = ldexp(1.0, ee);
}

// the s digits of y in (-1, 1): y 2^6 = d_1 + d_2 2^-7 + ..., each |d| <= 64
__device__ __forceinline__ void digits(double y, int s, int8_t* d) {
  double v = y * 64.0;
  for (int p = 0; p < s; ++p) {
    const double r = rint(v);
    d[p] = (int8_t)(int)r;
    v = (v - r) * 128.0;
  }
}

// byte offset of (row r, K byte k) inside a 128-byte-row swizzled tile
__device__ __forceinline__ int swz(int r, int k) { return r * KBYTES + ((((k >> 4) ^ (r & 7)) << 4) | (k & 15)); }

// A' slices. Row r of A': conjA ? column r of A (x(k, r) = A[k + r lda]) : row r (A[r + k lda]);
// real K index 2k, 2k+1 = Re, Im of element k. One thread per (row, 16-byte chunk = 8 complex).
__global__ void k_oz_split_a(int conjA, int M, int K, const double2* __restrict__ A, long long lda,
                             const int* __restrict__ e, int s, int tiles_m, int nkb, int8_t* __restrict__ out) {
  const long long nchunk = (long long)nkb * (KBYTES / 16);
  const long long total = (long long)tiles_m * BM * nchunk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int r;
    long long ch;
    if (conjA) {          // consecutive threads walk a row (contiguous column of A)
      r = (int)(t / nchunk);
      ch = t % nchunk;
    } else {              // consecutive threads walk the rows (contiguous in A)
      r = (int)(t % ((long long)tiles_m * BM));
      ch = t / ((long long)tiles_m * BM);
    }
    if (r >= M) continue;
    const int kb = (int)(ch / (KBYTES / 16)), c16 = (int)(ch % (KBYTES / 16));
    const int k0 = (kb * KBYTES + c16 * 16) >> 1;          // first complex element of the chunk
    const double scl = ldexp(1.0, -e[r]);
    int8_t d[kMaxSlices][16];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = k0 + u;
      double2 v = make_double2(0.0, 0.0);
      if (k < K) v = conjA ? A[(size_t)r * lda + k] : A[(size_t)k * lda + r];
      int8_t dr[kMaxSlices], di[kMaxSlices];
      digits(v.x * scl, s, dr);
      digits(v.y * scl, s, di);
      for (int p = 0; p < s; ++p) {
        d[p][2 * u] = dr[p];
        d[p][2 * u + 1] = di[p];
      }
    }
    const int rb = r / BM, rr = r % BM;
    for (int p = 0; p < s; ++p) {
      int8_t* tile = out + (((size_t)p * tiles_m + rb) * nkb + kb) * kATile;
      *reinterpret_cast<int4*>(tile + swz(rr, c16 * 16)) = *reinterpret_cast<const int4*>(d[p]);
    }
  }
}

// B' slices: real rows 2j, 2j+1 from column j of B (conjA selects the pair of modes, see above).
// One thread per (column, 16-byte chunk).
__global__ void k_oz_split_b(int conjA, int N, int K, const double2* __restrict__ B, long long ldb,
                             const int* __restrict__ e, int s, int tiles_n, int nkb, int8_t* __restrict__ out) {
  const long long nchunk = (long long)nkb * (KBYTES / 16);
  const long long total = (long long)N * nchunk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t / nchunk);
    const long long ch = t % nchunk;
    const int kb = (int)(ch / (KBYTES / 16)), c16 = (int)(ch % (KBYTES / 16));
    const int k0 = (kb * KBYTES + c16 * 16) >> 1;
    const double scl = ldexp(1.0, -e[j]);
    int8_t d0[kMaxSlices][16], d1[kMaxSlices][16];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = k0 + u;
      double2 v = make_double2(0.0, 0.0);
      if (k < K) v = B[(size_t)j * ldb + k];
      const double br = v.x * scl, bi = v.y * scl;
      // op(A) = A  : rows (br, -bi), (bi, br);  op(A) = A^H: rows (br, bi), (bi, -br)
      const double r0a = br, r0b = conjA ? bi : -bi;
      const double r1a = bi, r1b = conjA ? -br : br;
      int8_t t0[kMaxSlices], t1[kMaxSlices], t2[kMaxSlices], t3[kMaxSlices];
      digits(r0a, s, t0);
      digits(r0b, s, t1);
      digits(r1a, s, t2);
      digits(r1b, s, t3);
      for (int p = 0; p < s; ++p) {
        d0[p][2 * u] = t0[p];
        d0[p][2 * u + 1] = t1[p];
        d1[p][2 * u] = t2[p];
        d1[p][2 * u + 1] = t3[p];
      }
    }
    for (int row = 0; row < 2; ++row) {
      const int r = 2 * j + row;
      const int rb = r / BN, rr = r % BN;
      for (int p = 0; p < s; ++p) {
        int8_t* tile = out + (((size_t)p * tiles_n + rb) * nkb + kb) * kBTile;
        *reinterpret_cast<int4*>(tile + swz(rr, c16 * 16)) = *reinterpret_cast<const int4*>(row ? d1[p] : d0[p]);
      }
    }
  }
}

int grid_for(long long work, int nsm) {
  return (int)std::max<long long>(1, std::min<long long>((work + 255) / 256, 8LL * nsm));
}

}  // namespace oz

// C = alpha op(A) B (+ C), complex128 column-major (see the head of this file)
int oz_zgemm(OzScratch& w, bool conjA, int M, int N, int K, const void* A, long long lda, const void* B, long long ldb,
             double alpha, bool accumulate, void* C, long long ldc, int slices, unsigned long long wait_ns,
             cudaStream_t st) {
  using namespace oz;
  if (M <= 0 || N <= 0) return kOk;
  if (slices < 1 || slices > kMaxSlices) return fail(kBadArg, "oz_zgemm: slices outside 1..8");
  cudaError_t e;
  if (K <= 0) {
    if (!accumulate) {
      e = cudaMemset2DAsync(C, 16 * (size_t)ldc, 0, 16 * (size_t)M, N, st);
      if (e != cudaSuccess) return cuda_fail(e, "oz_zgemm");
    }
    return kOk;
  }
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int s = slices;
  const int nkb = (int)((2LL * K + KBYTES - 1) / KBYTES);
  const int tiles_m = (M + BM - 1) / BM, tiles_n = (2 * N + BN - 1) / BN;
  // K splits: enough work items for every SM, every split at most kMaxKbPerItem K blocks
  const int tiles = tiles_m * tiles_n;
  int nsplit = std::max(1, (nkb + kMaxKbPerItem - 1) / kMaxKbPerItem);
  while (tiles * nsplit < nsm && nsplit * 8 <= nkb) ++nsplit;
  const int kbps = (nkb + nsplit - 1) / nsplit;
  nsplit = (nkb + kbps - 1) / kbps;
  const size_t abytes = (size_t)s * tiles_m * nkb * kATile, bbytes = (size_t)s * tiles_n * nkb * kBTile;
  int rs;
  if ((rs = w.a.ensure(abytes)) || (rs = w.b.ensure(bbytes)) || (rs = w.ea.ensure(sizeof(int) * (size_t)M)) ||
      (rs = w.eb.ensure(sizeof(int) * (size_t)N)) || (rs = w.sa.ensure(sizeof(double) * (size_t)M)) ||
      (rs = w.sb.ensure(sizeof(double) * (size_t)N)) || (rs = w.err.ensure(sizeof(int))))
    return rs;
  if (!w.err_init) {
    if ((e = cudaMemsetAsync(w.err.p, 0, sizeof(int), st)) != cudaSuccess) return cuda_fail(e, "oz_zgemm");
    w.err_init = true;
  }
  if (nsplit > 1 && (rs = w.part.ensure(16 * (size_t)nsplit * M * N))) return rs;
  const double2* a = (const double2*)A;
  const double2* b = (const double2*)B;
  if (conjA)
    k_oz_scale_cols<<<(M + 7) / 8, 256, 0, st>>>(K, M, a, lda, (int*)w.ea.p, (double*)w.sa.p);
  else
    k_oz_scale_rows<<<(M + 255) / 256, 256, 0, st>>>(M, K, a, lda, (int*)w.ea.p, (double*)w.sa.p);
  k_oz_scale_cols<<<(N + 7) / 8, 256, 0, st>>>(K, N, b, ldb, (int*)w.eb.p, (double*)w.sb.p);
  k_oz_split_a<<<grid_for((long long)tiles_m * BM * nkb * 8, nsm), 256, 0, st>>>(
      conjA ? 1 : 0, M, K, a, lda, (const int*)w.ea.p, s, tiles_m, nkb, (int8_t*)w.a.p);
  k_oz_split_b<<<grid_for((long long)N * nkb * 8, nsm), 256, 0, st>>>(conjA ? 1 : 0, N, K, b, ldb, (const int*)w.eb.p,
                                                                      s, tiles_n, nkb, (int8_t*)w.b.p);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "oz_zgemm splitting");
  Args g{};
  g.a = (const int8_t*)w.a.p;
  g.b = (const int8_t*)w.b.p;
  g.sa = (const double*)w.sa.p;
  g.sb = (const double*)w.sb.p;
  g.M = M;
  g.N = N;
  g.s = s;
  g.nkb = nkb;
  g.kb_per_split = kbps;
  g.nsplit = nsplit;
  g.tiles_m = tiles_m;
  g.tiles_n = tiles_n;
  g.alpha = alpha;
  g.accumulate = accumulate ? 1 : 0;
  g.c = (double2*)C;
  g.ldc = ldc;
  g.part = (double2*)w.part.p;
  g.err = (int*)w.err.p;
  g.wait_ns = wait_ns;
  const size_t smem = smem_bytes(s);
  if ((e = smem_limit((const void*)k_oz_gemm, (size_t)smem)) != cudaSuccess)
    return cuda_fail(e, "oz_zgemm attribute");
  const int items = tiles * nsplit;
  k_oz_gemm<<<std::min(items, nsm), kThreads, smem, st>>>(g);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "oz_zgemm launch");
  if (nsplit > 1) {
    k_oz_reduce<<<grid_for((long long)M * N, nsm), 256, 0, st>>>(M, N, nsplit, (const double2*)w.part.p, alpha,
                                                                accumulate ? 1 : 0, (double2*)C, ldc);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "oz_zgemm reduce");
  }
  return kOk;
}

int oz_read_error(OzScratch& w) {
  if (!w.err.p || !w.err_init) return kOk;
  int h = 0;
  cudaError_t e = cudaMemcpy(&h, w.err.p, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "oz error flag");
  if (!h) return kOk;
  cudaMemset(w.err.p, 0, sizeof(int));
  return fail(kTimeout, "int8 tensor-core GEMM: an mbarrier wait gave up");
}

}  // namespace cpwb
