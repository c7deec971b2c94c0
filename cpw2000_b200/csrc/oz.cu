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
// Kernel (one CTA per work item = 128 x 64 output tile x K range; 10 warps):
//   warp 0      producer: per K block the s B' slice tiles (one stage of a 2-deep ring), then
//               the s A' slice tiles two by two (3-deep ring of 32 KB stages); bulk copies
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
#include <type_traits>

#include "context.hpp"

namespace cpwb {
namespace oz {

constexpr int BM = 128;                 // rows of D per tile
constexpr int BN = 64;                  // real columns of D per tile (32 complex columns)
constexpr int KBYTES = 128;             // int8 K elements per K block
constexpr int kMaxSlices = 8;
constexpr int kAStages = 3;
constexpr int kAPer = 2;                // A' slice tiles per stage
constexpr int kBStages = 2;
constexpr int kATile = BM * KBYTES;     // 16 KB
constexpr int kBTile = BN * KBYTES;     // 8 KB
constexpr int kMaxKbPerItem = 448;      // K blocks per int32 accumulation: 8 pairs x 57,344 x 64^2 < 2^31
constexpr int kShortKb = 48;            // K blocks per work item by default (latency of one CTA)
constexpr int kDrainWarps = 8;          // 4 lane quarters x 2 column halves
constexpr int kThreads = 32 * (2 + kDrainWarps);
constexpr int kTmemCols = 512;
constexpr int kBarBytes = 256;
constexpr unsigned long long kWaitNs = 2000000000ull;

inline size_t smem_bytes(int s) {
  return 1024 + (size_t)kAStages * kAPer * kATile + (size_t)kBStages * s * kBTile + kBarBytes;
}

struct Args {
  const int8_t* a;             // tiled A' slices: s x RBM x NKB tiles
  const int8_t* b;             // tiled B' slices: s x RBN x NKB tiles
  const int* ea;               // row exponents of A' (M)
  const int* eb;               // column exponents of B (N)
  int M, N;                    // complex output dimensions (A' has M rows, B' has 2N rows)
  int s;                       // slices
  int nkb;                     // K blocks of K'
  int kb_per_split, nsplit;
  int tiles_m, tiles_n;        // tiles of 128 rows / 64 real columns
  double alpha;
  int accumulate;              // C += (nsplit == 1)
  int tri;                     // OzTri: triangular structure of the product
  double2* c;
  long long ldc;
  double2* part;               // nsplit > 1: partials [split][N][M]
  int* err;
  unsigned long long wait_ns;
};

// row exponents not raised by any nonzero element (all-zero rows: scale 1)
constexpr int kNoExp = (int)0x80808080;           // memset byte 0x80
__device__ __forceinline__ int chunk_exp(double mx) {
  int e = kNoExp;
  if (mx > 0.0) frexp(mx, &e);
  return e;
}
__device__ __forceinline__ int exp_or0(int e) { return e == kNoExp ? 0 : e; }

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
  int klim = g.nkb;
  if (g.tri == kOzUpperB) {
    // complex columns [32 nt, 32 nt + 32) of an upper-triangular B have no nonzero below row
    // 32 nt + 31: K blocks (64 complex rows each) from (nt + 2) / 2 on contribute nothing
    klim = min(klim, (w.nt + 2) >> 1);
  } else if (g.tri == kOzLowerOut && 32 * w.nt > w.mt * BM + BM - 1) {
    klim = 0;                      // the tile lies strictly above the diagonal: written as zeros
  }
  w.nblk = max(0, min(klim, w.kb0 + g.kb_per_split) - w.kb0);
  w.rows_a = min(BM, g.M - w.m0);
  w.rows_b = min(BN, 2 * g.N - w.n0);
  return w;
}

__global__ void __launch_bounds__(kThreads, 1) k_oz_gemm(const Args g) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* aring = base;                                  // kAStages x kAPer x 16 KB
  unsigned char* bring = base + kAStages * kAPer * kATile;      // kBStages x s x 8 KB
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
          // then the A' slice tiles, kAPer per stage
          for (int p0 = 0; p0 < s; p0 += kAPer) {
            const int sa = (int)(ga % kAStages);
            const long long r = ga / kAStages;
            if (r > 0 && !mbar_wait(smem_u32(&a_empty[sa]), (uint32_t)((r - 1) & 1), &failed, g.wait_ns)) {
              failed = 1;
              atomicExch(g.err, 1);
              break;
            }
            const int np = min(kAPer, s - p0);
            const uint32_t fa = smem_u32(&a_full[sa]);
            mbar_expect_tx(fa, (uint32_t)np * bytes_a);
            for (int u = 0; u < np; ++u) {
              const int8_t* src = g.a + (((size_t)(p0 + u) * g.tiles_m + w.mt) * nkb + kb) * kATile;
              bulk_load(smem_u32(aring + ((size_t)sa * kAPer + u) * kATile), src, bytes_a, fa);
            }
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
          // descriptors: the start-address field is the byte address / 16, so moving by q tiles and
          // ks 32-byte K steps adds (q kBTile + 32 ks) / 16 to it
          const uint64_t db = smem_desc(smem_u32(bring + sb * bslot));
          for (int p0 = 0; p0 < s && ok; p0 += kAPer) {
            const int sa = (int)(ga % kAStages);
            if (!mbar_wait(smem_u32(&a_full[sa]), (uint32_t)((ga / kAStages) & 1), &failed, g.wait_ns)) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n");
            const int np = min(kAPer, s - p0);
            for (int u = 0; u < np; ++u) {
              const int p = p0 + u;
              const uint64_t da = smem_desc(smem_u32(aring + ((size_t)sa * kAPer + u) * kATile));
              for (int q = 0; q + p < s; ++q) {
                const uint32_t tacc = tmem + (uint32_t)((p + q) * BN);
#pragma unroll
                for (int ks = 0; ks < KBYTES / 32; ++ks) {
                  // the first product of group p + q in this work item starts the accumulator
                  const uint32_t acc = (i == 0 && p == 0 && ks == 0) ? 0u : 1u;
                  mma_i8(tacc, da + (uint64_t)(2 * ks), db + (uint64_t)(q * (kBTile >> 4) + 2 * ks), idesc, acc);
                }
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
          uint32_t r[4][8];
#pragma unroll
          for (int j = 0; j < 4; ++j) tmem_ld8(lane_base + (uint32_t)(grp * BN + 32 * half + 8 * j), r[j]);
          asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
          for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int t = 0; t < 8; ++t) acc[8 * j + t] += (double)(int)r[j][t] * wgt;
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(acce));
      // rows of this lane, 16 complex columns of this half, in two groups of 8 whose column
      // exponents and (when accumulating) old C values are all loaded before the first store,
      // so that their latencies overlap instead of adding up column by column
      const int i = w.m0 + 32 * quarter + lane;
      if (i < g.M) {
        const int ei = exp_or0(g.ea[i]);
        const int j0 = (w.n0 + 32 * half) >> 1;
        const bool add_old = g.nsplit == 1 && g.accumulate;
#pragma unroll
        for (int c0 = 0; c0 < 16; c0 += 8) {
          int ej[8];
          double2 o[8];
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            const int j = j0 + c0 + c;
            ej[c] = j < g.N ? exp_or0(g.eb[j]) : 0;
            o[c] = add_old && j < g.N ? g.c[(size_t)j * g.ldc + i] : make_double2(0.0, 0.0);
          }
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            const int j = j0 + c0 + c;
            if (j < g.N) {
              const double sc = ldexp(1.0, ei + ej[c]);
              double re = acc[2 * (c0 + c)] * sc, im = acc[2 * (c0 + c) + 1] * sc;
              if (g.nsplit > 1) {
                g.part[((size_t)w.split * g.N + j) * g.M + i] = make_double2(re, im);
              } else {
                re = re * g.alpha + o[c].x;
                im = im * g.alpha + o[c].y;
                g.c[(size_t)j * g.ldc + i] = make_double2(re, im);
              }
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

// Row exponents: e with max |x| < 2^e over the row (frexp of the maximum). The reductions run in
// parallel over K chunks and meet in an atomicMax of the exponent (the exponent of the maximum is
// the maximum of the exponents); all-zero chunks leave the initial kNoExp (-> scale 1).

constexpr int kExpChunk = 4096;                   // K elements per block of the column reduction

// per column of a complex block (rows K, ld): grid (ncol, K chunks), 256 threads
__global__ void __launch_bounds__(256) k_oz_exp_cols(int K, int ncol, const double2* __restrict__ x, long long ldx,
                                                     int* __restrict__ e) {
  const int col = blockIdx.x;
  const int k0 = blockIdx.y * kExpChunk, k1 = min(K, k0 + kExpChunk);
  const double2* p = x + (size_t)col * ldx;
  double mx = 0.0;
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) mx = fmax(mx, fmax(fabs(p[k].x), fabs(p[k].y)));
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  __shared__ double wm[8];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mx = fmax(mx, wm[w]);
    const int ce = chunk_exp(fmax(mx, wm[0]));
    if (ce != kNoExp) atomicMax(&e[col], ce);
  }
}

constexpr int kExpRowChunk = 32;                  // K elements per thread of the row reduction

// per row of a complex block (M rows, K columns, ld): thread per (row, K chunk), coalesced over rows
__global__ void __launch_bounds__(256) k_oz_exp_rows(int M, int K, const double2* __restrict__ x, long long ldx,
                                                     int* __restrict__ e) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  const int k0 = blockIdx.y * kExpRowChunk, k1 = min(K, k0 + kExpRowChunk);
  double mx = 0.0;
  for (int k = k0; k < k1; ++k) {
    const double2 v = x[(size_t)k * ldx + i];
    mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
  }
  const int ce = chunk_exp(mx);
  if (ce != kNoExp) atomicMax(&e[i], ce);
}

// The digits of y in (-1, 1): y 2^6 = d_1 + d_2 2^-7 + ..., each |d| <= 64, taken by rounding to
// the nearest integer and scaling the exact remainder by 2^7 (the split kernels below).

// byte offset of (row r, K byte k) inside a 128-byte-row swizzled tile
__device__ __forceinline__ int swz(int r, int k) { return r * KBYTES + ((((k >> 4) ^ (r & 7)) << 4) | (k & 15)); }

// A' slices. Row r of A': conjA ? column r of A (x(k, r) = A[k + r lda]) : row r (A[r + k lda]);
// real K index 2k, 2k+1 = Re, Im of element k. One thread per (row, 16-byte chunk = 8 complex);
// the slice count is a template parameter so that the digits stay in registers.
template <int S>
__global__ void __launch_bounds__(256) k_oz_split_a(int conjA, int M, int K, const double2* __restrict__ A,
                                                    long long lda, const int* __restrict__ e, int tiles_m, int nkb,
                                                    int8_t* __restrict__ out) {
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
    const double scl = ldexp(1.0, -exp_or0(e[r]));
    uint32_t w[S][4];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = k0 + u;
      double2 v = make_double2(0.0, 0.0);
      if (k < K) v = conjA ? A[(size_t)r * lda + k] : A[(size_t)k * lda + r];
      double vr = v.x * scl * 64.0, vi = v.y * scl * 64.0;
#pragma unroll
      for (int p = 0; p < S; ++p) {
        const double dr = rint(vr), di = rint(vi);
        const uint32_t pair = ((uint32_t)(uint8_t)(int8_t)(int)dr) | ((uint32_t)(uint8_t)(int8_t)(int)di << 8);
        const int word = u >> 1, sh = (u & 1) * 16;
        if (sh == 0) w[p][word] = pair; else w[p][word] |= pair << 16;
        vr = (vr - dr) * 128.0;
        vi = (vi - di) * 128.0;
      }
    }
    const int rb = r / BM, rr = r % BM;
#pragma unroll
    for (int p = 0; p < S; ++p) {
      int8_t* tile = out + (((size_t)p * tiles_m + rb) * nkb + kb) * kATile;
      *reinterpret_cast<uint4*>(tile + swz(rr, c16 * 16)) = make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
    }
  }
}

// B' slices: real rows 2j, 2j+1 from column j of B (conjA selects the pair of modes, see above).
// One thread per (column, 16-byte chunk); the slice count is a template parameter.
template <int S>
__global__ void __launch_bounds__(256) k_oz_split_b(int conjA, int N, int K, const double2* __restrict__ B,
                                                    long long ldb, const int* __restrict__ e, int tiles_n, int nkb,
                                                    int8_t* __restrict__ out) {
  const long long nchunk = (long long)nkb * (KBYTES / 16);
  const long long total = (long long)N * nchunk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t / nchunk);
    const long long ch = t % nchunk;
    const int kb = (int)(ch / (KBYTES / 16)), c16 = (int)(ch % (KBYTES / 16));
    const int k0 = (kb * KBYTES + c16 * 16) >> 1;
    const double scl = ldexp(1.0, -exp_or0(e[j])) * 64.0;
    uint32_t w0[S][4], w1[S][4];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = k0 + u;
      double2 v = make_double2(0.0, 0.0);
      if (k < K) v = B[(size_t)j * ldb + k];
      const double br = v.x * scl, bi = v.y * scl;
      // op(A) = A  : rows (br, -bi), (bi, br);  op(A) = A^H: rows (br, bi), (bi, -br)
      double a0 = br, a1 = conjA ? bi : -bi, b0 = bi, b1 = conjA ? -br : br;
#pragma unroll
      for (int p = 0; p < S; ++p) {
        const double d0 = rint(a0), d1 = rint(a1), d2 = rint(b0), d3 = rint(b1);
        const uint32_t q0 = ((uint32_t)(uint8_t)(int8_t)(int)d0) | ((uint32_t)(uint8_t)(int8_t)(int)d1 << 8);
        const uint32_t q1 = ((uint32_t)(uint8_t)(int8_t)(int)d2) | ((uint32_t)(uint8_t)(int8_t)(int)d3 << 8);
        const int word = u >> 1, sh = (u & 1) * 16;
        if (sh == 0) {
          w0[p][word] = q0;
          w1[p][word] = q1;
        } else {
          w0[p][word] |= q0 << 16;
          w1[p][word] |= q1 << 16;
        }
        a0 = (a0 - d0) * 128.0;
        a1 = (a1 - d1) * 128.0;
        b0 = (b0 - d2) * 128.0;
        b1 = (b1 - d3) * 128.0;
      }
    }
#pragma unroll
    for (int row = 0; row < 2; ++row) {
      const int r = 2 * j + row;
      const int rb = r / BN, rr = r % BN;
#pragma unroll
      for (int p = 0; p < S; ++p) {
        int8_t* tile = out + (((size_t)p * tiles_n + rb) * nkb + kb) * kBTile;
        const uint4 q = row ? make_uint4(w1[p][0], w1[p][1], w1[p][2], w1[p][3])
                            : make_uint4(w0[p][0], w0[p][1], w0[p][2], w0[p][3]);
        *reinterpret_cast<uint4*>(tile + swz(rr, c16 * 16)) = q;
      }
    }
  }
}

// run f with the slice count as a compile-time constant
template <class F> void with_slices(int s, F f) {
  switch (s) {
    case 1: f(std::integral_constant<int, 1>{}); break;
    case 2: f(std::integral_constant<int, 2>{}); break;
    case 3: f(std::integral_constant<int, 3>{}); break;
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 5: f(std::integral_constant<int, 5>{}); break;
    case 6: f(std::integral_constant<int, 6>{}); break;
    case 7: f(std::integral_constant<int, 7>{}); break;
    default: f(std::integral_constant<int, 8>{}); break;
  }
}

int grid_for(long long work, int nsm) {
  return (int)std::max<long long>(1, std::min<long long>((work + 255) / 256, 8LL * nsm));
}

}  // namespace oz

// Split A' (op(A), M x K complex) into `slices` int8 tiles with its row scales; reusable by
// every product with the same A (the projectors of a k-point).
int oz_prepare_a(OzOperand& op, bool conjA, int M, int K, const void* A, long long lda, int slices, cudaStream_t st) {
  using namespace oz;
  op.ready = false;
  if (slices < 1 || slices > kMaxSlices) return fail(kBadArg, "oz_zgemm: slices outside 1..8");
  op.M = M;
  op.K = K;
  op.s = slices;
  op.conj = conjA;
  if (M <= 0 || K <= 0) {
    op.ready = true;
    return kOk;
  }
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  op.nkb = (int)((2LL * K + KBYTES - 1) / KBYTES);
  op.tiles_m = (M + BM - 1) / BM;
  int rs;
  if ((rs = op.tiles.ensure((size_t)slices * op.tiles_m * op.nkb * kATile)) ||
      (rs = op.e.ensure(sizeof(int) * (size_t)M)))
    return rs;
  const double2* a = (const double2*)A;
  cudaError_t e0 = cudaMemsetAsync(op.e.p, 0x80, sizeof(int) * (size_t)M, st);
  if (e0 != cudaSuccess) return cuda_fail(e0, "oz_zgemm");
  if (conjA)
    k_oz_exp_cols<<<dim3((unsigned)M, (unsigned)((K + kExpChunk - 1) / kExpChunk)), 256, 0, st>>>(K, M, a, lda,
                                                                                               (int*)op.e.p);
  else
    k_oz_exp_rows<<<dim3((unsigned)((M + 255) / 256), (unsigned)((K + kExpRowChunk - 1) / kExpRowChunk)), 256, 0,
                    st>>>(M, K, a, lda, (int*)op.e.p);
  with_slices(slices, [&](auto sc) {
    k_oz_split_a<decltype(sc)::value><<<grid_for((long long)op.tiles_m * BM * op.nkb * 8, nsm), 256, 0, st>>>(
        conjA ? 1 : 0, M, K, a, lda, (const int*)op.e.p, op.tiles_m, op.nkb, (int8_t*)op.tiles.p);
  });
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "oz_zgemm splitting");
  op.ready = true;
  return kOk;
}

// C = alpha op(A) B (+ C) with op(A) prepared by oz_prepare_a
int oz_gemm_prepared(OzScratch& w, const OzOperand& op, int N, const void* B, long long ldb, double alpha,
                     bool accumulate, void* C, long long ldc, unsigned long long wait_ns, cudaStream_t st, int tri) {
  using namespace oz;
  const int M = op.M, K = op.K, s = op.s;
  if (M <= 0 || N <= 0) return kOk;
  if (!op.ready) return fail(kNotReady, "oz_zgemm: operand not prepared");
  if (tri != kOzFull && tri != kOzLowerOut && tri != kOzUpperB) return fail(kBadArg, "oz_zgemm: unknown triangular mode");
  if ((tri == kOzLowerOut && M != N) || (tri == kOzUpperB && K != N))
    return fail(kBadArg, "oz_zgemm: triangular mode needs a square operand");
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
  const int nkb = op.nkb, tiles_m = op.tiles_m;
  const int tiles_n = (2 * N + BN - 1) / BN;
  // K splits: every split at most kMaxKbPerItem K blocks; among those, the count whose waves of
  // work items over the SMs finish first (waves x K blocks per item), fewer splits on ties
  const int tiles = tiles_m * tiles_n;
  // K blocks per work item at most: the exactness bound, and a latency bound (CPW_B200_OZ_MAX_KB,
  // default kShortKb) that keeps every CTA short, so that other streams' kernels (several
  // k-points in flight) find free SMs within ~0.2 ms instead of waiting behind long items
  const int max_kb = [] {
    const char* v = getenv("CPW_B200_OZ_MAX_KB");
    const int x = v ? atoi(v) : kShortKb;
    return std::max(1, std::min(kMaxKbPerItem, x > 0 ? x : kMaxKbPerItem));
  }();
  const int nmin = std::max(1, (nkb + max_kb - 1) / max_kb);
  int nsplit = nmin;
  long long best = -1;
  for (int ns = nmin; ns <= std::min(nkb, nmin + 96); ++ns) {
    const long long kbps_t = (nkb + ns - 1) / ns;
    const long long ns_eff = (nkb + kbps_t - 1) / kbps_t;
    const long long waves = ((long long)tiles * ns_eff + nsm - 1) / nsm;
    const long long cost = waves * (kbps_t + 4);        // + the drain and partial store of an item
    if (best < 0 || cost < best) {
      best = cost;
      nsplit = (int)ns_eff;
    }
  }
  const int kbps = (nkb + nsplit - 1) / nsplit;
  nsplit = (nkb + kbps - 1) / kbps;
  const size_t bbytes = (size_t)s * tiles_n * nkb * kBTile;
  int rs;
  if ((rs = w.b.ensure(bbytes)) || (rs = w.eb.ensure(sizeof(int) * (size_t)N)) || (rs = w.err.ensure(sizeof(int))))
    return rs;
  if (!w.err_init) {
    if ((e = cudaMemsetAsync(w.err.p, 0, sizeof(int), st)) != cudaSuccess) return cuda_fail(e, "oz_zgemm");
    w.err_init = true;
  }
  if (nsplit > 1 && (rs = w.part.ensure(16 * (size_t)nsplit * M * N))) return rs;
  const double2* b = (const double2*)B;
  if ((e = cudaMemsetAsync(w.eb.p, 0x80, sizeof(int) * (size_t)N, st)) != cudaSuccess) return cuda_fail(e, "oz_zgemm");
  k_oz_exp_cols<<<dim3((unsigned)N, (unsigned)((K + kExpChunk - 1) / kExpChunk)), 256, 0, st>>>(K, N, b, ldb,
                                                                                             (int*)w.eb.p);
  with_slices(s, [&](auto sc) {
    k_oz_split_b<decltype(sc)::value><<<grid_for((long long)N * nkb * 8, nsm), 256, 0, st>>>(
        op.conj ? 1 : 0, N, K, b, ldb, (const int*)w.eb.p, tiles_n, nkb, (int8_t*)w.b.p);
  });
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "oz_zgemm splitting");
  Args g{};
  g.a = (const int8_t*)op.tiles.p;
  g.b = (const int8_t*)w.b.p;
  g.ea = (const int*)op.e.p;
  g.eb = (const int*)w.eb.p;
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
  g.tri = tri;
  g.c = (double2*)C;
  g.ldc = ldc;
  g.part = (double2*)w.part.p;
  g.err = (int*)w.err.p;
  g.wait_ns = wait_ns;
  const size_t smem = smem_bytes(s);
  if ((e = smem_limit((const void*)k_oz_gemm, smem)) != cudaSuccess) return cuda_fail(e, "oz_zgemm attribute");
  const int items = tiles * nsplit;
  // one CTA per work item: the hardware places CTAs on whichever SMs are free, so a GEMM that
  // shares the GPU with other contexts' kernels is not held up by a few late CTAs of a fixed
  // round-robin assignment (the kernel still loops when given fewer CTAs than items)
  k_oz_gemm<<<items, kThreads, smem, st>>>(g);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "oz_zgemm launch");
  if (nsplit > 1) {
    k_oz_reduce<<<grid_for((long long)M * N, nsm), 256, 0, st>>>(M, N, nsplit, (const double2*)w.part.p, alpha,
                                                                accumulate ? 1 : 0, (double2*)C, ldc);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "oz_zgemm reduce");
  }
  return kOk;
}

// C = alpha op(A) B (+ C), complex128 column-major (see the head of this file)
int oz_zgemm(OzScratch& w, bool conjA, int M, int N, int K, const void* A, long long lda, const void* B, long long ldb,
             double alpha, bool accumulate, void* C, long long ldc, int slices, unsigned long long wait_ns,
             cudaStream_t st, int tri) {
  if (M <= 0 || N <= 0) return kOk;
  if (int s = oz_prepare_a(w.aop, conjA, M, K, A, lda, slices, st)) return s;
  return oz_gemm_prepared(w, w.aop, N, B, ldb, alpha, accumulate, C, ldc, wait_ns, st, tri);
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
