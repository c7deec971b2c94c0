// Mixed-precision KB projector products on the 5th-generation tensor cores.
//
// The complex products of Src/cpw_lib/hk_psi_nl_c16.f90:82-97 written as real
// GEMMs in split TF32 (x = hi + lo, both TF32; a.b ~ hi.hi + hi.lo + lo.hi):
//
//   1. P = X^H psi:  [Re P; Im P] (2 nanl x nb) = A1 (2 nanl x 2 mtxd) . B1^T
//      A1 row a      = (xr_1, xi_1, xr_2, xi_2, ...) of projector a
//      A1 row nanl+a = (-xi_1, xr_1, ...)
//      B1 row n      = (psi_r(1,n), psi_i(1,n), ...), split by k_split_psi.
//      Split over K across work items; FP64 partials summed by k_reduce_p.
//   2. hpsi += (X D) P: (mtxd x 2 nb) = A2 (mtxd x 2 nanl) . B2^T with
//      A2 row i = (xd_r(i, :), xd_i(i, :)), B2 row 2n = (Pr(:,n), -Pi(:,n)),
//      B2 row 2n+1 = (Pi(:,n), Pr(:,n)): output columns 2n, 2n+1 are the real and
//      imaginary parts of hpsi(:, n), added in FP64.
//
// Operand layout in HBM ("tiled"): every operand is stored as 128-row x 32-float
// tiles, tile (row block rb, K block kb) at ((rb * nkb + kb) * 4096) floats, each
// tile already in the 128-byte-swizzled K-major order the tensor cores read
// (row r at r * 128 bytes, 16-byte chunk c at (c ^ (r & 7)) * 16). One pipeline
// stage is then four contiguous bulk copies (cp.async.bulk, no tensor map) of
// rows x 128 bytes, whole DRAM pages instead of 128-byte pieces of 128 rows.
//
// Kernel (persistent: grid <= SM count, work items = output tile x K range, 18 warps):
//   warp 0      producer: bulk copies of A hi/lo and B hi/lo into a 3-stage ring
//               (full/empty mbarriers);
//   warp 1      allocates 512 TMEM columns; one lane issues tcgen05.mma kind::tf32
//               (M 128, N <= 128, K 8): hi.hi into one of three rotating main
//               accumulators, restarted every `chain` K blocks; hi.lo and lo.hi into
//               a correction accumulator that spans the whole work item;
//   warps 2-17  drain: they read each finished main accumulator with tcgen05.ld and
//               add it into FP64 sums in registers (one row and 32 columns per
//               thread), release it, add the correction accumulator at the end of
//               the work item, and store the tile.
// The FP32 accumulation of the tensor cores shrinks a sum by a fixed fraction per
// accumulation step (measured: ~5e-7 relative on coherent sums over 16 steps), a
// bias, not noise. Restarting the hi.hi accumulator every K block (4 steps) keeps it
// near 1e-7; the correction terms are 2^-11 of the total, so their long chain adds
// nothing visible; the drain sums in FP64. Every mbarrier wait is bounded in time: on
// timeout the kernel sets an error flag, skips its stores, waits (bounded) for its
// copies and MMAs in flight, frees its TMEM and returns.
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>

#include "context.hpp"

namespace cpwb {
namespace tc {

constexpr int BM = 128, BN = 128, BK = 32;
constexpr int kStages = 3;
constexpr int kTileFloats = BM * BK;               // 4096 floats = 16 KB
constexpr int kTileBytes = kTileFloats * 4;
constexpr int kStageBytes = 4 * kTileBytes;        // A hi, A lo, B hi, B lo
constexpr int kDrainWarps = 16;                   // 4 lane quarters x 4 column slices
constexpr int kDrainCols = BN / (kDrainWarps / 4); // accumulator columns per drain thread
constexpr int kThreads = 32 * (2 + kDrainWarps);
constexpr int kBarBytes = 256;
constexpr int kPrefetch = 8;                       // K blocks fetched into L2 ahead of the shared-memory copies
constexpr int kEpiBytes = 1024;                    // per drain warp: 2 complex columns x 32 rows of FP64 staging
constexpr int kEpiCplx = kEpiBytes / (32 * 16);
constexpr int kSmemBytes = kStages * kStageBytes + 1024 + kBarBytes + kDrainWarps * kEpiBytes;
constexpr unsigned long long kWaitNs = 2000000000ull;   // 2 s per mbarrier wait at most
constexpr int kMainBufs = 3;                       // rotating hi.hi accumulators
constexpr int kTmemCols = 512;                     // correction 128 + 3 x hi.hi 128 (+128 unused)

// float offset of element (r, k) of a tiled operand with nkb K blocks
__host__ __device__ __forceinline__ size_t tiled_off(long long r, long long k, long long nkb) {
  return (size_t)(((r >> 7) * nkb + (k >> 5)) * kTileFloats) + (size_t)((r & 127) * 32) +
         (size_t)(((((k >> 2) & 7) ^ (r & 7)) << 2) | (k & 3));
}

struct GemmArgs {
  const float* a_hi;           // tiled, rows M (padded to 128), nkb K blocks
  const float* a_lo;
  const float* b_hi;           // tiled, rows N
  const float* b_lo;
  int M, N;                    // output rows / columns
  int nkb;                     // 32-wide K blocks in total
  int kb_per_split;            // K blocks per work item
  int nsplit;
  int chain;                   // K blocks per FP32 accumulation chain
  int tiles_m, tiles_n;
  int n_fast;                  // tile order: 1 = consecutive items share an m tile
  int terms;                   // 3: hi.hi + hi.lo + lo.hi; 4: also lo.lo
  double* out;                 // mode 0: out[split][n][M]; mode 1: complex128 hpsi, ld ldh
  long long ldh;
  int* err;
  unsigned long long wait_ns;  // limit of the hand-off waits between the roles
};

struct Item {
  int m0, n0, split, kb0, nblk, rows_a, rows_b, n_mma;
};

__device__ __forceinline__ Item item_of(const GemmArgs& g, int it) {
  Item w;
  const int tiles = g.tiles_m * g.tiles_n;
  w.split = it / tiles;
  const int tile = it - w.split * tiles;
  int mt, nt;
  if (g.n_fast) {
    nt = tile % g.tiles_n;
    mt = tile / g.tiles_n;
  } else {
    mt = tile % g.tiles_m;
    nt = tile / g.tiles_m;
  }
  w.m0 = mt * BM;
  w.n0 = nt * BN;
  w.kb0 = w.split * g.kb_per_split;
  w.nblk = max(0, min(g.nkb, w.kb0 + g.kb_per_split) - w.kb0);
  w.rows_a = min(BM, g.M - w.m0);
  w.rows_b = min(BN, g.N - w.n0);
  w.n_mma = min(BN, ((w.rows_b + 15) / 16) * 16);
  return w;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ float tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// K-major operand tile, 128-byte swizzle: 8-row groups 1024 bytes apart
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);               // start address
  d |= (uint64_t)1 << 16;                               // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)((1024 >> 4) & 0x3FFF) << 32;          // stride byte offset: 8 rows x 128 B
  d |= (uint64_t)1 << 46;                               // descriptor version
  d |= (uint64_t)2 << 61;                               // 128-byte swizzle
  return d;
}

__device__ __forceinline__ uint32_t instr_desc(int n) {
  return (1u << 4)                  // D format F32
         | (2u << 7)                // A TF32
         | (2u << 10)               // B TF32
         | ((uint32_t)(n >> 3) << 17)
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

// wait bounded in time (limit_ns); gives up early once another role has recorded a failure.
// The hand-offs between the roles use the caller's limit (GemmArgs::wait_ns, 2 s unless a
// failure-detection test shortens it); the waits for copies and MMAs already issued, before the
// CTA exits, always use kWaitNs: those complete on their own.
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

__device__ __forceinline__ void prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(src), "r"(bytes) : "memory");
}

// global[dst .. dst+bytes) += shared[src ..] in FP64, performed by the memory system
__device__ __forceinline__ void bulk_add_f64(void* dst, uint32_t src, uint32_t bytes) {
  asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], %2;\n" ::"l"(dst), "r"(src),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, 1) k_gemm_tf32x3(const GemmArgs g) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* tiles = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = reinterpret_cast<uint64_t*>(tiles + kStages * kStageBytes);
  uint64_t* full = bars;                     // [kStages] copies landed
  uint64_t* empty = bars + kStages;          // [kStages] MMAs that read the stage are done
  uint64_t* accf = bars + 2 * kStages;       // [kMainBufs] hi.hi accumulator ready for the drain
  uint64_t* acce = accf + kMainBufs;         // [kMainBufs] hi.hi accumulator drained
  uint64_t* corre = acce + kMainBufs;        // correction accumulator drained (end of a work item)
  uint64_t* done = corre + 1;                // all MMAs of this CTA complete
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  unsigned char* epi = tiles + kStages * kStageBytes + kBarBytes;   // drain-warp staging (mode 1)
  __shared__ volatile int failed;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nitems = g.tiles_m * g.tiles_n * g.nsplit;
  const int chain = max(1, g.chain);
  const size_t nkb = (size_t)g.nkb;

  if (threadIdx.x == 0) {
    failed = 0;
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    for (int b = 0; b < kMainBufs; ++b) {
      mbar_init(smem_u32(&accf[b]), 1);
      mbar_init(smem_u32(&acce[b]), kDrainWarps);
    }
    mbar_init(smem_u32(corre), kDrainWarps);
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
      long long gk = 0;                      // K blocks issued by this CTA (ring position)
      for (int it = blockIdx.x; it < nitems && !failed; it += gridDim.x) {
        const Item w = item_of(g, it);
        const float* ah = g.a_hi + (size_t)(w.m0 >> 7) * nkb * kTileFloats;
        const float* al = g.a_lo + (size_t)(w.m0 >> 7) * nkb * kTileFloats;
        const float* bh = g.b_hi + (size_t)(w.n0 >> 7) * nkb * kTileFloats;
        const float* bl = g.b_lo + (size_t)(w.n0 >> 7) * nkb * kTileFloats;
        const uint32_t bytes_a = (uint32_t)w.rows_a * 128u, bytes_b = (uint32_t)w.rows_b * 128u;
        auto prefetch = [&](int i) {
          const size_t o = (size_t)(w.kb0 + i) * kTileFloats;
          prefetch_l2(ah + o, bytes_a);
          prefetch_l2(al + o, bytes_a);
          prefetch_l2(bh + o, bytes_b);
          prefetch_l2(bl + o, bytes_b);
        };
        for (int i = 0; i < min(kPrefetch, w.nblk); ++i) prefetch(i);
        for (int i = 0; i < w.nblk; ++i, ++gk) {
          if (i + kPrefetch < w.nblk) prefetch(i + kPrefetch);
          const int s = (int)(gk % kStages);
          const long long r = gk / kStages;
          if (r > 0 && !mbar_wait(smem_u32(&empty[s]), (uint32_t)((r - 1) & 1), &failed, g.wait_ns)) {
            failed = 1;
            atomicExch(g.err, 1);
            break;
          }
          unsigned char* st = tiles + s * kStageBytes;
          const uint32_t fb = smem_u32(&full[s]);
          mbar_expect_tx(fb, 2u * (bytes_a + bytes_b));
          const size_t o = (size_t)(w.kb0 + i) * kTileFloats;
          bulk_load(smem_u32(st), ah + o, bytes_a, fb);
          bulk_load(smem_u32(st + kTileBytes), al + o, bytes_a, fb);
          bulk_load(smem_u32(st + 2 * kTileBytes), bh + o, bytes_b, fb);
          bulk_load(smem_u32(st + 3 * kTileBytes), bl + o, bytes_b, fb);
        }
      }
      // copies still in flight land before the CTA may exit
      for (long long i = (gk > kStages ? gk - kStages : 0); i < gk; ++i)
        if (!mbar_wait(smem_u32(&full[i % kStages]), (uint32_t)((i / kStages) & 1), nullptr)) atomicExch(g.err, 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      long long gk = 0;                      // K blocks consumed
      long long gq = 0;                      // accumulation chunks issued
      int nit = 0;                           // work items of this CTA so far
      const uint32_t tcorr = tmem;           // columns [0, 128): hi.lo + lo.hi of the whole work item
      for (int it = blockIdx.x; it < nitems && !failed; it += gridDim.x, ++nit) {
        const Item w = item_of(g, it);
        const uint32_t idesc = instr_desc(w.n_mma);
        const int nchunk = (w.nblk + chain - 1) / chain;
        // the previous work item's correction accumulator must have been read
        if (nit > 0 && !mbar_wait(smem_u32(corre), (uint32_t)((nit - 1) & 1), &failed, g.wait_ns)) {
          failed = 1;
          atomicExch(g.err, 1);
          break;
        }
        for (int q = 0; q < nchunk && !failed; ++q, ++gq) {
          const int b = (int)(gq % kMainBufs);
          if (gq >= kMainBufs &&
              !mbar_wait(smem_u32(&acce[b]), (uint32_t)((gq / kMainBufs - 1) & 1), &failed, g.wait_ns)) {
            failed = 1;
            atomicExch(g.err, 1);
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;\n");
          // hi.hi accumulator b: columns [128 (b + 1), +n_mma)
          const uint32_t tmain = tmem + (uint32_t)((b + 1) * BN);
          const int i0 = q * chain, i1 = min(w.nblk, i0 + chain);
          bool ok = true;
          for (int i = i0; i < i1; ++i, ++gk) {
            const int s = (int)(gk % kStages);
            if (!mbar_wait(smem_u32(&full[s]), (uint32_t)((gk / kStages) & 1), &failed, g.wait_ns)) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n");
            unsigned char* st = tiles + s * kStageBytes;
            const uint32_t ah = smem_u32(st), al = smem_u32(st + kTileBytes);
            const uint32_t bh = smem_u32(st + 2 * kTileBytes), bl = smem_u32(st + 3 * kTileBytes);
#pragma unroll
            for (int ks = 0; ks < BK / 8; ++ks) {
              const uint32_t off = ks * 32;     // 8 tf32 = 32 bytes along K inside the swizzled row
              const uint32_t acc = (i == i0 && ks == 0) ? 0u : 1u;
              const uint32_t accc = (i == 0 && ks == 0) ? 0u : 1u;
              mma_tf32(tmain, smem_desc(ah + off), smem_desc(bh + off), idesc, acc);    // hi.hi
              mma_tf32(tcorr, smem_desc(ah + off), smem_desc(bl + off), idesc, accc);   // hi.lo
              mma_tf32(tcorr, smem_desc(al + off), smem_desc(bh + off), idesc, 1u);     // lo.hi
              if (g.terms > 3) mma_tf32(tcorr, smem_desc(al + off), smem_desc(bl + off), idesc, 1u);
            }
            mma_commit(smem_u32(&empty[s]));
          }
          if (!ok) {
            failed = 1;
            atomicExch(g.err, 1);
            break;
          }
          mma_commit(smem_u32(&accf[b]));
        }
      }
      // every MMA of this thread completes before TMEM is freed
      mma_commit(smem_u32(done));
      if (!mbar_wait(smem_u32(done), 0u, nullptr)) atomicExch(g.err, 1);
    }
  } else {
    const int quarter = warp & 3, slice = (warp - 2) >> 2;
    const uint32_t lane_base = tmem + ((uint32_t)(32 * quarter) << 16);
    long long gq = 0;
    for (int it = blockIdx.x; it < nitems && !failed; it += gridDim.x) {
      const Item w = item_of(g, it);
      const int nchunk = (w.nblk + chain - 1) / chain;
      double acc[kDrainCols];
#pragma unroll
      for (int j = 0; j < kDrainCols; ++j) acc[j] = 0.0;
      bool ok = true;
      for (int q = 0; q < nchunk; ++q, ++gq) {
        const int b = (int)(gq % kMainBufs);
        if (!mbar_wait(smem_u32(&accf[b]), (uint32_t)((gq / kMainBufs) & 1), &failed, g.wait_ns)) {
          ok = false;
          failed = 1;
          atomicExch(g.err, 1);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n");
        const bool last = q == nchunk - 1;
        // the last chunk's commit also covers every correction MMA of the item: drain it too
        for (int pass = 0; pass < (last ? 2 : 1); ++pass) {
          const uint32_t col0 = pass == 0 ? (uint32_t)((b + 1) * BN) : 0u;
#pragma unroll
          for (int j = 0; j < kDrainCols / 8; ++j) {
            const int col = kDrainCols * slice + 8 * j;
            if (col < w.n_mma) {        // n_mma is a multiple of 16: whole 8-column pieces
              uint32_t r[8];
              tmem_ld8(lane_base + col0 + (uint32_t)col, r);
              asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
              for (int t = 0; t < 8; ++t) acc[8 * j + t] += (double)__uint_as_float(r[t]);
            }
          }
          asm volatile("tcgen05.fence::before_thread_sync;\n");
          __syncwarp();
          if (lane == 0) mbar_arrive(smem_u32(pass == 0 ? &acce[b] : corre));
        }
      }
      if (!ok || failed) break;
#define CPWB_ACC(j) (acc[j])
      const int m = w.m0 + 32 * quarter + lane;
      if (nchunk > 0 && w.m0 + 32 * quarter < g.M) {      // warp-uniform: the warp has valid rows
#pragma unroll
        for (int j = 0; j < kDrainCols / 16; ++j) {
          const int col = kDrainCols * slice + 16 * j;
          if (col < w.n_mma) {
            if (MODE == 0) {
#pragma unroll
              for (int t = 0; t < 16; ++t) {
                const int n = w.n0 + col + t;
                if (n < g.N && m < g.M) g.out[((size_t)w.split * g.N + n) * g.M + m] = CPWB_ACC(16 * j + t);
              }
            } else {
              // kEpiCplx complex columns at a time through this warp's staging slot: [column][32 rows]
              // of (re, im), then one bulk FP64 add of 32 rows (512 contiguous bytes of hpsi) per column
              double2* slot = reinterpret_cast<double2*>(epi + (warp - 2) * kEpiBytes);
              const int rows = min(32, g.M - (w.m0 + 32 * quarter));
#pragma unroll
              for (int hh = 0; hh < 8 / kEpiCplx; ++hh) {
                const int c0 = w.n0 + col + 2 * kEpiCplx * hh;   // first real output column of the round
                // the previous bulk adds must have finished reading the slot
                asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
                __syncwarp();
#pragma unroll
                for (int t = 0; t < kEpiCplx; ++t)
                  slot[t * 32 + lane] = make_double2(CPWB_ACC(16 * j + 2 * kEpiCplx * hh + 2 * t),
                                                     CPWB_ACC(16 * j + 2 * kEpiCplx * hh + 2 * t + 1));
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                __syncwarp();
                if (lane == 0) {
                  for (int t = 0; t < kEpiCplx; ++t)
                    if (c0 + 2 * t + 1 < g.N)
                      bulk_add_f64(reinterpret_cast<double2*>(g.out) + (size_t)((c0 >> 1) + t) * g.ldh + (m - lane),
                                   smem_u32(slot + t * 32), (uint32_t)rows * 16u);
                  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
                }
              }
            }
          }
        }
      }
    }
  }
#undef CPWB_ACC
  if (MODE == 1 && warp >= 2 && lane == 0) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;\n");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols));
  }
}

__device__ __forceinline__ void put_split(float* hi, float* lo, size_t o, double v0, double v1) {
  const float h0 = tf32((float)v0), h1 = tf32((float)v1);
  *reinterpret_cast<float2*>(hi + o) = make_float2(h0, h1);
  *reinterpret_cast<float2*>(lo + o) = make_float2(tf32((float)(v0 - (double)h0)), tf32((float)(v1 - (double)h1)));
}

// B1 (nb rows, K = 2 mtxd reals, tiled): row n = interleaved psi(:, n), zero beyond 2 mtxd
__global__ void k_split_psi(int nb, int mtxd, long long nkb, const C2<double>* __restrict__ psi, long long ldpsi,
                            float* __restrict__ hi, float* __restrict__ lo) {
  const long long pairs = nkb * 16;                    // complex entries per padded row
  const long long n = (long long)nb * pairs;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long r = t / pairs, i = t - r * pairs;
    C2<double> z = mk(0.0, 0.0);
    if (i < mtxd) z = psi[(size_t)r * ldpsi + i];
    put_split(hi, lo, tiled_off(r, 2 * i, nkb), z.x, z.y);
  }
}

// A1 (2 nanl rows, K = 2 mtxd, tiled) from X (anl, complex128 ld mtxd)
__global__ void k_prep_a1(int mtxd, int nanl, long long nkb, const C2<double>* __restrict__ x, float* __restrict__ hi,
                          float* __restrict__ lo) {
  const long long pairs = nkb * 16;
  const long long n = 2LL * nanl * pairs;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long row = t / pairs, i = t - row * pairs;
    const int a = (int)(row % nanl);
    C2<double> z = mk(0.0, 0.0);
    if (i < mtxd) z = x[(size_t)a * mtxd + i];
    if (row < nanl)
      put_split(hi, lo, tiled_off(row, 2 * i, nkb), z.x, z.y);
    else
      put_split(hi, lo, tiled_off(row, 2 * i, nkb), -z.y, z.x);
  }
}

// A2 (mtxd rows, K = 2 nanl, tiled) from X D (anld): row i = (xd_r(i, :), xd_i(i, :))
__global__ void k_prep_a2(int mtxd, int nanl, long long nkb, const C2<double>* __restrict__ xd, float* __restrict__ hi,
                          float* __restrict__ lo) {
  const long long pairs = nkb * 16;                    // K pairs per padded row
  const long long n = (long long)mtxd * pairs;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / pairs, k = 2 * (t - i * pairs);
    double v[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const long long kk = k + e;
      v[e] = 0.0;
      if (kk < 2 * nanl) {
        const int a = (int)(kk % nanl);
        const C2<double> z = xd[(size_t)a * mtxd + i];
        v[e] = kk < nanl ? z.x : z.y;
      }
    }
    put_split(hi, lo, tiled_off(i, k, nkb), v[0], v[1]);
  }
}

// A (m rows, K = 2 kk, tiled) from a complex128 column-major matrix a (ld lda): row i = (re a(i, :), im a(i, :))
__global__ void k_prep_arows(int m, int kk, long long lda, long long nkb, const C2<double>* __restrict__ a,
                             float* __restrict__ hi, float* __restrict__ lo) {
  const long long pairs = nkb * 16;
  const long long n = (long long)m * pairs;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    // consecutive threads take consecutive rows i (coalesced reads down a column)
    const long long i = t % m, k = 2 * (t / m);
    double v[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const long long kk2 = k + e;
      v[e] = 0.0;
      if (kk2 < 2LL * kk) {
        const long long l = kk2 % kk;
        const C2<double> z = a[(size_t)l * lda + i];
        v[e] = kk2 < kk ? z.x : z.y;
      }
    }
    put_split(hi, lo, tiled_off(i, k, nkb), v[0], v[1]);
  }
}

// B (2 n rows, K = 2 kk, tiled) from a complex128 kk x n matrix b (ld ldb):
// row 2j = (re b(:, j), -im b(:, j)), row 2j+1 = (im b(:, j), re b(:, j))
__global__ void k_prep_bcols(int kk, int n, long long ldb, long long nkb, const C2<double>* __restrict__ b,
                             float* __restrict__ hi, float* __restrict__ lo) {
  const long long kpad = nkb * 32;
  const long long total = (long long)n * kpad;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const long long j = t / kpad, k = t - j * kpad;
    double ev = 0.0, od = 0.0;
    if (k < 2LL * kk) {
      const long long l = k % kk;
      const C2<double> z = b[(size_t)j * ldb + l];
      ev = k < kk ? z.x : -z.y;
      od = k < kk ? z.y : z.x;
    }
    auto put = [&](long long row, double v) {
      const float h = tf32((float)v);
      const size_t o = tiled_off(row, k, nkb);
      hi[o] = h;
      lo[o] = tf32((float)(v - (double)h));
    };
    put(2 * j, ev);
    put(2 * j + 1, od);
  }
}

// P from the FP64 split-K partials part[z][n][2 nanl]; B2 (2 nb rows, K = 2 nanl, tiled):
// row 2n = (Pr, -Pi), row 2n+1 = (Pi, Pr). K entries beyond 2 nanl are cleared by the caller.
__global__ void k_reduce_p(int nanl, int nb, int nsplit, long long nkb, const double* __restrict__ part,
                           float* __restrict__ hi, float* __restrict__ lo) {
  const long long n = (long long)nanl * nb;
  const long long m2 = 2LL * nanl;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long a = t % nanl, b = t / nanl;
    double pr = 0.0, pi = 0.0;
    for (int z = 0; z < nsplit; ++z) {
      const double* pz = part + ((size_t)z * nb + b) * m2;
      pr += pz[a];
      pi += pz[nanl + a];
    }
    auto put = [&](long long row, long long k, double v) {
      const float h = tf32((float)v);
      const size_t o = tiled_off(row, k, nkb);
      hi[o] = h;
      lo[o] = tf32((float)(v - (double)h));
    };
    put(2 * b, a, pr);
    put(2 * b, nanl + a, -pi);
    put(2 * b + 1, a, pi);
    put(2 * b + 1, nanl + a, pr);
  }
}

inline size_t tiled_floats(long long rows, long long nkb) { return (size_t)((rows + 127) / 128) * nkb * kTileFloats; }

}  // namespace tc

namespace {

int env_int(const char* name, int dflt) {
  const char* v = getenv(name);
  return v ? atoi(v) : dflt;
}

int grid_for(long long work, int nsm) {
  return (int)std::max(1LL, std::min((long long)(8 * nsm), (work + 255) / 256));
}

}  // namespace

// the sticky error flag of the tensor-core kernels: zeroed when allocated, read and cleared by
// tc_check_error (a bounded wait that gave up in any launch since the last check reports)
int tc_error_flag(TcScratch& t) {
  if (t.err.p) return kOk;
  if (int s = t.err.ensure(sizeof(int))) return s;
  cudaError_t e = cudaMemset(t.err.p, 0, sizeof(int));
  return e == cudaSuccess ? kOk : cuda_fail(e, "tc error flag");
}

int tc_read_error(TcScratch& t) {
  if (!t.err.p) return kOk;
  int h = 0;
  cudaError_t e = cudaMemcpy(&h, t.err.p, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "tc error flag");
  if (!h) return kOk;
  cudaMemset(t.err.p, 0, sizeof(int));
  return fail(kTimeout, "tensor-core GEMM: an mbarrier wait gave up");
}

int tc_prepare_operands(int m, int na, const void* anl, const void* anld, DevBuf& a1buf, DevBuf& a2buf,
                        long long* nkb1_out, long long* nkb2_out, cudaStream_t st) {
  if (na == 0 || m == 0) return kOk;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long nkb1 = (2LL * m + tc::BK - 1) / tc::BK;
  const long long nkb2 = (2LL * na + tc::BK - 1) / tc::BK;
  const size_t fa1 = tc::tiled_floats(2 * na, nkb1), fa2 = tc::tiled_floats(m, nkb2);
  int s;
  if ((s = a1buf.ensure(sizeof(float) * 2 * fa1)) || (s = a2buf.ensure(sizeof(float) * 2 * fa2))) return s;
  float* a1 = (float*)a1buf.p;
  float* a2 = (float*)a2buf.p;
  tc::k_prep_a1<<<grid_for(2LL * na * nkb1 * 16, nsm), 256, 0, st>>>(m, na, nkb1, (const C2<double>*)anl, a1, a1 + fa1);
  tc::k_prep_a2<<<grid_for((long long)m * nkb2 * 16, nsm), 256, 0, st>>>(m, na, nkb2, (const C2<double>*)anld, a2,
                                                                          a2 + fa2);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "tensor-core projector preparation");
  *nkb1_out = nkb1;
  *nkb2_out = nkb2;
  return kOk;
}

int tc_prepare_projectors(cpw_b200_ctx* c) {
  if (c->nanl == 0 || c->mtxd == 0) return kOk;
  int s = tc_prepare_operands(c->mtxd, c->nanl, c->anl.p, c->anld.p, c->tc_a1, c->tc_a2, &c->tc_k1p, &c->tc_k2p,
                              c->stream);
  if (s) return s;
  c->tc_ready = true;
  return kOk;
}

// hpsi += X D X^H psi in split TF32 on the tensor cores (hpsi already holds the local part);
// a1/a2 are the tiled operands of tc_prepare_operands for (m, na); scratch and the error
// flag are the context's
int tc_nl_apply_ops(TcScratch& t, int m, int na, long long nkb1, long long nkb2, const float* a1, const float* a2,
                    int nb, const void* psi, long long ldpsi, void* hpsi, long long ldh, cudaStream_t st,
                    cudaEvent_t t0, cudaEvent_t t1, cudaEvent_t t2, int splits) {
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int chain = std::max(1, env_int("CPW_B200_TC_CHAIN", 1));
  const int terms = env_int("CPW_B200_TC_TERMS", 3) == 4 ? 4 : 3;

  // GEMM 1: (2 nanl) x nb, K = 2 mtxd, split over K so that the work items fill the SMs about once
  const int mt1 = (2 * na + tc::BM - 1) / tc::BM, nt1 = (nb + tc::BN - 1) / tc::BN;
  // splits: 0 = the split with the fewest waves per unit of K (ceil(tiles s / nsm) / s, a
  // smaller s unless a larger one is 3% better: Si64 8 tiles -> 18 splits, one wave; Si216
  // 56 tiles -> 21 splits, 8 waves at 99% of the SMs instead of 2 splits on 112 of 148),
  // > 0 that many, -d a d-th of the default
  int nsplit = 1;
  {
    const long long tiles = (long long)mt1 * nt1;
    const long long smax = std::max(1LL, std::min<long long>(nkb1, 16LL * nsm / tiles + 1));
    double best = 1e300;
    for (long long sp = 1; sp <= smax; ++sp) {
      const double cost = (double)((tiles * sp + nsm - 1) / nsm) / (double)sp;
      if (cost < best * 0.97) {
        best = cost;
        nsplit = (int)sp;
      }
    }
  }
  if (splits < 0) nsplit = std::max(1, nsplit / -splits);
  if (splits > 0) nsplit = (int)std::min<long long>(nkb1, splits);
  if (const int ks = env_int("CPW_B200_TC_SPLITS", 0)) nsplit = (int)std::max(1LL, std::min<long long>(nkb1, ks));
  const int kbps = (int)((nkb1 + nsplit - 1) / nsplit);
  nsplit = (int)((nkb1 + kbps - 1) / kbps);
  const size_t fb1 = tc::tiled_floats(nb, nkb1), fb2 = tc::tiled_floats(2 * nb, nkb2);
  int s;
  if ((s = t.b1.ensure(sizeof(float) * 2 * fb1)) ||
      (s = t.part.ensure(sizeof(double) * (size_t)nsplit * nb * 2 * na)) ||
      (s = t.b2.ensure(sizeof(float) * 2 * fb2)) || (s = tc_error_flag(t)))
    return s;
  float* b1 = (float*)t.b1.p;
  float* b2 = (float*)t.b2.p;
  const size_t fa1 = tc::tiled_floats(2 * na, nkb1), fa2 = tc::tiled_floats(m, nkb2);

  tc::GemmArgs g1{};
  g1.a_hi = a1;
  g1.a_lo = a1 + fa1;
  g1.b_hi = b1;
  g1.b_lo = b1 + fb1;
  g1.M = 2 * na;
  g1.N = nb;
  g1.nkb = (int)nkb1;
  g1.kb_per_split = kbps;
  g1.nsplit = nsplit;
  g1.chain = chain;
  g1.tiles_m = mt1;
  g1.tiles_n = nt1;
  g1.n_fast = 0;
  g1.terms = terms;
  g1.out = (double*)t.part.p;
  g1.err = (int*)t.err.p;
  g1.wait_ns = t.wait_ns;

  // GEMM 2: mtxd x (2 nb), K = 2 nanl, added into hpsi
  const int mt2 = (m + tc::BM - 1) / tc::BM, nt2 = (2 * nb + tc::BN - 1) / tc::BN;
  tc::GemmArgs g2{};
  g2.a_hi = a2;
  g2.a_lo = a2 + fa2;
  g2.b_hi = b2;
  g2.b_lo = b2 + fb2;
  g2.M = m;
  g2.N = 2 * nb;
  g2.nkb = (int)nkb2;
  g2.kb_per_split = (int)nkb2;
  g2.nsplit = 1;
  g2.chain = chain;
  g2.tiles_m = mt2;
  g2.tiles_n = nt2;
  g2.n_fast = 1;
  g2.terms = terms;
  g2.out = (double*)hpsi;
  g2.ldh = ldh;
  g2.err = (int*)t.err.p;
  g2.wait_ns = t.wait_ns;

  cudaError_t e;
  if ((e = smem_limit((const void*)tc::k_gemm_tf32x3<0>, (size_t)tc::kSmemBytes)) != cudaSuccess ||
      (e = smem_limit((const void*)tc::k_gemm_tf32x3<1>, (size_t)tc::kSmemBytes)) != cudaSuccess)
    return cuda_fail(e, "tensor-core GEMM attribute");
  const int items1 = mt1 * nt1 * nsplit, items2 = mt2 * nt2;
  if (t0) cudaEventRecord(t0, st);
  tc::k_split_psi<<<grid_for((long long)nb * nkb1 * 16, nsm), 256, 0, st>>>(nb, m, nkb1, (const C2<double>*)psi, ldpsi,
                                                                             b1, b1 + fb1);
  // one CTA per work item: the hardware places CTAs on whichever SMs are free, so a GEMM that
  // shares the GPU with other contexts' kernels is not held up by a few late CTAs of a fixed
  // round-robin assignment
  tc::k_gemm_tf32x3<0><<<items1, tc::kThreads, tc::kSmemBytes, st>>>(g1);
  if ((2LL * na) % tc::BK) {
    if ((e = cudaMemsetAsync(b2, 0, sizeof(float) * 2 * fb2, st)) != cudaSuccess) return cuda_fail(e, "tc nl");
  }
  tc::k_reduce_p<<<grid_for((long long)na * nb, nsm), 256, 0, st>>>(na, nb, nsplit, nkb2, (const double*)t.part.p,
                                                                    b2, b2 + fb2);
  if (t1) cudaEventRecord(t1, st);
  tc::k_gemm_tf32x3<1><<<items2, tc::kThreads, tc::kSmemBytes, st>>>(g2);
  if (t2) cudaEventRecord(t2, st);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "tensor-core projector GEMMs");
  return kOk;
}

int tc_nl_apply(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, void* hpsi, long long ldh, cudaStream_t st,
                cudaEvent_t t0, cudaEvent_t t1, cudaEvent_t t2) {
  if (!c->tc_ready) return fail(kNotReady, "tensor-core projectors not prepared");
  return tc_nl_apply_ops(c->tcs, c->mtxd, c->nanl, c->tc_k1p, c->tc_k2p, (const float*)c->tc_a1.p,
                         (const float*)c->tc_a2.p, nb, psi, ldpsi, hpsi, ldh, st, t0, t1, t2);
}

// C (m x n) = A (m x kk) B (kk x n) (accumulate: C += A B), complex128 column-major, in split TF32
// on the tensor cores
int tc_zgemm_nn(cpw_b200_ctx* c, int m, int n, int kk, const void* a, long long lda, const void* b, long long ldb,
                void* cm, long long ldc, cudaStream_t st, bool accumulate) {
  if (m <= 0 || n <= 0) return kOk;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e = cudaSuccess;
  if (!accumulate)
    e = cudaMemset2DAsync(cm, sizeof(C2<double>) * (size_t)ldc, 0, sizeof(C2<double>) * (size_t)m, n, st);
  if (e != cudaSuccess) return cuda_fail(e, "tc zgemm");
  if (kk <= 0) return kOk;
  const long long nkb = (2LL * kk + tc::BK - 1) / tc::BK;
  const size_t fa = tc::tiled_floats(m, nkb), fb = tc::tiled_floats(2LL * n, nkb);
  int s;
  if ((s = c->tc_ga.ensure(sizeof(float) * 2 * fa)) || (s = c->tc_gb.ensure(sizeof(float) * 2 * fb)) ||
      (s = tc_error_flag(c->tcs)))
    return s;
  float* ga = (float*)c->tc_ga.p;
  float* gb = (float*)c->tc_gb.p;
  tc::k_prep_arows<<<grid_for((long long)m * nkb * 16, nsm), 256, 0, st>>>(m, kk, lda, nkb, (const C2<double>*)a, ga,
                                                                           ga + fa);
  tc::k_prep_bcols<<<grid_for((long long)n * nkb * 32, nsm), 256, 0, st>>>(kk, n, ldb, nkb, (const C2<double>*)b, gb,
                                                                           gb + fb);
  const int mt = (m + tc::BM - 1) / tc::BM, nt = (2 * n + tc::BN - 1) / tc::BN;
  tc::GemmArgs g{};
  g.a_hi = ga;
  g.a_lo = ga + fa;
  g.b_hi = gb;
  g.b_lo = gb + fb;
  g.M = m;
  g.N = 2 * n;
  g.nkb = (int)nkb;
  g.kb_per_split = (int)nkb;
  g.nsplit = 1;
  g.chain = std::max(1, env_int("CPW_B200_TC_CHAIN", 1));
  g.tiles_m = mt;
  g.tiles_n = nt;
  g.n_fast = 1;
  g.terms = 3;
  g.out = (double*)cm;
  g.ldh = ldc;
  g.err = (int*)c->tcs.err.p;
  g.wait_ns = c->tcs.wait_ns;
  if ((e = smem_limit((const void*)tc::k_gemm_tf32x3<1>, (size_t)tc::kSmemBytes)) != cudaSuccess)
    return cuda_fail(e, "tensor-core GEMM attribute");
  tc::k_gemm_tf32x3<1><<<mt * nt, tc::kThreads, tc::kSmemBytes, st>>>(g);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "tensor-core zgemm");
  return kOk;
}

int tc_check_error(cpw_b200_ctx* c) {
  if (int s = tc_read_error(c->tcs)) return s;
  return oz_read_error(c->ozs);
}

namespace tc {
// Failure-detection self-test: one thread waits, through the same bounded wait as the GEMM
// roles, on an mbarrier that nothing arrives at; when the limit runs out it sets the sticky
// error flag and the kernel returns.
__global__ void k_wait_selftest(int* err, unsigned long long limit_ns) {
  __shared__ alignas(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(smem_u32(&bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(smem_u32(&bar), 0u, nullptr, limit_ns)) atomicExch(err, 1);
}
}  // namespace tc

int tc_wait_selftest(cpw_b200_ctx* c, unsigned long long limit_ns, cudaStream_t st) {
  if (int s = tc_error_flag(c->tcs)) return s;
  tc::k_wait_selftest<<<1, 32, 0, st>>>((int*)c->tcs.err.p, limit_ns);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? kOk : cuda_fail(e, "wait self-test launch");
}

}  // namespace cpwb
