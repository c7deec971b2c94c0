// Batched H|psi> over the k-points of one crystal (one FFT box, one potential).
//
// The reference applies H k-point by k-point (Src/cpw_lib/cpw_scf.f90:488 drives
// h_kb_dia -> ditsp_c16 -> hk_psi_c16 once per k). Here the bands of every k-point
// of a batch go through the local kernels together: the batch has one kept-plane /
// kept-row set (the union of the k-points' spheres), each k-point its own plane
// lists and kinetic diagonal relative to it, and the local kernels A and C read a
// per-band table (k-point, band) and a per-k descriptor, so one launch per stage
// covers all k-points and uneven plane-wave counts and band counts (kernel B only
// sees slabs). The projector products (each k has its own X) run for all k-points in three
// FP64 launches when the blocks are small (below; in every precision form: for blocks this small
// a tensor-core GEMM pipeline per k-point is mostly fixed cost), else per k-point: cuBLAS ZGEMMs
// in FP64 / MIXED, the split-TF32 tensor-core kernels in MIXED_TC.
//
// The first call for a given set of arrays and band counts autotunes the launch
// shape (slab chunk size, kernel B band grouping, split count of the tensor-core
// projection GEMM) by timing each candidate once, runs the chosen shape, and
// captures it into a CUDA graph; later calls with the same arrays replay the graph.
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <vector>

#include "../../include/cpw_b200.h"
#include "context.hpp"

using cpwb::C2;
using cpwb::DevBuf;
using cpwb::KDesc;
using cpwb::LocalPlan;
using cpwb::fail;
using cpwb::cuda_fail;

struct cpw_b200_kbatch {
  cpw_b200_ctx* c = nullptr;
  int nk = 0;
  int precision = 0;
  LocalPlan plan{};
  std::vector<int> mtxd, nanl;
  std::unique_ptr<DevBuf[]> start, idx, pos, ekpg, anl, anld, tca1, tca2;
  std::vector<long long> nkb1, nkb2;
  std::vector<char> tc_ready;
  DevBuf kdesc_d, bref_d, proj, blas_ws, slab;
  // projector products of all k-points in three launches (FP64 / MIXED, small blocks)
  DevBuf nl_d, nl_part;
  bool nl_batched = false;
  long long nl_ptot = 0;
  int nl_mmax = 0;
  cpwb::TcScratch tcs;    // own scratch: a captured call keeps these pointers
  cudaStream_t st = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr, t0 = nullptr, t1 = nullptr;
  // autotuned launch shape
  bool tuned = false;
  int tune_chunk = 0, tune_bgroups = 0, tune_splits = 0;
  float tune_ms = 0.f;
  int tune_candidates = 0;
  // captured call
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<long long> key;
  long long graph_launches = 0, captures = 0;

  ~cpw_b200_kbatch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (st) cudaStreamDestroy(st);
  }
};

namespace {

constexpr size_t kBlasWorkspace = 32u << 20;

struct Call {
  std::vector<int> nb;
  std::vector<const void*> psi;
  std::vector<void*> hpsi;
  std::vector<long long> ldpsi, ldh;
  int total = 0;
};

// Projector products of every k-point of the batch at once (FP64, every precision form), for blocks of at
// most kNlMax projectors and kNlMax bands per k-point. Per k-point ZGEMMs of a few dozen
// projectors and bands are latency-bound launches (two per k-point, one after the other); here
//   k_batch_proj:   partial P_k = X_k^H psi_k over a slice of plane waves, per (k, slice)
//   k_batch_reduce: P_k = sum of the slices, times nothing (xnlkb sits in X D)
//   k_batch_expand: hpsi_k += (X D)_k P_k, one thread per plane wave of each k
// (hk_psi_nl_c16.f90:82-96), in a fixed order: the result does not depend on timing.
struct NlDesc {
  const C2<double>* x;
  const C2<double>* xd;
  int m, na, nb;
  long long poff;      // offset of P_k (na x nb) in the concatenated P
};
constexpr int kNlMax = 64, kNlSlices = 8, kNlRows = 16, kNlThreads = 256;
constexpr int kNlPer = kNlMax * kNlMax / kNlThreads;   // outputs per thread
constexpr int kNlSmem = kNlMax * kNlMax * (int)sizeof(C2<double>);

__global__ void __launch_bounds__(kNlThreads)
k_batch_proj(const NlDesc* __restrict__ nd, const KDesc* __restrict__ kd, C2<double>* __restrict__ part,
             long long ptot) {
  __shared__ C2<double> xs[kNlRows][kNlMax], ps[kNlRows][kNlMax];
  const NlDesc D = nd[blockIdx.x];
  if (D.na == 0 || D.nb == 0 || D.m == 0) return;
  const C2<double>* psi = kd[blockIdx.x].psi;
  const long long ldpsi = kd[blockIdx.x].ldpsi;
  const int per = (D.m + kNlSlices - 1) / kNlSlices;
  const int r0 = blockIdx.y * per, r1 = min(D.m, r0 + per);
  const int nout = D.na * D.nb, tid = threadIdx.x;
  C2<double> acc[kNlPer];
#pragma unroll
  for (int t = 0; t < kNlPer; ++t) acc[t] = cpwb::mk<double>(0.0, 0.0);
  for (int i0 = r0; i0 < r1; i0 += kNlRows) {
    const int nr = min(kNlRows, r1 - i0);
    __syncthreads();
    for (int it = tid; it < kNlRows * kNlMax; it += kNlThreads) {
      const int r = it % kNlRows, c = it / kNlRows;
      const bool in = r < nr;
      xs[r][c] = in && c < D.na ? D.x[(size_t)c * D.m + i0 + r] : cpwb::mk<double>(0.0, 0.0);
      ps[r][c] = in && c < D.nb ? psi[(size_t)c * ldpsi + i0 + r] : cpwb::mk<double>(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < kNlPer; ++t) {
      const int o = tid + t * kNlThreads;
      if (o < nout) {
        const int j = o % D.na, n = o / D.na;
        C2<double> a = acc[t];
#pragma unroll 4
        for (int r = 0; r < kNlRows; ++r) {
          const C2<double> xv = xs[r][j], pv = ps[r][n];
          // conj(x) * psi
          a.x = fma(xv.x, pv.x, fma(xv.y, pv.y, a.x));
          a.y = fma(xv.x, pv.y, fma(-xv.y, pv.x, a.y));
        }
        acc[t] = a;
      }
    }
  }
#pragma unroll
  for (int t = 0; t < kNlPer; ++t) {
    const int o = tid + t * kNlThreads;
    if (o < nout) part[(size_t)blockIdx.y * ptot + D.poff + o] = acc[t];
  }
}

__global__ void k_batch_reduce(const C2<double>* __restrict__ part, C2<double>* __restrict__ P, long long ptot) {
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < ptot; o += (long long)gridDim.x * blockDim.x) {
    C2<double> a = part[o];
    for (int sl = 1; sl < kNlSlices; ++sl) {
      const C2<double> b = part[(size_t)sl * ptot + o];
      a.x += b.x;
      a.y += b.y;
    }
    P[o] = a;
  }
}

__global__ void __launch_bounds__(128)
k_batch_expand(const NlDesc* __restrict__ nd, const KDesc* __restrict__ kd, const C2<double>* __restrict__ P) {
  extern __shared__ __align__(16) unsigned char nl_smem[];
  C2<double>* pk = reinterpret_cast<C2<double>*>(nl_smem);   // P_k, na x nb
  const NlDesc D = nd[blockIdx.y];
  if (D.na == 0 || D.nb == 0 || D.m == 0) return;
  for (int o = threadIdx.x; o < D.na * D.nb; o += blockDim.x) pk[o] = P[D.poff + o];
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D.m) return;
  C2<double>* hp = kd[blockIdx.y].hpsi;
  const long long ldh = kd[blockIdx.y].ldh;
  constexpr int kB = 8;
  for (int n0 = 0; n0 < D.nb; n0 += kB) {
    C2<double> acc[kB];
#pragma unroll
    for (int t = 0; t < kB; ++t) acc[t] = cpwb::mk<double>(0.0, 0.0);
    for (int j = 0; j < D.na; ++j) {
      const C2<double> x = D.xd[(size_t)j * D.m + i];
#pragma unroll
      for (int t = 0; t < kB; ++t) {
        if (n0 + t < D.nb) {
          const C2<double> p = pk[j + (n0 + t) * D.na];
          acc[t].x = fma(x.x, p.x, fma(-x.y, p.y, acc[t].x));
          acc[t].y = fma(x.x, p.y, fma(x.y, p.x, acc[t].y));
        }
      }
    }
#pragma unroll
    for (int t = 0; t < kB; ++t)
      if (n0 + t < D.nb) {
        C2<double>& h = hp[(size_t)(n0 + t) * ldh + i];
        h.x += acc[t].x;
        h.y += acc[t].y;
      }
  }
}

// one pass of the batched H|psi> with a given launch shape, on b->st (capturable: no
// allocation or host synchronisation once the buffers exist)
int run_once(cpw_b200_kbatch* b, const Call& call, int chunk, int bgroups, int splits) {
  cpw_b200_ctx* c = b->c;
  LocalPlan q = b->plan;
  q.kdesc = (const KDesc*)b->kdesc_d.p;
  q.bref = (const int2*)b->bref_d.p;
  q.bgroups = bgroups;
  const bool f32 = b->precision != 0;
  const size_t esz = f32 ? sizeof(C2<float>) : sizeof(C2<double>);
  const size_t per_band = esz * (size_t)q.nz * (size_t)q.plane;
  int s;
  if ((s = b->slab.ensure(per_band * (size_t)chunk))) return s;
  for (int b0 = 0; b0 < call.total; b0 += chunk) {
    const int nbc = std::min(chunk, call.total - b0);
    cudaError_t e;
    // the per-call pointer arguments are unused in batch mode (the descriptors hold them)
    if (f32)
      e = cpwb::launch_local<float>(q, nbc, b0, nullptr, 0, nullptr, 0, nullptr, nullptr, nullptr, nullptr,
                                    (const float*)c->v32.p, (const C2<float>*)c->tw32[0].p,
                                    (const C2<float>*)c->tw32[1].p, (const C2<float>*)c->tw32[2].p,
                                    (C2<float>*)b->slab.p, b->st, nullptr);
    else
      e = cpwb::launch_local<double>(q, nbc, b0, nullptr, 0, nullptr, 0, nullptr, nullptr, nullptr, nullptr,
                                     (const double*)c->v64.p, (const C2<double>*)c->tw64[0].p,
                                     (const C2<double>*)c->tw64[1].p, (const C2<double>*)c->tw64[2].p,
                                     (C2<double>*)b->slab.p, b->st, nullptr);
    if (e != cudaSuccess) return cuda_fail(e, "kbatch local kernels");
  }
  if (b->nl_batched) {
    const NlDesc* nd = (const NlDesc*)b->nl_d.p;
    const KDesc* kd = (const KDesc*)b->kdesc_d.p;
    C2<double>* part = (C2<double>*)b->nl_part.p;
    C2<double>* P = (C2<double>*)b->proj.p;
    k_batch_proj<<<dim3(b->nk, kNlSlices), kNlThreads, 0, b->st>>>(nd, kd, part, b->nl_ptot);
    k_batch_reduce<<<296, 256, 0, b->st>>>(part, P, b->nl_ptot);
    k_batch_expand<<<dim3((b->nl_mmax + 127) / 128, b->nk), 128, kNlSmem, b->st>>>(nd, kd, P);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? cpwb::kOk : cuda_fail(e, "kbatch projector kernels");
  }
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
  for (int k = 0; k < b->nk; ++k) {
    const int na = b->nanl[k], m = b->mtxd[k], nb = call.nb[k];
    if (na == 0 || nb == 0 || m == 0) continue;
    if (b->precision == 2 && b->tc_ready[k]) {
      if ((s = cpwb::tc_nl_apply_ops(b->tcs, m, na, b->nkb1[k], b->nkb2[k], (const float*)b->tca1[k].p,
                                     (const float*)b->tca2[k].p, nb, call.psi[k], call.ldpsi[k], call.hpsi[k],
                                     call.ldh[k], b->st, nullptr, nullptr, nullptr, splits)))
        return s;
      continue;
    }
    // P = X^H psi (hk_psi_nl_c16.f90:82); hpsi += (X D) P (:87-96)
    cublasStatus_t bs = cublasZgemm(c->blas, CUBLAS_OP_C, CUBLAS_OP_N, na, nb, m, &one,
                                    (const cuDoubleComplex*)b->anl[k].p, m, (const cuDoubleComplex*)call.psi[k],
                                    (int)call.ldpsi[k], &zero, (cuDoubleComplex*)b->proj.p, na);
    if (bs != CUBLAS_STATUS_SUCCESS) return fail(cpwb::kCublas, "kbatch zgemm X^H psi");
    bs = cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, m, nb, na, &one, (const cuDoubleComplex*)b->anld[k].p, m,
                     (const cuDoubleComplex*)b->proj.p, na, &one, (cuDoubleComplex*)call.hpsi[k], (int)call.ldh[k]);
    if (bs != CUBLAS_STATUS_SUCCESS) return fail(cpwb::kCublas, "kbatch zgemm X D P");
  }
  return cpwb::kOk;
}

}  // namespace

extern "C" {

int cpw_b200_kbatch_create(cpw_b200_ctx* c, int nk, const int* mtxd, const int* const* isort, const int* kgv, int ng,
                           const double* const* ekpg, const int* kmscr, cpw_b200_kbatch** out) {
  if (!c || !out) return fail(cpwb::kBadArg, "kbatch_create: null argument");
  *out = nullptr;
  if (nk < 1 || !mtxd || !isort || !kgv || !ekpg || !kmscr || ng < 1)
    return fail(cpwb::kBadArg, "kbatch_create: invalid arguments");
  for (int k = 0; k < nk; ++k)
    if (mtxd[k] < 0 || (mtxd[k] > 0 && (!isort[k] || !ekpg[k])))
      return fail(cpwb::kBadArg, "kbatch_create: invalid k-point basis");
  int s;
  // the context's box (twiddles, potential layout); the context keeps k-point 0 as its own basis
  if (!c->have_basis || c->plan.n1 != kmscr[3] || c->plan.n2 != kmscr[4] || c->plan.n3 != kmscr[5] ||
      c->ident != kmscr[6]) {
    if ((s = cpwb::ctx_set_basis(c, mtxd[0], isort[0], kgv, ng, ekpg[0], kmscr))) return s;
  }
  std::unique_ptr<cpw_b200_kbatch> b(new cpw_b200_kbatch);
  b->c = c;
  b->nk = nk;
  b->precision = c->precision;
  b->mtxd.assign(mtxd, mtxd + nk);
  b->nanl.assign(nk, 0);
  b->start.reset(new DevBuf[nk]);
  b->idx.reset(new DevBuf[nk]);
  b->pos.reset(new DevBuf[nk]);
  b->ekpg.reset(new DevBuf[nk]);
  b->anl.reset(new DevBuf[nk]);
  b->anld.reset(new DevBuf[nk]);
  b->tca1.reset(new DevBuf[nk]);
  b->tca2.reset(new DevBuf[nk]);
  b->nkb1.assign(nk, 0);
  b->nkb2.assign(nk, 0);
  b->tc_ready.assign(nk, 0);
  // union of the spheres: the common kept planes and rows
  std::vector<std::vector<int>> g(nk);
  int kd[3] = {0, 0, 0};
  for (int k = 0; k < nk; ++k) {
    g[k].resize(3 * (size_t)mtxd[k]);
    for (int i = 0; i < mtxd[k]; ++i) {
      const int it = isort[k][i];
      if (it < 1 || it > ng) return fail(cpwb::kBadArg, "kbatch_create: isort out of range of kgv");
      for (int j = 0; j < 3; ++j) {
        const int v = kgv[3 * (size_t)(it - 1) + j];
        g[k][3 * (size_t)i + j] = v;
        kd[j] = std::max(kd[j], std::abs(v));
      }
    }
  }
  if ((s = cpwb::plan_for_box(c, kd, kmscr, &b->plan))) return s;
  for (int k = 0; k < nk; ++k) {
    std::vector<int> st_, id_, ps_;
    cpwb::plane_lists(b->plan, mtxd[k], g[k].data(), st_, id_, ps_);
    if ((s = cpwb::upload(b->start[k], st_.data(), st_.size() * sizeof(int)))) return s;
    if (mtxd[k] > 0) {
      if ((s = cpwb::upload(b->idx[k], id_.data(), id_.size() * sizeof(int))) ||
          (s = cpwb::upload(b->pos[k], ps_.data(), ps_.size() * sizeof(int))) ||
          (s = cpwb::upload(b->ekpg[k], ekpg[k], (size_t)mtxd[k] * sizeof(double))))
        return s;
    }
  }
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreate(&b->t0)) != cudaSuccess || (e = cudaEventCreate(&b->t1)) != cudaSuccess)
    return cuda_fail(e, "kbatch_create");
  *out = b.release();
  return cpwb::kOk;
}

int cpw_b200_kbatch_destroy(cpw_b200_kbatch* b) {
  if (b) {
    cudaDeviceSynchronize();
    delete b;
  }
  return cpwb::kOk;
}

int cpw_b200_kbatch_set_projectors(cpw_b200_kbatch* b, int ik, int nanl, const void* anlga, long long ld,
                                   const double* xnlkb) {
  if (!b) return fail(cpwb::kBadArg, "kbatch_set_projectors: null batch");
  if (ik < 0 || ik >= b->nk) return fail(cpwb::kBadArg, "kbatch_set_projectors: k-point index out of range");
  const int m = b->mtxd[ik];
  if (nanl < 0 || (nanl > 0 && (!anlga || !xnlkb || ld < m)))
    return fail(cpwb::kBadArg, "kbatch_set_projectors: invalid projector arrays");
  b->nanl[ik] = nanl;
  b->tc_ready[ik] = 0;
  if (nanl == 0 || m == 0) return cpwb::kOk;
  // X (first m rows of each column) and X diag(xnlkb), packed with leading dimension m
  const C2<double>* x = (const C2<double>*)anlga;
  std::vector<C2<double>> h((size_t)m * nanl), hd((size_t)m * nanl);
  for (int a = 0; a < nanl; ++a)
    for (int i = 0; i < m; ++i) {
      const C2<double> v = x[(size_t)a * ld + i];
      h[(size_t)a * m + i] = v;
      hd[(size_t)a * m + i] = cpwb::mk<double>(v.x * xnlkb[a], v.y * xnlkb[a]);
    }
  int s;
  if ((s = cpwb::upload(b->anl[ik], h.data(), h.size() * sizeof(C2<double>))) ||
      (s = cpwb::upload(b->anld[ik], hd.data(), hd.size() * sizeof(C2<double>))))
    return s;
  if (b->precision == 2) {
    if ((s = cpwb::tc_prepare_operands(m, nanl, b->anl[ik].p, b->anld[ik].p, b->tca1[ik], b->tca2[ik], &b->nkb1[ik],
                                       &b->nkb2[ik], b->st)))
      return s;
    b->tc_ready[ik] = 1;
  }
  // a captured call refers to the old operands
  b->key.clear();
  return cpwb::kOk;
}

int cpw_b200_kbatch_hk_psi_device(cpw_b200_kbatch* b, const int* nb, void* const* psi, const long long* ldpsi,
                                  void* const* hpsi, const long long* ldh, void* stream) {
  if (!b) return fail(cpwb::kBadArg, "kbatch_hk_psi: null batch");
  cpw_b200_ctx* c = b->c;
  if (!c->have_pot) return fail(cpwb::kNotReady, "kbatch_hk_psi: set the potential on the context first");
  if (c->precision != b->precision)
    return fail(cpwb::kBadArg, "kbatch_hk_psi: the context precision changed since the batch was created");
  if (!nb || !psi || !hpsi || !ldpsi || !ldh) return fail(cpwb::kBadArg, "kbatch_hk_psi: null argument");
  Call call;
  call.nb.assign(nb, nb + b->nk);
  call.psi.resize(b->nk);
  call.hpsi.resize(b->nk);
  call.ldpsi.assign(ldpsi, ldpsi + b->nk);
  call.ldh.assign(ldh, ldh + b->nk);
  std::vector<long long> key;
  key.push_back(b->precision);
  for (int k = 0; k < b->nk; ++k) {
    if (nb[k] < 0) return fail(cpwb::kBadArg, "kbatch_hk_psi: negative band count");
    if (nb[k] > 0 && (!psi[k] || !hpsi[k] || ldpsi[k] < b->mtxd[k] || ldh[k] < b->mtxd[k]))
      return fail(cpwb::kBadArg, "kbatch_hk_psi: invalid wavefunction block");
    call.psi[k] = psi[k];
    call.hpsi[k] = hpsi[k];
    call.total += nb[k] > 0 && b->mtxd[k] > 0 ? nb[k] : 0;
    key.insert(key.end(), {(long long)nb[k], (long long)(uintptr_t)psi[k], (long long)(uintptr_t)hpsi[k], ldpsi[k],
                           ldh[k]});
  }
  if (call.total == 0) return cpwb::kOk;
  cudaStream_t user = (cudaStream_t)stream;
  cudaError_t e;
  if ((e = cudaEventRecord(b->ev_in, user)) != cudaSuccess || (e = cudaStreamWaitEvent(b->st, b->ev_in, 0)) != cudaSuccess)
    return cuda_fail(e, "kbatch_hk_psi");
  int s;
  if (b->exec && key == b->key) {
    if ((e = cudaGraphLaunch(b->exec, b->st)) != cudaSuccess) return cuda_fail(e, "kbatch graph launch");
    ++b->graph_launches;
  } else {
    // descriptor and band tables of this call
    std::vector<KDesc> kd(b->nk);
    std::vector<int2> br;
    br.reserve(call.total);
    size_t maxproj = 0;
    for (int k = 0; k < b->nk; ++k) {
      kd[k].psi = (const C2<double>*)psi[k];
      kd[k].hpsi = (C2<double>*)hpsi[k];
      kd[k].ldpsi = ldpsi[k];
      kd[k].ldh = ldh[k];
      kd[k].plane_start = (const int*)b->start[k].p;
      kd[k].pw_idx = (const int*)b->idx[k].p;
      kd[k].pw_pos = (const int*)b->pos[k].p;
      kd[k].ekpg = (const double*)b->ekpg[k].p;
      if (b->mtxd[k] > 0)
        for (int j = 0; j < nb[k]; ++j) br.push_back(make_int2(k, j));
      maxproj = std::max(maxproj, (size_t)b->nanl[k] * std::max(nb[k], 0));
    }
    if ((s = cpwb::upload(b->kdesc_d, kd.data(), kd.size() * sizeof(KDesc))) ||
        (s = cpwb::upload(b->bref_d, br.data(), br.size() * sizeof(int2))) ||
        (s = b->proj.ensure(std::max<size_t>(maxproj, 1) * sizeof(C2<double>))) ||
        (s = b->blas_ws.ensure(kBlasWorkspace)))
      return s;
    // all projector products in three launches when every block is small (FP64 / MIXED);
    // CPW_B200_KBATCH_NL=0 keeps one ZGEMM pair per k-point
    {
      const char* v = getenv("CPW_B200_KBATCH_NL");
      bool small = !(v && atoi(v) == 0);
      std::vector<NlDesc> nd(b->nk);
      long long poff = 0;
      int mmax = 0;
      for (int k = 0; k < b->nk && small; ++k) {
        const int na = b->nanl[k], nbk = std::max(nb[k], 0), m = b->mtxd[k];
        if (na > kNlMax || nbk > kNlMax) small = false;
        nd[k].x = (const C2<double>*)b->anl[k].p;
        nd[k].xd = (const C2<double>*)b->anld[k].p;
        nd[k].m = (na > 0 && nbk > 0) ? m : 0;
        nd[k].na = na;
        nd[k].nb = nbk;
        nd[k].poff = poff;
        poff += (long long)na * nbk;
        mmax = std::max(mmax, m);
      }
      b->nl_batched = small && poff > 0;
      if (b->nl_batched) {
        b->nl_ptot = poff;
        b->nl_mmax = mmax;
        cudaError_t ea = cpwb::smem_limit((const void*)k_batch_expand, (size_t)kNlSmem);
        if (ea != cudaSuccess) return cuda_fail(ea, "kbatch attribute");
        if ((s = cpwb::upload(b->nl_d, nd.data(), nd.size() * sizeof(NlDesc))) ||
            (s = b->nl_part.ensure((size_t)kNlSlices * poff * sizeof(C2<double>))) ||
            (s = b->proj.ensure((size_t)poff * sizeof(C2<double>))))
          return s;
      }
    }
    cublasSetStream(c->blas, b->st);
    cublasSetWorkspace(c->blas, b->blas_ws.p, kBlasWorkspace);
    // slab memory for all bands at once, within the context's slab budget
    const size_t esz = b->precision ? sizeof(C2<float>) : sizeof(C2<double>);
    const size_t per_band = esz * (size_t)b->plan.nz * (size_t)b->plan.plane;
    const int cap = (int)std::max<size_t>(1, std::min<size_t>((size_t)call.total, c->slab_budget / per_band));
    if (!b->tuned) {
      std::vector<int> chunks = {cap};
      for (int d : {2, 4})
        if ((cap + d - 1) / d >= 16) chunks.push_back((cap + d - 1) / d);
      const int bgs[3] = {1, 2, 4};
      const int sps[2] = {0, -4};   // heuristic split count, a quarter of it
      if ((s = run_once(b, call, chunks[0], 0, 0))) return s;   // warm-up, allocates everything
      float best = 1e30f;
      b->tune_candidates = 0;
      for (int ch : chunks)
        for (int bg : bgs)
          for (int sp : sps) {
            if (sp != 0 && b->precision != 2) continue;
            cudaEventRecord(b->t0, b->st);
            if ((s = run_once(b, call, ch, bg, sp))) return s;
            cudaEventRecord(b->t1, b->st);
            if ((e = cudaEventSynchronize(b->t1)) != cudaSuccess) return cuda_fail(e, "kbatch autotune");
            float ms = 0.f;
            cudaEventElapsedTime(&ms, b->t0, b->t1);
            ++b->tune_candidates;
            if (ms < best) {
              best = ms;
              b->tune_chunk = ch;
              b->tune_bgroups = bg;
              b->tune_splits = sp;
            }
          }
      b->tune_ms = best;
      b->tuned = true;
    }
    const int chunk = std::min(b->tune_chunk, cap);
    if ((s = run_once(b, call, chunk, b->tune_bgroups, b->tune_splits))) return s;
    // capture the same sequence for the next calls with these arrays
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->key.clear();
    if ((e = cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return cuda_fail(e, "kbatch capture");
    s = run_once(b, call, chunk, b->tune_bgroups, b->tune_splits);
    cudaGraph_t gr = nullptr;
    e = cudaStreamEndCapture(b->st, &gr);
    if (s) {
      if (gr) cudaGraphDestroy(gr);
      return s;
    }
    if (e != cudaSuccess) return cuda_fail(e, "kbatch capture");
    b->graph = gr;
    if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess) return cuda_fail(e, "kbatch instantiate");
    b->key = key;
    ++b->captures;
  }
  if ((e = cudaEventRecord(b->ev_out, b->st)) != cudaSuccess || (e = cudaStreamWaitEvent(user, b->ev_out, 0)) != cudaSuccess)
    return cuda_fail(e, "kbatch_hk_psi");
  return cpwb::kOk;
}

int cpw_b200_kbatch_synchronize(cpw_b200_kbatch* b) {
  if (!b) return fail(cpwb::kBadArg, "kbatch_synchronize: null batch");
  cudaError_t e = cudaStreamSynchronize(b->st);
  if (e != cudaSuccess) return cuda_fail(e, "kbatch_synchronize");
  return cpwb::tc_read_error(b->tcs);
}

int cpw_b200_kbatch_info(cpw_b200_kbatch* b, long long* out, int n) {
  if (!b || !out) return fail(cpwb::kBadArg, "kbatch_info: null argument");
  const long long v[8] = {b->tuned ? 1 : 0, b->tune_chunk, b->tune_bgroups, b->tune_splits,
                          (long long)(1000.0 * b->tune_ms), b->tune_candidates, b->graph_launches, b->captures};
  for (int i = 0; i < n && i < 8; ++i) out[i] = v[i];
  return cpwb::kOk;
}

}  // extern "C"
