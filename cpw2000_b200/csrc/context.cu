// Device state for one k-point: basis plane lists, potential, projectors, and
// the H|psi> driver (local kernels per band chunk, then the KB projector
// GEMMs of Src/cpw_lib/hk_psi_nl_c16.f90:82-97).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "context.hpp"

namespace cpwb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }
int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  return fail(kCuda, std::string(what) + ": " + cudaGetErrorString(e));
}

cudaEvent_t StageTimer::take() {
  if (used < pool.size()) return pool[used++];
  if (pool.size() >= 65536) return nullptr;
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  pool.push_back(e);
  ++used;
  return e;
}
StageTimer::~StageTimer() {
  for (cudaEvent_t e : pool) cudaEventDestroy(e);
}

int DevBuf::ensure(size_t need) {
  if (need <= bytes && p) return kOk;
  // a buffer that grows takes 1.5x (at least) of its old size, rounded to 2 MiB: buffers sized by
  // the eigensolver's growing blocks are then reallocated a few times per solve instead of every
  // iteration (cudaFree synchronises the whole device, stalling every context that shares it)
  if (p) need = std::max(need, bytes + bytes / 2);
  if (need > (1u << 20)) need = (need + (2u << 20) - 1) & ~(size_t)((2u << 20) - 1);
  release();
  if (need == 0) return kOk;
  cudaError_t e = cudaMalloc(&p, need);
  if (e != cudaSuccess) {
    p = nullptr;
    bytes = 0;
    return cuda_fail(e, "cudaMalloc");
  }
  bytes = need;
  return kOk;
}
void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

// Split n = r1*r2 with both factors supported radices, as balanced as possible.
bool factor(int n, FftDim& d) {
  int best = -1;
  for (int r1 = 1; r1 <= 16; ++r1) {
    if (n % r1) continue;
    int r2 = n / r1;
    if (!radix_ok(r1) || !radix_ok(r2) || r1 > r2) continue;
    best = r1;
  }
  if (best < 0) return false;
  d.n = n;
  d.r1 = best;
  d.r2 = n / best;
  return true;
}

// W_n^k = exp(-2 pi i k / n), k = 0..n-1, in long double then rounded.
void twiddles(int n, std::vector<double>& out) {
  out.resize(2 * (size_t)n);
  const long double tp = 6.283185307179586476925286766559005768L;
  for (int k = 0; k < n; ++k) {
    long double a = tp * (long double)k / (long double)n;
    out[2 * k] = (double)cosl(a);
    out[2 * k + 1] = (double)-sinl(a);
  }
}

// host -> device copy that has landed when it returns (a pageable cudaMemcpy may return
// before its DMA completes; work on non-blocking streams must not see a partial copy)
int upload(DevBuf& b, const void* h, size_t bytes) {
  int s = b.ensure(bytes);
  if (s) return s;
  cudaError_t e = cudaMemcpy(b.p, h, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
  return e == cudaSuccess ? kOk : cuda_fail(e, "cudaMemcpy H2D");
}

static size_t max_smem_optin(int dev) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return (size_t)v;
}

int plan_for_box(cpw_b200_ctx* c, const int kd[3], const int* kmscr, LocalPlan* out) {
  const int n1 = kmscr[3], n2 = kmscr[4], n3 = kmscr[5];
  LocalPlan p{};
  p.n1 = n1; p.n2 = n2; p.n3 = n3;
  if (!factor(n1, p.dx) || !factor(n2, p.dy) || !factor(n3, p.dz))
    return fail(kUnsupported, "set_basis: FFT length is not a product of two radices in {1..6,8,9,10,12,16} (max 256)");
  if (kd[0] > (n1 - 1) / 2 || kd[1] > (n2 - 1) / 2 || kd[2] > (n3 - 1) / 2) {
    char buf[256];
    snprintf(buf, sizeof buf, "hk_psi_c16: dimension of k index= %d %d %d exceeds %d %d %d", kd[0], kd[1], kd[2],
             (n1 - 1) / 2, (n2 - 1) / 2, (n3 - 1) / 2);
    return fail(kWrap, buf);
  }
  p.kd1 = kd[0]; p.kd2 = kd[1]; p.kd3 = kd[2];
  p.nx = 2 * kd[0] + 1; p.ny = 2 * kd[1] + 1; p.nz = 2 * kd[2] + 1;
  p.plane = (long long)n1 * n2;
  p.rowp = n1 + 1;
  const size_t cmax = max_smem_optin(c->device);
  const size_t esz = c->precision ? sizeof(C2<float>) : sizeof(C2<double>);
  p.tcol = 32;
  while (p.tcol > 4 && esz * ((size_t)p.ny * p.rowp + (size_t)p.n2 * p.tcol + n1 + n2) > cmax) p.tcol /= 2;
  if (esz * ((size_t)p.ny * p.rowp + (size_t)p.n2 * p.tcol + n1 + n2) > cmax)
    return fail(kUnsupported, "set_basis: plane does not fit in shared memory");
  int smsm = 0;
  cudaDeviceGetAttribute(&smsm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->device);
  p.cb = column_tile(esz, p, cmax, (size_t)smsm);
  *out = p;
  return kOk;
}

void plane_lists(const LocalPlan& p, int mtxd, const int* g, std::vector<int>& start, std::vector<int>& idx,
                 std::vector<int>& pos) {
  const int n1 = p.n1, n2 = p.n2, n3 = p.n3;
  // plane lists: basis sorted by kept z-plane
  std::vector<int> zi(mtxd);
  start.assign(p.nz + 1, 0);
  for (int i = 0; i < mtxd; ++i) {
    int k3 = g[3 * (size_t)i + 2];
    if (k3 < 0) k3 += n3;
    zi[i] = idx_to_kept(k3, p.kd3, n3, p.nz);
    start[zi[i] + 1]++;
  }
  for (int z = 0; z < p.nz; ++z) start[z + 1] += start[z];
  std::vector<int> fillp(start.begin(), start.end() - 1);
  idx.assign(mtxd, 0);
  pos.assign(mtxd, 0);
  for (int i = 0; i < mtxd; ++i) {
    int k1 = g[3 * (size_t)i], k2 = g[3 * (size_t)i + 1];
    if (k1 < 0) k1 += n1;
    if (k2 < 0) k2 += n2;
    const int yi = idx_to_kept(k2, p.kd2, n2, p.ny);
    const int e = fillp[zi[i]]++;
    idx[e] = i;
    pos[e] = (yi << 16) | k1;
  }
}

int ctx_set_basis(cpw_b200_ctx* c, int mtxd, const int* isort, const int* kgv, int ng, const double* ekpg,
                  const int* kmscr) {
  if (mtxd < 0 || ng < 0) return fail(kBadArg, "set_basis: negative mtxd or ng");
  const int n1 = kmscr[3], n2 = kmscr[4], n3 = kmscr[5];
  if (n1 < 2 || n2 < 2 || n3 < 2) return fail(kBadArg, "set_basis: FFT dimension less than 2");
  if (n1 > 65535 || n2 > 65535 || n3 > 65535) return fail(kUnsupported, "set_basis: FFT dimension too large");
  if (kmscr[6] < n1) return fail(kBadArg, "set_basis: leading dimension kmscr(7) smaller than n1");
  // sphere extent and wraparound check (hk_psi_c16.f90:145-172)
  int kd[3] = {0, 0, 0};
  std::vector<int> g(3 * (size_t)mtxd);
  for (int i = 0; i < mtxd; ++i) {
    const int it = isort[i];
    if (it < 1 || it > ng) return fail(kBadArg, "set_basis: isort out of range of kgv");
    for (int j = 0; j < 3; ++j) {
      const int k = kgv[3 * (size_t)(it - 1) + j];
      g[3 * (size_t)i + j] = k;
      kd[j] = std::max(kd[j], std::abs(k));
    }
  }
  LocalPlan p{};
  if (int s = plan_for_box(c, kd, kmscr, &p)) return s;
  std::vector<int> start, idx, pos;
  plane_lists(p, mtxd, g.data(), start, idx, pos);
  int s;
  if ((s = upload(c->plane_start, start.data(), start.size() * sizeof(int)))) return s;
  if (mtxd > 0) {
    if ((s = upload(c->pw_idx, idx.data(), idx.size() * sizeof(int)))) return s;
    if ((s = upload(c->pw_pos, pos.data(), pos.size() * sizeof(int)))) return s;
    if ((s = upload(c->ekpg, ekpg, (size_t)mtxd * sizeof(double)))) return s;
    if ((s = upload(c->kgvb, g.data(), g.size() * sizeof(int)))) return s;
  }
  const int ns[3] = {n1, n2, n3};
  for (int d = 0; d < 3; ++d) {
    std::vector<double> tw;
    twiddles(ns[d], tw);
    std::vector<float> tw32(tw.begin(), tw.end());
    if ((s = upload(c->tw64[d], tw.data(), tw.size() * sizeof(double)))) return s;
    if ((s = upload(c->tw32[d], tw32.data(), tw32.size() * sizeof(float)))) return s;
  }
  c->plan = p;
  c->mtxd = mtxd;
  c->ident = kmscr[6];
  c->have_pot = false;  // the box may have changed
  c->have_basis = true;
  return kOk;
}

int ctx_set_potential(cpw_b200_ctx* c, const double* vscr, long long nscr) {
  if (!c->have_basis) return fail(kNotReady, "set_potential: call set_basis first (box size)");
  const LocalPlan& p = c->plan;
  const int n1 = p.n1, n2 = p.n2, n3 = p.n3;
  const long long id = c->ident;
  if (nscr < id * n2 * (long long)n3) return fail(kBadArg, "set_potential: vscr smaller than id*n2*n3");
  const double inv = 1.0 / ((double)n1 * n2 * n3);
  std::vector<double> v((size_t)n1 * n2 * n3);
  std::vector<float> vf(v.size());
  for (int z = 0; z < n3; ++z)
    for (int y = 0; y < n2; ++y)
      for (int x = 0; x < n1; ++x) {
        const size_t o = ((size_t)z * n2 + y) * n1 + x;
        v[o] = vscr[((size_t)z * n2 + y) * id + x] * inv;
        vf[o] = (float)v[o];
      }
  int s;
  if ((s = upload(c->v64, v.data(), v.size() * sizeof(double)))) return s;
  if ((s = upload(c->v32, vf.data(), vf.size() * sizeof(float)))) return s;
  c->pot_n[0] = n1; c->pot_n[1] = n2; c->pot_n[2] = n3;
  c->have_pot = true;
  return kOk;
}

__global__ void k_scale_cols(const C2<double>* __restrict__ a, C2<double>* __restrict__ b, const double* __restrict__ s,
                             long long rows, int cols, long long lda, long long ldb) {
  const long long n = rows * cols;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long j = t / rows, i = t - j * rows;
    const C2<double> v = a[j * lda + i];
    b[j * ldb + i] = mk<double>(v.x * s[j], v.y * s[j]);
  }
}

__global__ void k_copy_cols(const C2<double>* __restrict__ a, C2<double>* __restrict__ b, long long rows, int cols,
                            long long lda, long long ldb) {
  const long long n = rows * cols;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long j = t / rows, i = t - j * rows;
    b[j * ldb + i] = a[j * lda + i];
  }
}

int ctx_set_projectors(cpw_b200_ctx* c, int nanl, const double* anlga, int ld, const double* xnlkb, bool on_device) {
  if (!c->have_basis) return fail(kNotReady, "set_projectors: call set_basis first");
  if (nanl < 0) return fail(kBadArg, "set_projectors: nanl < 0");
  const long long m = c->mtxd;
  if (nanl > 0 && ld < m) return fail(kBadArg, "set_projectors: leading dimension smaller than mtxd");
  c->nanl = nanl;
  if (nanl == 0 || m == 0) return kOk;
  int s;
  const size_t bytes = (size_t)m * nanl * sizeof(C2<double>);
  if ((s = c->anl.ensure(bytes))) return s;
  if ((s = c->anld.ensure(bytes))) return s;
  DevBuf dx;
  if ((s = dx.ensure((size_t)nanl * sizeof(double)))) return s;
  cudaError_t e;
  if (on_device) {
    e = cudaMemcpyAsync(dx.p, xnlkb, nanl * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "set_projectors copy");
    k_copy_cols<<<1184, 256, 0, c->stream>>>((const C2<double>*)anlga, (C2<double>*)c->anl.p, m, nanl, ld, m);
  } else {
    e = cudaMemcpy2DAsync(c->anl.p, m * sizeof(C2<double>), anlga, (size_t)ld * sizeof(C2<double>),
                          m * sizeof(C2<double>), nanl, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "set_projectors copy");
    e = cudaMemcpyAsync(dx.p, xnlkb, nanl * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "set_projectors copy");
  }
  k_scale_cols<<<1184, 256, 0, c->stream>>>((const C2<double>*)c->anl.p, (C2<double>*)c->anld.p,
                                            (const double*)dx.p, m, nanl, m, m);
  c->xnl_h.resize(nanl);
  e = cudaMemcpyAsync(c->xnl_h.data(), dx.p, nanl * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "set_projectors copy");
  c->tc_ready = false;
  c->oz_nl_ready = false;
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "set_projectors");
  if (c->precision == 2) return tc_prepare_projectors(c);
  return kOk;
}

static int blas_fail(cublasStatus_t st, const char* what) {
  return fail(kCublas, std::string(what) + ": cuBLAS status " + std::to_string((int)st));
}

int ctx_hkpsi_device(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, void* hpsi, long long ldh,
                     cudaStream_t st, bool with_kinetic, bool with_nl) {
  if (!c->have_basis || !c->have_pot) return fail(kNotReady, "hk_psi: basis and potential must be set");
  if (nb < 0) return fail(kBadArg, "hk_psi: neig < 0");
  if (nb == 0 || c->mtxd == 0) return kOk;
  if (ldpsi < c->mtxd || ldh < c->mtxd) return fail(kBadArg, "hk_psi: leading dimension smaller than mtxd");
  const LocalPlan& p = c->plan;
  const bool f32 = c->precision != 0;
  const size_t esz = f32 ? sizeof(C2<float>) : sizeof(C2<double>);
  const size_t per_band = esz * (size_t)p.nz * (size_t)p.plane;
  int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)nb, c->slab_budget / per_band));
  int s;
  if ((s = c->slab.ensure(per_band * (size_t)chunk))) return s;
  const C2<double>* ps = (const C2<double>*)psi;
  C2<double>* hp = (C2<double>*)hpsi;
  const double* ek = with_kinetic ? (const double*)c->ekpg.p : nullptr;
  // FP64 projector products of the MIXED form: the projection P = X^H psi needs psi only, so it
  // runs on the projection stream beside the FP32 local kernels (filling the SMs their tails leave
  // idle; Si216 28.5 -> 27.7 ms); the expansion follows the local kernels on st. The FP64 form
  // gains 0.5-1% this way and keeps both on st, so that its stage timers time each kernel alone.
  // CPW_B200_NL_OVERLAP=1 / 0 forces either way.
  const bool i8_nl = with_nl && c->nanl > 0 && c->nl_slices > 0;
  const bool cublas_nl = with_nl && c->nanl > 0 && !i8_nl && !(c->precision == 2 && c->tc_ready);
  bool overlap = false;
  cudaEvent_t ov_t0 = nullptr, ov_t1 = nullptr;
  if (cublas_nl) {
    const char* v = getenv("CPW_B200_NL_OVERLAP");
    overlap = v ? atoi(v) != 0 : c->precision == 1;
  }
  if (overlap) {
    cudaError_t e;
    if (!c->s_nl && (e = cudaStreamCreateWithFlags(&c->s_nl, cudaStreamNonBlocking)) != cudaSuccess)
      return cuda_fail(e, "hk_psi stream");
    if (!c->blas_nl) {
      if (cublasCreate(&c->blas_nl) != CUBLAS_STATUS_SUCCESS) {
        c->blas_nl = nullptr;
        return fail(kCublas, "cublasCreate failed");
      }
    }
    for (auto& ev : c->ov_ev)
      if (!ev && (e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return cuda_fail(e, "event");
    if ((s = c->proj.ensure((size_t)c->nanl * nb * sizeof(C2<double>)))) return s;
    if ((e = cudaEventRecord(c->ov_ev[0], st)) != cudaSuccess || (e = cudaStreamWaitEvent(c->s_nl, c->ov_ev[0], 0)) != cudaSuccess)
      return cuda_fail(e, "hk_psi overlap");
    ov_t0 = c->timer.on ? c->timer.take() : nullptr;
    ov_t1 = c->timer.on ? c->timer.take() : nullptr;
    if (ov_t0) cudaEventRecord(ov_t0, c->s_nl);
    cublasSetStream(c->blas_nl, c->s_nl);
    const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
    // P = X^H psi (hk_psi_nl_c16.f90:82)
    if (cublasZgemm(c->blas_nl, CUBLAS_OP_C, CUBLAS_OP_N, c->nanl, nb, c->mtxd, &one, (const cuDoubleComplex*)c->anl.p,
                    c->mtxd, (const cuDoubleComplex*)psi, (int)ldpsi, &zero, (cuDoubleComplex*)c->proj.p,
                    c->nanl) != CUBLAS_STATUS_SUCCESS)
      return fail(kCublas, "zgemm X^H psi");
    if (ov_t1) cudaEventRecord(ov_t1, c->s_nl);
    if ((e = cudaEventRecord(c->ov_ev[1], c->s_nl)) != cudaSuccess) return cuda_fail(e, "hk_psi overlap");
  }
  for (int b0 = 0; b0 < nb; b0 += chunk) {
    const int nbc = std::min(chunk, nb - b0);
    cudaError_t e;
    cudaEvent_t evs[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t* ev = nullptr;
    if (c->timer.on) {
      for (int k = 0; k < 4; ++k) evs[k] = c->timer.take();
      if (evs[0] && evs[1] && evs[2] && evs[3]) ev = evs;
    }
    if (f32) {
      e = launch_local<float>(p, nbc, b0, ps, ldpsi, hp, ldh, (const int*)c->plane_start.p, (const int*)c->pw_idx.p,
                              (const int*)c->pw_pos.p, ek, (const float*)c->v32.p, (const C2<float>*)c->tw32[0].p,
                              (const C2<float>*)c->tw32[1].p, (const C2<float>*)c->tw32[2].p,
                              (C2<float>*)c->slab.p, st, ev);
    } else {
      e = launch_local<double>(p, nbc, b0, ps, ldpsi, hp, ldh, (const int*)c->plane_start.p,
                               (const int*)c->pw_idx.p, (const int*)c->pw_pos.p, ek, (const double*)c->v64.p,
                               (const C2<double>*)c->tw64[0].p, (const C2<double>*)c->tw64[1].p,
                               (const C2<double>*)c->tw64[2].p, (C2<double>*)c->slab.p, st, ev);
    }
    if (e != cudaSuccess) return cuda_fail(e, "hk_psi local kernels");
    if (ev) {
      c->timer.mark(kStInvXY, ev[0], ev[1]);
      c->timer.mark(kStZVloc, ev[1], ev[2]);
      c->timer.mark(kStFwdXY, ev[2], ev[3]);
    }
  }
  if (overlap) {
    cudaError_t e;
    if ((e = cudaStreamWaitEvent(st, c->ov_ev[1], 0)) != cudaSuccess) return cuda_fail(e, "hk_psi overlap");
    cudaEvent_t t1 = c->timer.on ? c->timer.take() : nullptr, t2 = c->timer.on ? c->timer.take() : nullptr;
    if (t1) cudaEventRecord(t1, st);
    cublasSetStream(c->blas, st);
    const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
    // hpsi += (X D) P (hk_psi_nl_c16.f90:87-96)
    if (cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, c->mtxd, nb, c->nanl, &one, (const cuDoubleComplex*)c->anld.p,
                    c->mtxd, (const cuDoubleComplex*)c->proj.p, c->nanl, &one, (cuDoubleComplex*)hpsi,
                    (int)ldh) != CUBLAS_STATUS_SUCCESS)
      return fail(kCublas, "zgemm X D P");
    if (t2) cudaEventRecord(t2, st);
    c->timer.mark(kStNlProj, ov_t0, ov_t1);
    c->timer.mark(kStNlExpand, t1, t2);
    return kOk;
  }
  if (with_nl && c->nanl > 0) {
    if ((s = c->proj.ensure((size_t)c->nanl * nb * sizeof(C2<double>)))) return s;
    cublasSetStream(c->blas, st);
    const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
    cublasStatus_t bs;
    cudaEvent_t t0 = c->timer.on ? c->timer.take() : nullptr, t1 = c->timer.on ? c->timer.take() : nullptr;
    cudaEvent_t t2 = c->timer.on ? c->timer.take() : nullptr;
    if (i8_nl) {
      // projector products on the int8 tensor cores (oz.cu): X and X D split into int8 tiles once
      // per projector set, psi and P per call
      if (!c->oz_nl_ready || c->oz_x.s != c->nl_slices) {
        if ((s = oz_prepare_a(c->oz_x, true, c->nanl, c->mtxd, c->anl.p, c->mtxd, c->nl_slices, st)) ||
            (s = oz_prepare_a(c->oz_xd, false, c->mtxd, c->nanl, c->anld.p, c->mtxd, c->nl_slices, st)))
          return s;
        c->oz_nl_ready = true;
      }
      if (t0) cudaEventRecord(t0, st);
      // P = X^H psi (hk_psi_nl_c16.f90:82); hpsi += (X D) P (:87-96)
      if ((s = oz_gemm_prepared(c->ozs, c->oz_x, nb, psi, ldpsi, 1.0, false, c->proj.p, c->nanl, c->tcs.wait_ns, st)))
        return s;
      if (t1) cudaEventRecord(t1, st);
      if ((s = oz_gemm_prepared(c->ozs, c->oz_xd, nb, c->proj.p, c->nanl, 1.0, true, hpsi, ldh, c->tcs.wait_ns, st)))
        return s;
      if (t2) cudaEventRecord(t2, st);
      c->timer.mark(kStNlProj, t0, t1);
      c->timer.mark(kStNlExpand, t1, t2);
      return kOk;
    }
    if (c->precision == 2 && c->tc_ready) {
      // opt-in mixed form: split-TF32 tensor-core products (nl_tc.cu)
      if ((s = tc_nl_apply(c, nb, psi, ldpsi, hpsi, ldh, st, t0, t1, t2))) return s;
      c->timer.mark(kStNlProj, t0, t1);
      c->timer.mark(kStNlExpand, t1, t2);
      return kOk;
    }
    if (t0) cudaEventRecord(t0, st);
    // P = X^H psi (hk_psi_nl_c16.f90:82); hpsi += (X D) P (:87-96)
    bs = cublasZgemm(c->blas, CUBLAS_OP_C, CUBLAS_OP_N, c->nanl, nb, c->mtxd, &one, (const cuDoubleComplex*)c->anl.p,
                     c->mtxd, (const cuDoubleComplex*)psi, (int)ldpsi, &zero, (cuDoubleComplex*)c->proj.p, c->nanl);
    if (bs != CUBLAS_STATUS_SUCCESS) return blas_fail(bs, "zgemm X^H psi");
    if (t1) cudaEventRecord(t1, st);
    bs = cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, c->mtxd, nb, c->nanl, &one, (const cuDoubleComplex*)c->anld.p,
                     c->mtxd, (const cuDoubleComplex*)c->proj.p, c->nanl, &one, (cuDoubleComplex*)hpsi, (int)ldh);
    if (bs != CUBLAS_STATUS_SUCCESS) return blas_fail(bs, "zgemm X D P");
    if (t2) cudaEventRecord(t2, st);
    c->timer.mark(kStNlProj, t0, t1);
    c->timer.mark(kStNlExpand, t1, t2);
  }
  return kOk;
}

}  // namespace cpwb
