// Screened local potential on the FFT mesh built on the device: the step before H|psi> in the
// SCF, Src/cpw_lib/pot_local.f90:104-186. The potential given per star (veff, one value per
// prototype G) is unfolded onto the mesh (Src/mesh/mesh_unfold.f90 with lwrap: every G of
// every star, value veff(star) conj(phase) or conj(veff(star)) phase by the sign of conj,
// summed where G vectors wrap onto the same point), transformed with the reference's
// unscaled backward transform (e^{+iG.r}, cfft_c16 mode -1), checked to be real (the largest
// imaginary part is returned; pot_local stops above 1e-6) and written as vscr(id, n2, n3)
// together with its extrema. Optionally the result becomes the context's potential without
// leaving the device (the H|psi> kernels read V/N in [z][y][x] order, FP64 and FP32).
//
// The mesh transform is three passes of batched line transforms, one per axis, each line done
// as the same four-step pair of register DFT passes the H|psi> kernels use (csrc/cplx.cuh),
// 16 lines per CTA staged in shared memory.
#include <math.h>
#include <stdio.h>

#include <string>
#include <vector>

#include "context.hpp"

namespace cpwb {

namespace {

constexpr int kLines = 16;
constexpr int kThreads = 256;
constexpr int kRedBlocks = 296;

__global__ void k_unfold(int ng, const int* __restrict__ kgv, const int* __restrict__ inds,
                         const C2<double>* __restrict__ veff, const C2<double>* __restrict__ phase,
                         const double* __restrict__ cj, int n1, int n2, int n3, C2<double>* __restrict__ box) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
    int k1 = kgv[3 * i] % n1, k2 = kgv[3 * i + 1] % n2, k3 = kgv[3 * i + 2] % n3;
    k1 += k1 < 0 ? n1 : 0;
    k2 += k2 < 0 ? n2 : 0;
    k3 += k3 < 0 ? n3 : 0;
    const C2<double> d = veff[inds[i] - 1], ph = phase[i];
    // den * conj(phase), or conj(den) * phase
    const C2<double> v = cj[i] > 0.0 ? mk<double>(d.x * ph.x + d.y * ph.y, d.y * ph.x - d.x * ph.y)
                                     : mk<double>(d.x * ph.x + d.y * ph.y, d.x * ph.y - d.y * ph.x);
    C2<double>* o = box + ((size_t)k3 * n2 + k2) * n1 + k1;
    atomicAdd(&o->x, v.x);
    atomicAdd(&o->y, v.y);
  }
}

// Backward transform (e^{+i}, unscaled) of nlines lines of length n = r1*r2 in place: element e
// of line j sits at (j % nfast) * sfast + (j / nfast) * sslow + e * es.
__global__ void __launch_bounds__(kThreads)
k_lines_backward(C2<double>* __restrict__ box, FftDim d, long long es, long long nfast, long long sfast,
                 long long sslow, long long nlines, const C2<double>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = d.n, r1 = d.r1, r2 = d.r2;
  C2<double>* T = reinterpret_cast<C2<double>*>(smem_raw);
  C2<double>* w = T + (size_t)n * kLines;
  const int tid = threadIdx.x, nt = blockDim.x;
  const long long l0 = (long long)blockIdx.x * kLines;
  const int nl = (int)min((long long)kLines, nlines - l0);
  auto base = [&](int l) { const long long j = l0 + l; return (j % nfast) * sfast + (j / nfast) * sslow; };
  for (int i = tid; i < n; i += nt) w[i] = tw[i];
  if (es == 1) {
    for (int it = tid; it < n * kLines; it += nt) {
      const int e = it % n, l = it / n;
      if (l < nl) T[(size_t)e * kLines + l] = box[base(l) + e];
    }
  } else {
    for (int it = tid; it < n * kLines; it += nt) {
      const int l = it % kLines, e = it / kLines;
      if (l < nl) T[(size_t)e * kLines + l] = box[base(l) + e * es];
    }
  }
  __syncthreads();
  for (int it = tid; it < kLines * r2; it += nt) {
    const int l = it % kLines, n2i = it / kLines;
    if (l < nl) {
      with_radix<0>(r1, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<double> v[RR];
#pragma unroll
        for (int a = 0; a < RR; ++a) v[a] = T[(size_t)(r2 * a + n2i) * kLines + l];
        DFT<RR, +1, double>::run(v);
#pragma unroll
        for (int a = 0; a < RR; ++a)
          T[(size_t)(r2 * a + n2i) * kLines + l] = a == 0 ? v[0] : cmulc<double>(v[a], w[n2i * a]);
      });
    }
  }
  __syncthreads();
  for (int it = tid; it < kLines * r1; it += nt) {
    const int l = it % kLines, k1 = it / kLines;
    if (l < nl) {
      with_radix<0>(r2, [&](auto rc_) {
        constexpr int RR = decltype(rc_)::value;
        C2<double> v[RR];
#pragma unroll
        for (int a = 0; a < RR; ++a) v[a] = T[(size_t)(r2 * k1 + a) * kLines + l];
        DFT<RR, +1, double>::run(v);
        const long long b = base(l);
#pragma unroll
        for (int a = 0; a < RR; ++a) box[b + (long long)(k1 + r1 * a) * es] = v[a];
      });
    }
  }
}

// Real part out (vscr with leading dimension id, and V/N for the H|psi> kernels), per-block
// max / min of the real part and max |imaginary part|.
__global__ void __launch_bounds__(kThreads)
k_pot_finish(const C2<double>* __restrict__ box, int n1, int n2, int n3, int id, double inv,
             double* __restrict__ vscr, double* __restrict__ v64, float* __restrict__ v32,
             double* __restrict__ part) {
  __shared__ double s_max[kThreads], s_min[kThreads], s_im[kThreads];
  double vmax = -INFINITY, vmin = INFINITY, im = 0.0;
  const long long ntot = (long long)n1 * n2 * n3;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ntot; t += (long long)gridDim.x * blockDim.x) {
    const C2<double> v = box[t];
    const long long x = t % n1, yz = t / n1;
    vmax = fmax(vmax, v.x);
    vmin = fmin(vmin, v.x);
    im = fmax(im, fabs(v.y));
    if (vscr) {
      vscr[yz * id + x] = v.x;
      if (x == n1 - 1)
        for (int p = n1; p < id; ++p) vscr[yz * id + p] = 0.0;
    }
    if (v64) {
      v64[t] = v.x * inv;
      v32[t] = (float)(v.x * inv);
    }
  }
  const int tid = threadIdx.x;
  s_max[tid] = vmax;
  s_min[tid] = vmin;
  s_im[tid] = im;
  __syncthreads();
  for (int h = kThreads / 2; h > 0; h >>= 1) {
    if (tid < h) {
      s_max[tid] = fmax(s_max[tid], s_max[tid + h]);
      s_min[tid] = fmin(s_min[tid], s_min[tid + h]);
      s_im[tid] = fmax(s_im[tid], s_im[tid + h]);
    }
    __syncthreads();
  }
  if (tid == 0) {
    part[3 * blockIdx.x] = s_max[0];
    part[3 * blockIdx.x + 1] = s_min[0];
    part[3 * blockIdx.x + 2] = s_im[0];
  }
}

}  // namespace

int ctx_pot_local(cpw_b200_ctx* c, int n1, int n2, int n3, int id, int ng, const int* kgv, const double* veff,
                  const double* phase, const double* conj, const int* inds, double* vscr, double* vmax,
                  double* vmin, double* cmax, bool install) {
  if (install && (!c->have_basis || c->plan.n1 != n1 || c->plan.n2 != n2 || c->plan.n3 != n3))
    return fail(kNotReady, "pot_local: the context's k-point box differs from the potential's mesh");
  FftDim dims[3];
  const int ns[3] = {n1, n2, n3};
  for (int a = 0; a < 3; ++a)
    if (!factor(ns[a], dims[a])) return fail(kUnsupported, "pot_local: FFT length is not a product of two supported radices");
  const size_t ntot = (size_t)n1 * n2 * n3;
  int s;
  int nst = 0;
  for (int i = 0; i < ng; ++i) nst = inds[i] > nst ? inds[i] : nst;
  DevBuf d_kgv, d_inds, d_veff, d_phase, d_conj, box, d_vscr, part, tw[3];
  if ((s = box.ensure(ntot * sizeof(C2<double>)))) return s;
  if ((s = part.ensure((size_t)3 * kRedBlocks * sizeof(double)))) return s;
  if (ng > 0 &&
      ((s = upload(d_kgv, kgv, (size_t)3 * ng * sizeof(int))) || (s = upload(d_inds, inds, (size_t)ng * sizeof(int))) ||
       (s = upload(d_veff, veff, (size_t)nst * sizeof(C2<double>))) ||
       (s = upload(d_phase, phase, (size_t)ng * sizeof(C2<double>))) ||
       (s = upload(d_conj, conj, (size_t)ng * sizeof(double)))))
    return s;
  for (int a = 0; a < 3; ++a) {
    std::vector<double> t;
    twiddles(ns[a], t);
    if ((s = upload(tw[a], t.data(), t.size() * sizeof(double)))) return s;
  }
  if (vscr && (s = d_vscr.ensure((size_t)id * n2 * n3 * sizeof(double)))) return s;
  if (install && ((s = c->v64.ensure(ntot * sizeof(double))) || (s = c->v32.ensure(ntot * sizeof(float))))) return s;
  cudaStream_t st = c->stream;
  cudaError_t e = cudaMemsetAsync(box.p, 0, ntot * sizeof(C2<double>), st);
  if (e != cudaSuccess) return cuda_fail(e, "pot_local memset");
  if (ng > 0)
    k_unfold<<<(ng + kThreads - 1) / kThreads, kThreads, 0, st>>>(
        ng, (const int*)d_kgv.p, (const int*)d_inds.p, (const C2<double>*)d_veff.p, (const C2<double>*)d_phase.p,
        (const double*)d_conj.p, n1, n2, n3, (C2<double>*)box.p);
  // x lines (contiguous), y lines (stride n1), z lines (stride n1 n2); lines numbered x-fastest
  const long long es[3] = {1, n1, (long long)n1 * n2};
  const long long nfast[3] = {n2, n1, n1};
  const long long sfast[3] = {n1, 1, 1};
  const long long sslow[3] = {(long long)n1 * n2, (long long)n1 * n2, n1};
  for (int a = 0; a < 3; ++a) {
    const long long nlines = (long long)(ntot / ns[a]);
    const size_t sm = sizeof(C2<double>) * ((size_t)ns[a] * kLines + ns[a]);
    if ((e = smem_limit((const void*)k_lines_backward, (size_t)sm)) != cudaSuccess)
      return cuda_fail(e, "pot_local attribute");
    k_lines_backward<<<(unsigned)((nlines + kLines - 1) / kLines), kThreads, sm, st>>>(
        (C2<double>*)box.p, dims[a], es[a], nfast[a], sfast[a], sslow[a], nlines, (const C2<double>*)tw[a].p);
  }
  k_pot_finish<<<kRedBlocks, kThreads, 0, st>>>((const C2<double>*)box.p, n1, n2, n3, id, 1.0 / (double)ntot,
                                                 vscr ? (double*)d_vscr.p : nullptr,
                                                 install ? (double*)c->v64.p : nullptr,
                                                 install ? (float*)c->v32.p : nullptr, (double*)part.p);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "pot_local kernels");
  std::vector<double> hp((size_t)3 * kRedBlocks);
  if ((e = cudaMemcpyAsync(hp.data(), part.p, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return cuda_fail(e, "pot_local copy");
  if (vscr && (e = cudaMemcpyAsync(vscr, d_vscr.p, (size_t)id * n2 * n3 * sizeof(double), cudaMemcpyDeviceToHost, st)) !=
                  cudaSuccess)
    return cuda_fail(e, "pot_local copy");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "pot_local");
  double mx = -INFINITY, mn = INFINITY, im = 0.0;
  for (int b = 0; b < kRedBlocks; ++b) {
    mx = fmax(mx, hp[3 * b]);
    mn = fmin(mn, hp[3 * b + 1]);
    im = fmax(im, hp[3 * b + 2]);
  }
  if (vmax) *vmax = mx;
  if (vmin) *vmin = mn;
  if (cmax) *cmax = im;
  // pot_local.f90:168-175 stops when the potential is not real
  if (im > 1000.0 * 1e-9) {
    if (install) c->have_pot = false;
    char buf[120];
    snprintf(buf, sizeof buf, "pot_local: complex potential, cmax = %.4e", im);
    return fail(kBadArg, buf);
  }
  if (install) {
    c->pot_n[0] = n1; c->pot_n[1] = n2; c->pot_n[2] = n3;
    c->have_pot = true;
  }
  return kOk;
}

}  // namespace cpwb
