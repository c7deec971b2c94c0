// The small dense Hamiltonian of the eigensolver's start basis on the device, the set-up step
// Src/ALFA/hamilt_kb.f90:1-234 (called per k-point through h_kb_dia before ditsp_c16):
//   hamk(i, i) = hdiag(i)
//   hamk(i, j) = veff(s) conj(phase(n)) + sum_type [sum_l vq_l(q_i) vq_l(q_j) nkb_l P_l(cos)]
//                sfact(type, s) conj(phase(n))  (conjugated when conj(n) = -1),   i > j,
// with n the G vector G_i - G_j (through the cube index indv), s its star, q = |k + G|,
// vq_l(q) = v_l(q) q^l / sqrt(vcell) from the quadratic interpolation of the KB table, cos the
// angle between k + G_i and k + G_j from |G_i - G_j|^2 = 2 ek(s), and hamk(j, i) = conj(hamk(i, j)).
//
// The reference fills the mtxd^2 / 2 entries in one loop on the host, recomputing vq for both
// plane waves of every pair. Here one kernel tabulates vq_l(q_i) per plane wave and type, and a
// second computes one entry per thread (both triangles written), straight into device memory
// where the eigensolver reads it.
#include <math.h>
#include <stdio.h>

#include <vector>

#include "../../include/cpw_b200.h"
#include "context.hpp"

namespace cpwb {
namespace {

constexpr int kLmaxH = 3;

// fac v_l(q) q^l for every plane wave, type and l (hamilt_kb.f90:172-198): out[(i * ntype + t) * 4 + l]
__global__ void k_hk_vq(int mtxd, int ntype, const double* __restrict__ qmod, const double* __restrict__ vkb,
                        int row, const int* __restrict__ nqnl, const double* __restrict__ delq,
                        const int* __restrict__ nkb, double fac, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= mtxd) return;
  const double q = qmod[i];
  for (int t = 0; t < ntype; ++t) {
    const double xn = q / delq[t];
    int n = (int)floor(xn + 0.5);
    if (n < 0) n = 0;
    for (int l = 0; l <= kLmaxH; ++l) {
      double v = 0.0;
      if (n < nqnl[t] - 1 && nkb[t * 4 + l] != 0) {
        const double* tab = vkb + ((size_t)t * 4 + l) * row + 2;      // tab[n] = vkb(n)
        const double x = xn - n;
        v = tab[n] * (1.0 + x) * (1.0 - x) + (tab[n + 1] * (1.0 + x) - tab[n - 1] * (1.0 - x)) * x / 2;
        double ql = 1.0;
        for (int p = 0; p < l; ++p) ql *= q;
        v = fac * v * ql;
      }
      out[((size_t)i * ntype + t) * 4 + l] = v;
    }
  }
}

struct HkArgs {
  int mtxd, ntype;
  const double* hdiag;
  const int* isort;          // 0-based into kgv
  const double* qmod;
  const int* kgv;            // (3, ng)
  const double2* phase;
  const double* conj;
  const int* inds;           // 0-based stars
  int kmax[3];
  const int* indv;           // 1-based G index per cube point, 0 = none
  const double* ek;
  const double2* sfact;      // (mxdtyp, ns)
  int ldsf;
  const double2* veff;
  const double* vq;          // k_hk_vq's table
  const int* nkb;            // (ntype, 4)
  double2* hamk;
  long long ldh;
};

__global__ void k_hamilt_kb(HkArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (i >= a.mtxd || j >= a.mtxd) return;
  if (j == i) {
    a.hamk[(size_t)i * a.ldh + i] = make_double2(a.hdiag[i], 0.0);
    return;
  }
  if (j > i) return;
  double2 h = make_double2(0.0, 0.0);
  const int gi = a.isort[i], gj = a.isort[j];
  const int imx = 2 * a.kmax[0] + 1, jmx = 2 * a.kmax[1] + 1, kmx = 2 * a.kmax[2] + 1;
  const int kxd = a.kgv[3 * gi] - a.kgv[3 * gj] + a.kmax[0] + 1;
  const int kyd = a.kgv[3 * gi + 1] - a.kgv[3 * gj + 1] + a.kmax[1] + 1;
  const int kzd = a.kgv[3 * gi + 2] - a.kgv[3 * gj + 2] + a.kmax[2] + 1;
  if (kxd >= 1 && kxd <= imx && kyd >= 1 && kyd <= jmx && kzd >= 1 && kzd <= kmx) {
    const int kadd = a.indv[((size_t)(kxd - 1) * jmx + kyd - 1) * kmx + kzd - 1];
    if (kadd != 0) {
      const int n = kadd - 1, st = a.inds[n];
      const double2 ph = make_double2(a.phase[n].x, -a.phase[n].y);     // conjg(phase)
      const double2 ve = a.veff[st];
      h = make_double2(ve.x * ph.x - ve.y * ph.y, ve.x * ph.y + ve.y * ph.x);
      const double qi = a.qmod[i], qj = a.qmod[j];
      const double eps = (double)1.0e-9f;                                 // a default-real literal (:92)
      double gama = 1.0;
      if (qi > eps && qj > eps) gama = (qi * qi + qj * qj - 2 * a.ek[st]) / (qi * qj * 2);
      const double plg[4] = {1.0, gama, (3 * gama * gama - 1.0) / 2, gama * (5 * gama * gama - 3.0) / 2};
      for (int t = 0; t < a.ntype; ++t) {
        const double* vi = a.vq + ((size_t)i * a.ntype + t) * 4;
        const double* vj = a.vq + ((size_t)j * a.ntype + t) * 4;
        double vnl = 0.0;
        for (int l = 0; l <= kLmaxH; ++l) vnl += vi[l] * vj[l] * a.nkb[t * 4 + l] * plg[l];
        const double2 sf = a.sfact[(size_t)st * a.ldsf + t];
        const double2 sp = make_double2(sf.x * ph.x - sf.y * ph.y, sf.x * ph.y + sf.y * ph.x);
        h.x += vnl * sp.x;
        h.y += vnl * sp.y;
      }
      if (a.conj[n] < 0.0) h.y = -h.y;
    }
  }
  a.hamk[(size_t)j * a.ldh + i] = h;
  a.hamk[(size_t)i * a.ldh + j] = make_double2(h.x, -h.y);
}

// metric determinant (vcell^2), as adot_to_bdot computes the volume
double det3(const double* m) {
  return m[0] * (m[4] * m[8] - m[7] * m[5]) - m[3] * (m[1] * m[8] - m[7] * m[2]) + m[6] * (m[1] * m[5] - m[4] * m[2]);
}

}  // namespace

int hamilt_kb_device(cpw_b200_ctx* c, int mtxd, const double* hdiag, const int* isort, const double* qmod, int ng,
                     const int* kgv, const double* phase, const double* conj, const int* inds, const int* kmax,
                     const int* indv, const double* ek, const double* sfact, const double* veff, const int* nqnl,
                     const double* delqnl, const double* vkb, const int* nkb, int ntype, const double* adot,
                     void* hamk, long long ldh, int mxdtyp, int mxdgve, int mxdnst, int mxdcub, int mxdlqp,
                     int mxddim) {
  if (mtxd < 0 || mtxd > mxddim) return fail(kBadArg, "hamilt_kb: mtxd out of range of mxddim");
  if (ng > mxdgve) return fail(kBadArg, "hamilt_kb: ng > mxdgve");
  if (ntype < 0 || ntype > mxdtyp) return fail(kBadArg, "hamilt_kb: ntype out of range of mxdtyp");
  if (ldh < mtxd) return fail(kBadArg, "hamilt_kb: leading dimension of hamk smaller than mtxd");
  if (mtxd == 0) return kOk;
  if (!hamk) return fail(kBadArg, "hamilt_kb: null hamk");
  const long long ncube = (long long)(2 * kmax[0] + 1) * (2 * kmax[1] + 1) * (2 * kmax[2] + 1);
  if (ncube > mxdcub) return fail(kBadArg, "hamilt_kb: cube of kmax larger than mxdcub");
  int ns = 0;
  for (int n = 0; n < ng; ++n) {
    if (inds[n] < 1 || inds[n] > mxdnst) return fail(kBadArg, "hamilt_kb: inds out of range of mxdnst");
    ns = std::max(ns, inds[n]);
  }
  for (int i = 0; i < mtxd; ++i)
    if (isort[i] < 1 || isort[i] > ng) return fail(kBadArg, "hamilt_kb: isort out of range of ng");
  for (long long t = 0; t < ncube; ++t)
    if (indv[t] < 0 || indv[t] > ng) return fail(kBadArg, "hamilt_kb: indv out of range of ng");
  const double vc2 = det3(adot);
  if (!(vc2 > 1e-10)) return fail(kBadArg, "hamilt_kb: metric adot not positive definite");
  const double fac = 1.0 / sqrt(sqrt(vc2));
  int nqmax = 0;
  for (int t = 0; t < ntype; ++t) {
    if (nqnl[t] > mxdlqp) return fail(kBadArg, "hamilt_kb: nqnl > mxdlqp");
    nqmax = std::max(nqmax, nqnl[t]);
  }
  // host staging in compact layouts: 0-based indices, kgv (3, ng), vkb rows of nqmax + 3 from q
  // index -2 for spin-orbit channel 0, nkb (ntype, 4)
  std::vector<int> is0(mtxd), in0(std::max(ng, 1)), nk(std::max(ntype, 1) * 4, 0);
  for (int i = 0; i < mtxd; ++i) is0[i] = isort[i] - 1;
  for (int n = 0; n < ng; ++n) in0[n] = inds[n] - 1;
  const int row = nqmax + 3;
  std::vector<double> tab((size_t)std::max(ntype, 1) * 4 * row, 0.0);
  const size_t ldq = (size_t)mxdlqp + 3;
  for (int t = 0; t < ntype; ++t)
    for (int l = 0; l <= kLmaxH; ++l) {
      nk[t * 4 + l] = nkb[l + 4 * (1 + 3 * t)];                    // nkb(l, 0, t)
      const double* src = vkb + ldq * (l + 4 * (1 + 3 * (size_t)t));
      for (int n = 0; n < nqnl[t] + 3 && n < (int)ldq; ++n) tab[((size_t)t * 4 + l) * row + n] = src[n];
    }
  int s;
  DevBuf d_hd, d_is, d_q, d_kgv, d_ph, d_cj, d_in, d_indv, d_ek, d_sf, d_ve, d_tab, d_nq, d_dq, d_nk, d_vq;
  if ((s = upload(d_hd, hdiag, sizeof(double) * mtxd)) || (s = upload(d_is, is0.data(), sizeof(int) * mtxd)) ||
      (s = upload(d_q, qmod, sizeof(double) * mtxd)) || (s = upload(d_kgv, kgv, sizeof(int) * 3 * (size_t)ng)) ||
      (s = upload(d_ph, phase, 16 * (size_t)ng)) || (s = upload(d_cj, conj, sizeof(double) * (size_t)ng)) ||
      (s = upload(d_in, in0.data(), sizeof(int) * (size_t)ng)) ||
      (s = upload(d_indv, indv, sizeof(int) * (size_t)ncube)) || (s = upload(d_ek, ek, sizeof(double) * (size_t)ns)) ||
      (s = upload(d_sf, sfact, 16 * (size_t)mxdtyp * ns)) || (s = upload(d_ve, veff, 16 * (size_t)ns)) ||
      (s = upload(d_tab, tab.data(), sizeof(double) * tab.size())) ||
      (s = upload(d_nq, nqnl, sizeof(int) * (size_t)std::max(ntype, 1))) ||
      (s = upload(d_dq, delqnl, sizeof(double) * (size_t)std::max(ntype, 1))) ||
      (s = upload(d_nk, nk.data(), sizeof(int) * nk.size())) ||
      (s = d_vq.ensure(sizeof(double) * 4 * (size_t)mtxd * std::max(ntype, 1))))
    return s;
  cudaStream_t st = c->stream;
  k_hk_vq<<<(mtxd + 127) / 128, 128, 0, st>>>(mtxd, ntype, (const double*)d_q.p, (const double*)d_tab.p, row,
                                              (const int*)d_nq.p, (const double*)d_dq.p, (const int*)d_nk.p, fac,
                                              (double*)d_vq.p);
  HkArgs a{};
  a.mtxd = mtxd;
  a.ntype = ntype;
  a.hdiag = (const double*)d_hd.p;
  a.isort = (const int*)d_is.p;
  a.qmod = (const double*)d_q.p;
  a.kgv = (const int*)d_kgv.p;
  a.phase = (const double2*)d_ph.p;
  a.conj = (const double*)d_cj.p;
  a.inds = (const int*)d_in.p;
  for (int k = 0; k < 3; ++k) a.kmax[k] = kmax[k];
  a.indv = (const int*)d_indv.p;
  a.ek = (const double*)d_ek.p;
  a.sfact = (const double2*)d_sf.p;
  a.ldsf = mxdtyp;
  a.veff = (const double2*)d_ve.p;
  a.vq = (const double*)d_vq.p;
  a.nkb = (const int*)d_nk.p;
  a.hamk = (double2*)hamk;
  a.ldh = ldh;
  k_hamilt_kb<<<dim3((unsigned)((mtxd + 127) / 128), (unsigned)mtxd), 128, 0, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "hamilt_kb kernels");
  // the staging buffers are freed at return: finish with them first
  e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? kOk : cuda_fail(e, "hamilt_kb");
}

}  // namespace cpwb
