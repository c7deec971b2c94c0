// Kleinman-Bylander projectors of one k-point built on the device, the set-up step of
// Src/omp/proj_nl_kb_c16.f90:23-275 (called once per k-point before hk_psi_c16, through
// h_kb_dia): anlga(i, ind) = e^{-2 pi i G_i.tau} * rylm_lm(k+G_i) * i^l * v_l(|k+G_i|) / sqrt(vcell)
// with v_l quadratically interpolated in the (1/q^l) KB table (:226-240), projector order
// type -> l -> m -> atom (:170-184) and xnlkb(ind) = nkb(l, type) (:266).
//
// The reference fills anlga on the host with one OpenMP thread per plane wave and the caller
// then uploads mtxd x nanl complex numbers (Si216: 1.2 GB) for every k-point. Here one thread
// per plane wave computes k+G, |k+G| and the solid harmonics once, then writes a chunk of
// projector columns (coalesced over plane waves), both X and X.diag(xnlkb), straight into the
// context. The phase uses sincospi of -2 G.tau (the product 2 pi G.tau is never rounded).
#include <math.h>
#include <stdio.h>

#include <string>
#include <vector>

#include "context.hpp"

namespace cpwb {

namespace {

constexpr int kLmax = 3;            // hard-coded maximum angular momentum of the reference (LMAX)
constexpr int kProjPerThread = 16;  // projector columns written by one thread

struct ProjEntry {
  int type, atom, l, m;             // atom: index into the packed tau array
};

struct ProjGeom {
  double bvec[9];                   // column-major, bvec(:, j) = b_j
  double rk[3];
  double fac;                       // 1/sqrt(vcell)
  int nq_max;                       // table row length is nq_max + 3 (q index -2 .. nq_max)
};

// r^l sqrt(4 pi/(2l+1)) times the real combinations of Y_lm, Src/numeric/ylm_rc.f90:82-106
// (the same polynomials as the host restatement).
__device__ __forceinline__ double rylm_lm(int l, int m, double x, double y, double z) {
  switch (l) {
    case 0:
      return 1.0;
    case 1:
      return m < 0 ? y : (m == 0 ? z : x);
    case 2: {
      const double s3 = 1.7320508075688772935;
      switch (m) {
        case -2: return s3 * x * y;
        case -1: return s3 * z * y;
        case 0: return 0.5 * (2 * z * z - x * x - y * y);
        case 1: return s3 * z * x;
        default: return 0.8660254037844386468 * (x * x - y * y);
      }
    }
    default: {
      switch (m) {
        case -3: return 0.7905694150420948330 * (3 * x * x - y * y) * y;
        case -2: return 3.8729833462074168852 * z * x * y;
        case -1: return 0.6123724356957945245 * (4 * z * z - x * x - y * y) * y;
        case 0: return 0.5 * (2 * z * z - 3 * x * x - 3 * y * y) * z;
        case 1: return 0.6123724356957945245 * (4 * z * z - x * x - y * y) * x;
        case 2: return 1.9364916731037084426 * (x * x - y * y) * z;
        default: return -0.7905694150420948330 * (3 * y * y - x * x) * x;
      }
    }
  }
}

__global__ void __launch_bounds__(128)
k_proj_nl_kb(int mtxd, int nanl, const int* __restrict__ kgvb, ProjGeom g, const ProjEntry* __restrict__ ent,
             const double* __restrict__ tau, const double* __restrict__ vkb, const int* __restrict__ nqnl,
             const double* __restrict__ delq, const double* __restrict__ xnl, C2<double>* __restrict__ anl,
             C2<double>* __restrict__ anld, long long ld) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= mtxd) return;
  const int p0 = blockIdx.y * kProjPerThread;
  const int p1 = min(nanl, p0 + kProjPerThread);
  const double g0 = kgvb[3 * i], g1 = kgvb[3 * i + 1], g2 = kgvb[3 * i + 2];
  const double q0 = g.rk[0] + g0, q1 = g.rk[1] + g1, q2 = g.rk[2] + g2;
  const double x = g.bvec[0] * q0 + g.bvec[3] * q1 + g.bvec[6] * q2;
  const double y = g.bvec[1] * q0 + g.bvec[4] * q1 + g.bvec[7] * q2;
  const double z = g.bvec[2] * q0 + g.bvec[5] * q1 + g.bvec[8] * q2;
  const double qi = sqrt(x * x + y * y + z * z);
  const int row = g.nq_max + 3;
  for (int ind = p0; ind < p1; ++ind) {
    const ProjEntry e = ent[ind];
    // structure phase e^{-2 pi i G.tau} (proj_nl_kb_c16.f90:210-218)
    const double* t = tau + 3 * e.atom;
    double s, c;
    sincospi(-2.0 * (g0 * t[0] + g1 * t[1] + g2 * t[2]), &s, &c);
    // v_l(q) by quadratic interpolation (:226-240); nint rounds halves away from zero
    const double xni = qi / delq[e.type];
    int ni = (int)floor(xni + 0.5);
    if (ni < 0) ni = 0;
    double vq = 0.0;
    if (ni < nqnl[e.type] - 1) {
      const double* v = vkb + ((size_t)e.type * (kLmax + 1) + e.l) * row + 2;   // v[n] = vkb(n)
      const double xi = xni - ni;
      vq = v[ni] * (1.0 + xi) * (1.0 - xi) + 0.5 * (v[ni + 1] * (1.0 + xi) - v[ni - 1] * (1.0 - xi)) * xi;
      vq *= g.fac;
    }
    const double r = rylm_lm(e.l, e.m, x, y, z) * vq;
    // (c + i s) * r * i^l
    double re = c * r, im = s * r;
    switch (e.l & 3) {
      case 1: { const double t0 = re; re = -im; im = t0; break; }
      case 2: re = -re; im = -im; break;
      case 3: { const double t0 = re; re = im; im = -t0; break; }
      default: break;
    }
    const size_t o = (size_t)ind * ld + i;
    anl[o] = mk<double>(re, im);
    anld[o] = mk<double>(re * xnl[ind], im * xnl[ind]);
  }
}

// avec by the Cholesky-type factorisation of the metric (Src/crystal/adot_to_avec.f90),
// bvec = 2 pi avec^{-T}; returns false when the metric is not positive definite.
bool adot_to_bvec(const double* adot, double* bvec, double* vcell) {
  auto A = [&](int r, int c) { return adot[r + 3 * c]; };
  double a[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};   // a[row][col]
  if (A(0, 0) < 1e-10) return false;
  a[0][0] = sqrt(A(0, 0));
  a[0][1] = A(0, 1) / a[0][0];
  const double a22 = A(1, 1) - a[0][1] * a[0][1];
  if (a22 < 1e-10) return false;
  a[1][1] = sqrt(a22);
  a[0][2] = A(0, 2) / a[0][0];
  a[1][2] = (A(1, 2) - a[0][1] * a[0][2]) / a[1][1];
  const double a33 = A(2, 2) - a[1][2] * a[1][2] - a[0][2] * a[0][2];
  if (a33 < 1e-10) return false;
  a[2][2] = sqrt(a33);
  // inverse of the upper-triangular avec
  double inv[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  inv[0][0] = 1 / a[0][0];
  inv[1][1] = 1 / a[1][1];
  inv[2][2] = 1 / a[2][2];
  inv[0][1] = -a[0][1] * inv[1][1] * inv[0][0];
  inv[1][2] = -a[1][2] * inv[2][2] * inv[1][1];
  inv[0][2] = -(a[0][1] * inv[1][2] + a[0][2] * inv[2][2]) * inv[0][0];
  const double twopi = 6.283185307179586476925286766559;
  for (int r = 0; r < 3; ++r)
    for (int cc = 0; cc < 3; ++cc) bvec[r + 3 * cc] = twopi * inv[cc][r];   // (avec^{-1})^T
  *vcell = a[0][0] * a[1][1] * a[2][2];
  return true;
}

}  // namespace

int ctx_proj_nl_kb(cpw_b200_ctx* c, const double* rkpt, int ntype, const int* natom, const double* rat, int mxdatm,
                   const double* adot, const int* nqnl, const double* delqnl, const double* vkb, int mxdlqp,
                   const int* nkb, int nanl, double* xnlkb_out, void* anlga_out, long long ld_out) {
  if (!c->have_basis) return fail(kNotReady, "proj_nl_kb: call set_basis first");
  if (ntype < 0 || mxdatm < 0 || mxdlqp < 0 || nanl < 0) return fail(kBadArg, "proj_nl_kb: negative dimension");
  const long long m = c->mtxd;
  // projector table and the consistency checks of proj_nl_kb_c16.f90:133-166
  auto nkb_at = [&](int l, int k) { return nkb[l + (kLmax + 1) * (1 + 3 * k)]; };   // nkb(l, 0, k)
  std::vector<ProjEntry> ent;
  std::vector<double> xnl, tau;
  std::vector<int> atom0(ntype + 1, 0);
  int lmx = 0;
  for (int k = 0; k < ntype; ++k) {
    if (natom[k] < 0 || natom[k] > mxdatm) return fail(kBadArg, "proj_nl_kb: natom out of range of mxdatm");
    atom0[k + 1] = atom0[k] + natom[k];
    for (int l = 0; l <= kLmax; ++l)
      if (nkb_at(l, k) != 0) lmx = l > lmx ? l : lmx;
  }
  for (int k = 0; k < ntype; ++k)
    for (int a = 0; a < natom[k]; ++a)
      for (int j = 0; j < 3; ++j) tau.push_back(rat[j + 3 * (a + (size_t)mxdatm * k)]);
  for (int k = 0; k < ntype; ++k)
    for (int l = 0; l <= lmx; ++l) {
      if (nkb_at(l, k) == 0) continue;
      for (int mm = -l; mm <= l; ++mm)
        for (int a = 0; a < natom[k]; ++a) {
          ent.push_back(ProjEntry{k, atom0[k] + a, l, mm});
          xnl.push_back((double)nkb_at(l, k));
        }
    }
  if ((int)ent.size() != nanl) {
    char buf[160];
    snprintf(buf, sizeof buf, "proj_nl_kb: inconsistent value of nanl %d should be %d", nanl, (int)ent.size());
    return fail(kBadArg, buf);
  }
  int nq_max = 0;
  for (int k = 0; k < ntype; ++k) {
    if (nqnl[k] > mxdlqp) return fail(kBadArg, "proj_nl_kb: nqnl > mxdlqp");
    if (delqnl[k] <= 0 && nqnl[k] > 1) return fail(kBadArg, "proj_nl_kb: delqnl not positive");
    nq_max = nqnl[k] > nq_max ? nqnl[k] : nq_max;
  }
  ProjGeom g{};
  double vcell = 0;
  if (!adot_to_bvec(adot, g.bvec, &vcell)) return fail(kBadArg, "proj_nl_kb: metric adot not positive definite");
  for (int j = 0; j < 3; ++j) g.rk[j] = rkpt[j];
  g.fac = 1.0 / sqrt(vcell);
  g.nq_max = nq_max;
  // vkb(-2:nq, l, 0, k) of every type and l, rows of nq_max + 3
  const int row = nq_max + 3;
  std::vector<double> tab((size_t)(ntype > 0 ? ntype : 1) * (kLmax + 1) * row, 0.0);
  const size_t ldq = (size_t)mxdlqp + 3;
  for (int k = 0; k < ntype; ++k)
    for (int l = 0; l <= kLmax; ++l) {
      const double* src = vkb + ldq * (l + (kLmax + 1) * (1 + 3 * (size_t)k));
      for (int n = 0; n < nqnl[k] + 3 && n < (int)ldq; ++n) tab[((size_t)k * (kLmax + 1) + l) * row + n] = src[n];
    }

  c->nanl = nanl;
  c->tc_ready = false;
  if (xnlkb_out)
    for (int j = 0; j < nanl; ++j) xnlkb_out[j] = xnl[j];
  c->xnl_h = xnl;
  if (nanl == 0 || m == 0) return kOk;
  int s;
  const size_t bytes = (size_t)m * nanl * sizeof(C2<double>);
  if ((s = c->anl.ensure(bytes)) || (s = c->anld.ensure(bytes))) return s;
  DevBuf d_ent, d_tau, d_tab, d_nq, d_dq, d_xnl;
  if ((s = upload(d_ent, ent.data(), ent.size() * sizeof(ProjEntry))) ||
      (s = upload(d_tau, tau.data(), tau.size() * sizeof(double))) ||
      (s = upload(d_tab, tab.data(), tab.size() * sizeof(double))) ||
      (s = upload(d_nq, nqnl, (size_t)ntype * sizeof(int))) ||
      (s = upload(d_dq, delqnl, (size_t)ntype * sizeof(double))) ||
      (s = upload(d_xnl, xnl.data(), xnl.size() * sizeof(double))))
    return s;
  const dim3 grid((unsigned)((m + 127) / 128), (unsigned)((nanl + kProjPerThread - 1) / kProjPerThread));
  k_proj_nl_kb<<<grid, 128, 0, c->stream>>>((int)m, nanl, (const int*)c->kgvb.p, g, (const ProjEntry*)d_ent.p,
                                            (const double*)d_tau.p, (const double*)d_tab.p, (const int*)d_nq.p,
                                            (const double*)d_dq.p, (const double*)d_xnl.p, (C2<double>*)c->anl.p,
                                            (C2<double>*)c->anld.p, m);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "proj_nl_kb kernel");
  if (anlga_out) {
    if (ld_out < m) return fail(kBadArg, "proj_nl_kb: leading dimension of anlga smaller than mtxd");
    e = cudaMemcpy2DAsync(anlga_out, (size_t)ld_out * sizeof(C2<double>), c->anl.p, (size_t)m * sizeof(C2<double>),
                          (size_t)m * sizeof(C2<double>), nanl, cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "proj_nl_kb copy");
  }
  // the small tables are freed at return: finish with them first
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "proj_nl_kb");
  if (c->precision == 2) return tc_prepare_projectors(c);
  return kOk;
}

}  // namespace cpwb
