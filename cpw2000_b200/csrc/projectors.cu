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

// The solid harmonics as homogeneous polynomials: rylm(l, m) = sum of c x^a y^b z^cz over at
// most three monomials (the polynomials of rylm_lm above, Src/numeric/ylm_rc.f90:82-106), so
// that their Cartesian gradient and Hessian (ylm_rc's derivatives for nder = 1, 2) follow from
// the exponents. Entry l*l + l + m.
struct Mono {
  double c;
  int e[3];
};
__constant__ Mono c_mono[16][3];
__constant__ int c_nmono[16];

// value, gradient g[k] and Hessian h[3 i + j] of rylm(l, m) from the powers p[k][0..3] of x, y, z
__device__ __forceinline__ void rylm_der(int l, int m, const double (&p)[3][4], double& v, double (&g)[3],
                                         double (&h)[9]) {
  const int idx = l * l + l + m;
  v = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) g[k] = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) h[k] = 0.0;
  for (int t = 0; t < c_nmono[idx]; ++t) {
    const Mono mo = c_mono[idx][t];
    v += mo.c * p[0][mo.e[0]] * p[1][mo.e[1]] * p[2][mo.e[2]];
    for (int i = 0; i < 3; ++i) {
      if (mo.e[i] == 0) continue;
      int ei[3] = {mo.e[0], mo.e[1], mo.e[2]};
      const double ci = mo.c * ei[i];
      --ei[i];
      g[i] += ci * p[0][ei[0]] * p[1][ei[1]] * p[2][ei[2]];
      for (int j = 0; j < 3; ++j) {
        if (ei[j] == 0) continue;
        int ej[3] = {ei[0], ei[1], ei[2]};
        const double cj = ci * ej[j];
        --ej[j];
        h[3 * i + j] += cj * p[0][ej[0]] * p[1][ej[1]] * p[2][ej[2]];
      }
    }
  }
}

// multiply (re, im) by i^l
__device__ __forceinline__ C2<double> times_il(double re, double im, int l) {
  switch (l & 3) {
    case 1: return mk<double>(-im, re);
    case 2: return mk<double>(-re, -im);
    case 3: return mk<double>(im, -re);
    default: return mk<double>(re, im);
  }
}

// Src/omp/proj_nl_kb_der_c16.f90:190-396: the projectors and, for nder >= 1, 2, their first and
// second derivatives with respect to the k-point's lattice coordinates, one thread per plane wave
// and a chunk of projector columns. Layouts of the reference: anl(ld, nanl), dan(ld, mxdanl, 3),
// d2an(ld, mxdanl, 3, 3).
__global__ void __launch_bounds__(128)
k_proj_nl_kb_der(int mtxd, int nanl, int nder, const int* __restrict__ kgvb, ProjGeom g, const double* __restrict__ bdot,
                 const ProjEntry* __restrict__ ent, const double* __restrict__ tau, const double* __restrict__ vkb,
                 const int* __restrict__ nqnl, const double* __restrict__ delq, C2<double>* __restrict__ anl,
                 C2<double>* __restrict__ dan, C2<double>* __restrict__ d2an, long long ld, long long mxdanl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= mtxd) return;
  const int p0 = blockIdx.y * kProjPerThread;
  const int p1 = min(nanl, p0 + kProjPerThread);
  const double g0 = kgvb[3 * i], g1 = kgvb[3 * i + 1], g2 = kgvb[3 * i + 2];
  const double qk[3] = {g.rk[0] + g0, g.rk[1] + g1, g.rk[2] + g2};
  double qc[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) qc[r] = g.bvec[r] * qk[0] + g.bvec[r + 3] * qk[1] + g.bvec[r + 6] * qk[2];
  const double qi = sqrt(qc[0] * qc[0] + qc[1] * qc[1] + qc[2] * qc[2]);
  // |k+G| and its derivatives in lattice coordinates (:196-228); ill defined at q -> 0
  const bool lqi = qi > 1.0e-8;
  double dq[3] = {0, 0, 0}, d2q[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (lqi) {
#pragma unroll
    for (int n = 0; n < 3; ++n) dq[n] = (bdot[n] * qk[0] + bdot[n + 3] * qk[1] + bdot[n + 6] * qk[2]) / qi;
#pragma unroll
    for (int n = 0; n < 3; ++n)
#pragma unroll
      for (int mm = 0; mm < 3; ++mm) d2q[3 * n + mm] = bdot[n + 3 * mm] / qi - dq[n] * dq[mm] / qi;
  }
  double pw[3][4];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    pw[k][0] = 1.0;
    pw[k][1] = qc[k];
    pw[k][2] = qc[k] * qc[k];
    pw[k][3] = pw[k][2] * qc[k];
  }
  const int row = g.nq_max + 3;
  for (int ind = p0; ind < p1; ++ind) {
    const ProjEntry e = ent[ind];
    const double* t = tau + 3 * e.atom;
    double sn, cs;
    sincospi(-2.0 * (g0 * t[0] + g1 * t[1] + g2 * t[2]), &sn, &cs);
    // v_l(q) and its q derivatives from the quadratic interpolation (:259-285)
    const double dl = delq[e.type];
    const double xni = qi / dl;
    int ni = (int)floor(xni + 0.5);
    if (ni < 0) ni = 0;
    double vq = 0.0, dv = 0.0, d2v = 0.0;
    if (ni < nqnl[e.type] - 1) {
      const double* v = vkb + ((size_t)e.type * (kLmax + 1) + e.l) * row + 2;
      const double xi = xni - ni;
      vq = g.fac * (v[ni] * (1.0 + xi) * (1.0 - xi) + 0.5 * (v[ni + 1] * (1.0 + xi) - v[ni - 1] * (1.0 - xi)) * xi);
      dv = g.fac * (-2.0 * xi * v[ni] + 0.5 * (v[ni + 1] * (1.0 + 2.0 * xi) - v[ni - 1] * (1.0 - 2.0 * xi))) / dl;
      d2v = g.fac * (-2.0 * v[ni] + v[ni + 1] + v[ni - 1]) / (dl * dl);
    }
    double ry, gc[3], hc[9];
    rylm_der(e.l, e.m, pw, ry, gc, hc);
    const size_t o = (size_t)ind * ld + i;
    {
      const double r = ry * vq;
      anl[o] = times_il(cs * r, sn * r, e.l);
    }
    if (nder < 1) continue;
    double dr[3];      // drylm/drk(n) = sum_k drylm/dqc(k) bvec(k, n)
#pragma unroll
    for (int n = 0; n < 3; ++n) dr[n] = gc[0] * g.bvec[3 * n] + gc[1] * g.bvec[3 * n + 1] + gc[2] * g.bvec[3 * n + 2];
#pragma unroll
    for (int n = 0; n < 3; ++n) {
      const double r = dr[n] * vq + ry * dv * dq[n];
      dan[(size_t)i + ld * ((size_t)ind + mxdanl * n)] = times_il(cs * r, sn * r, e.l);
    }
    if (nder < 2) continue;
    // d2rylm/drk2(j, n) = sum_{a, b} bvec(a, j) d2rylm/dqc2(a, b) bvec(b, n)
    double hb[9];       // hb[a + 3 n] = sum_b hc(a, b) bvec(b, n)
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int n = 0; n < 3; ++n)
        hb[a + 3 * n] = hc[3 * a] * g.bvec[3 * n] + hc[3 * a + 1] * g.bvec[3 * n + 1] + hc[3 * a + 2] * g.bvec[3 * n + 2];
#pragma unroll
    for (int n = 0; n < 3; ++n)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const double d2r = g.bvec[3 * j] * hb[3 * n] + g.bvec[3 * j + 1] * hb[1 + 3 * n] + g.bvec[3 * j + 2] * hb[2 + 3 * n];
        double r;
        if (lqi) {
          r = d2r * vq + dr[n] * dv * dq[j] + dr[j] * dv * dq[n] + ry * d2v * dq[n] * dq[j] + ry * dv * d2q[3 * j + n];
        } else {
          r = d2r * vq + ry * d2v * bdot[j + 3 * n];
        }
        d2an[(size_t)i + ld * ((size_t)ind + mxdanl * (j + 3 * n))] = times_il(cs * r, sn * r, e.l);
      }
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

// The projector table of proj_nl_kb_c16.f90:133-184 (order type -> l -> m -> atom, with the
// reference's consistency checks), the atom positions, the vkb rows of every type and l, and
// the cell geometry.
struct ProjTables {
  std::vector<ProjEntry> ent;
  std::vector<double> xnl, tau, tab;
  ProjGeom g{};
  double bdot[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
};

int proj_tables(const double* rkpt, int ntype, const int* natom, const double* rat, int mxdatm, const double* adot,
                const int* nqnl, const double* delqnl, const double* vkb, int mxdlqp, const int* nkb, int nanl,
                ProjTables* t) {
  if (ntype < 0 || mxdatm < 0 || mxdlqp < 0 || nanl < 0) return fail(kBadArg, "proj_nl_kb: negative dimension");
  auto nkb_at = [&](int l, int k) { return nkb[l + (kLmax + 1) * (1 + 3 * k)]; };   // nkb(l, 0, k)
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
      for (int j = 0; j < 3; ++j) t->tau.push_back(rat[j + 3 * (a + (size_t)mxdatm * k)]);
  for (int k = 0; k < ntype; ++k)
    for (int l = 0; l <= lmx; ++l) {
      if (nkb_at(l, k) == 0) continue;
      for (int mm = -l; mm <= l; ++mm)
        for (int a = 0; a < natom[k]; ++a) {
          t->ent.push_back(ProjEntry{k, atom0[k] + a, l, mm});
          t->xnl.push_back((double)nkb_at(l, k));
        }
    }
  if ((int)t->ent.size() != nanl) {
    char buf[160];
    snprintf(buf, sizeof buf, "proj_nl_kb: inconsistent value of nanl %d should be %d", nanl, (int)t->ent.size());
    return fail(kBadArg, buf);
  }
  int nq_max = 0;
  for (int k = 0; k < ntype; ++k) {
    if (nqnl[k] > mxdlqp) return fail(kBadArg, "proj_nl_kb: nqnl > mxdlqp");
    if (delqnl[k] <= 0 && nqnl[k] > 1) return fail(kBadArg, "proj_nl_kb: delqnl not positive");
    nq_max = nqnl[k] > nq_max ? nqnl[k] : nq_max;
  }
  double vcell = 0;
  if (!adot_to_bvec(adot, t->g.bvec, &vcell)) return fail(kBadArg, "proj_nl_kb: metric adot not positive definite");
  for (int j = 0; j < 3; ++j) t->g.rk[j] = rkpt[j];
  t->g.fac = 1.0 / sqrt(vcell);
  t->g.nq_max = nq_max;
  for (int r = 0; r < 3; ++r)      // bdot = bvec^T bvec (the reciprocal metric)
    for (int cc = 0; cc < 3; ++cc)
      t->bdot[r + 3 * cc] = t->g.bvec[3 * r] * t->g.bvec[3 * cc] + t->g.bvec[3 * r + 1] * t->g.bvec[3 * cc + 1] +
                            t->g.bvec[3 * r + 2] * t->g.bvec[3 * cc + 2];
  // vkb(-2:nq, l, 0, k) of every type and l, rows of nq_max + 3
  const int row = nq_max + 3;
  t->tab.assign((size_t)(ntype > 0 ? ntype : 1) * (kLmax + 1) * row, 0.0);
  const size_t ldq = (size_t)mxdlqp + 3;
  for (int k = 0; k < ntype; ++k)
    for (int l = 0; l <= kLmax; ++l) {
      const double* src = vkb + ldq * (l + (kLmax + 1) * (1 + 3 * (size_t)k));
      for (int n = 0; n < nqnl[k] + 3 && n < (int)ldq; ++n) t->tab[((size_t)k * (kLmax + 1) + l) * row + n] = src[n];
    }
  return kOk;
}

}  // namespace

int ctx_proj_nl_kb(cpw_b200_ctx* c, const double* rkpt, int ntype, const int* natom, const double* rat, int mxdatm,
                   const double* adot, const int* nqnl, const double* delqnl, const double* vkb, int mxdlqp,
                   const int* nkb, int nanl, double* xnlkb_out, void* anlga_out, long long ld_out) {
  if (!c->have_basis) return fail(kNotReady, "proj_nl_kb: call set_basis first");
  const long long m = c->mtxd;
  ProjTables T;
  if (int s = proj_tables(rkpt, ntype, natom, rat, mxdatm, adot, nqnl, delqnl, vkb, mxdlqp, nkb, nanl, &T)) return s;
  std::vector<ProjEntry>& ent = T.ent;
  std::vector<double>& xnl = T.xnl;
  std::vector<double>& tau = T.tau;
  std::vector<double>& tab = T.tab;
  ProjGeom& g = T.g;
  c->nanl = nanl;
  c->tc_ready = false;
  c->oz_nl_ready = false;
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

int ctx_proj_nl_kb_der(cpw_b200_ctx* c, int nder, const double* rkpt, int ntype, const int* natom, const double* rat,
                       int mxdatm, const double* adot, const int* nqnl, const double* delqnl, const double* vkb,
                       int mxdlqp, const int* nkb, int nanl, double* xnlkb_out, void* anlga, long long ld,
                       long long mxdanl, void* danlgadrk, void* d2anlgadrk2) {
  if (!c->have_basis) return fail(kNotReady, "proj_nl_kb_der: call set_basis first");
  if (nder < 0 || nder > 2) return fail(kBadArg, "proj_nl_kb_der_c16: cannot calculate derivatives of that order");
  const long long m = c->mtxd;
  ProjTables T;
  if (int s = proj_tables(rkpt, ntype, natom, rat, mxdatm, adot, nqnl, delqnl, vkb, mxdlqp, nkb, nanl, &T)) return s;
  if (nanl > mxdanl) return fail(kBadArg, "proj_nl_kb_der: increase mxdanl");
  if (xnlkb_out)
    for (int j = 0; j < nanl; ++j) xnlkb_out[j] = T.xnl[j];
  if (nanl == 0 || m == 0) return kOk;
  if (ld < m) return fail(kBadArg, "proj_nl_kb_der: leading dimension smaller than mtxd");
  if (!anlga || (nder > 0 && !danlgadrk) || (nder > 1 && !d2anlgadrk2))
    return fail(kBadArg, "proj_nl_kb_der: null output array for the requested derivatives");
  // the solid harmonics' monomials (ylm_rc.f90:82-106), l*l + l + m
  Mono mono[16][3] = {};
  int nmono[16] = {};
  auto put = [&](int l, int mm, double cf, int a, int b, int cz) {
    const int idx = l * l + l + mm;
    mono[idx][nmono[idx]++] = Mono{cf, {a, b, cz}};
  };
  const double s3 = sqrt(3.0), s58 = sqrt(5.0 / 8.0), s15 = sqrt(15.0), s38 = sqrt(3.0 / 8.0), s154 = sqrt(15.0 / 4.0),
               s34 = sqrt(0.75);
  put(0, 0, 1.0, 0, 0, 0);
  put(1, -1, 1.0, 0, 1, 0);
  put(1, 0, 1.0, 0, 0, 1);
  put(1, 1, 1.0, 1, 0, 0);
  put(2, -2, s3, 1, 1, 0);
  put(2, -1, s3, 0, 1, 1);
  put(2, 0, 1.0, 0, 0, 2), put(2, 0, -0.5, 2, 0, 0), put(2, 0, -0.5, 0, 2, 0);
  put(2, 1, s3, 1, 0, 1);
  put(2, 2, s34, 2, 0, 0), put(2, 2, -s34, 0, 2, 0);
  put(3, -3, 3 * s58, 2, 1, 0), put(3, -3, -s58, 0, 3, 0);
  put(3, -2, s15, 1, 1, 1);
  put(3, -1, 4 * s38, 0, 1, 2), put(3, -1, -s38, 2, 1, 0), put(3, -1, -s38, 0, 3, 0);
  put(3, 0, 1.0, 0, 0, 3), put(3, 0, -1.5, 2, 0, 1), put(3, 0, -1.5, 0, 2, 1);
  put(3, 1, 4 * s38, 1, 0, 2), put(3, 1, -s38, 3, 0, 0), put(3, 1, -s38, 1, 2, 0);
  put(3, 2, s154, 2, 0, 1), put(3, 2, -s154, 0, 2, 1);
  put(3, 3, -3 * s58, 1, 2, 0), put(3, 3, s58, 3, 0, 0);
  cudaError_t e;
  if ((e = cudaMemcpyToSymbolAsync(c_mono, mono, sizeof mono, 0, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess ||
      (e = cudaMemcpyToSymbolAsync(c_nmono, nmono, sizeof nmono, 0, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess)
    return cuda_fail(e, "proj_nl_kb_der tables");
  int s;
  DevBuf d_ent, d_tau, d_tab, d_nq, d_dq, d_bdot;
  if ((s = upload(d_ent, T.ent.data(), T.ent.size() * sizeof(ProjEntry))) ||
      (s = upload(d_tau, T.tau.data(), T.tau.size() * sizeof(double))) ||
      (s = upload(d_tab, T.tab.data(), T.tab.size() * sizeof(double))) ||
      (s = upload(d_nq, nqnl, (size_t)ntype * sizeof(int))) ||
      (s = upload(d_dq, delqnl, (size_t)ntype * sizeof(double))) || (s = upload(d_bdot, T.bdot, sizeof T.bdot)))
    return s;
  const dim3 grid((unsigned)((m + 127) / 128), (unsigned)((nanl + kProjPerThread - 1) / kProjPerThread));
  k_proj_nl_kb_der<<<grid, 128, 0, c->stream>>>((int)m, nanl, nder, (const int*)c->kgvb.p, T.g,
                                                (const double*)d_bdot.p, (const ProjEntry*)d_ent.p,
                                                (const double*)d_tau.p, (const double*)d_tab.p, (const int*)d_nq.p,
                                                (const double*)d_dq.p, (C2<double>*)anlga, (C2<double>*)danlgadrk,
                                                (C2<double>*)d2anlgadrk2, ld, mxdanl);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "proj_nl_kb_der kernel");
  // the small tables are freed at return: finish with them first
  e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? kOk : cuda_fail(e, "proj_nl_kb_der");
}

}  // namespace cpwb
