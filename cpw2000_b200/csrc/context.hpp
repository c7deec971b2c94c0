// Per-k-point device state shared by the H|psi> and eigensolver entry points.
#pragma once
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "hkpsi_local.cuh"

struct cpw_b200_ctx;

namespace cpwb {

// Status codes of the C ABI (also in include/cpw_b200.h).
enum Status : int {
  kOk = 0,
  kBadArg = 1,        // invalid dimension / argument (the reference would stop)
  kWrap = 2,          // basis wraps around the FFT box (hk_psi_c16.f90:161-172)
  kUnsupported = 3,   // FFT length not factorable into supported radices, or too large
  kNotReady = 4,      // basis / potential not set
  kNotConverged = 5,  // eigensolver: see ifail
  kCuda = -1,         // CUDA runtime error
  kCublas = -2,       // cuBLAS error
  kCusolver = -3,     // cuSOLVER error
  kTimeout = -4,      // a bounded device wait gave up
};

// Stage timers: CUDA events recorded around every kernel of a stage while
// enabled; read back (with one synchronisation) by timing_end.
enum Stage : int { kStInvXY = 0, kStZVloc = 1, kStFwdXY = 2, kStNlProj = 3, kStNlExpand = 4, kStEig = 5, kNumStages = 8 };
struct StageTimer {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  struct Rec { int stage; cudaEvent_t a, b; };
  std::vector<Rec> recs;
  cudaEvent_t take();                       // nullptr when the pool is exhausted
  void mark(int stage, cudaEvent_t a, cudaEvent_t b) { if (a && b) recs.push_back({stage, a, b}); }
  ~StageTimer();
};

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int ensure(size_t need);
  void release();
  ~DevBuf() { release(); }
};

int ditsp_device(cpw_b200_ctx* c, int ipr, int* ifail, int icmax, int iguess, double epspsi, int* neig_io, int mtxds,
                 void* psi, long long ldp, void* hpsi, const double* hamsm, int mxdsml, const double* hdiag,
                 int mxdbnd, double* ei, long long* ihkpsum, cudaStream_t st, double* itlog = nullptr,
                 int itlog_rows = 0);
// the local plan of a box for sphere half-widths kd (checks the radix split and the wraparound)
int plan_for_box(cpw_b200_ctx* c, const int kd[3], const int* kmscr, LocalPlan* out);
// the kept-plane lists of a basis (g: 3 x mtxd integer G vectors) on plan p
void plane_lists(const LocalPlan& p, int mtxd, const int* g, std::vector<int>& start, std::vector<int>& idx,
                 std::vector<int>& pos);
int upload(DevBuf& b, const void* h, size_t bytes);
// n = r1*r2 with both factors supported radices (false if none); W_n^k = e^{-2 pi i k/n}
bool factor(int n, FftDim& d);
void twiddles(int n, std::vector<double>& out);
int ctx_pot_local(cpw_b200_ctx* c, int n1, int n2, int n3, int id, int ng, const int* kgv, const double* veff,
                  const double* phase, const double* conj, const int* inds, double* vscr, double* vmax,
                  double* vmin, double* cmax, bool install);
// per-call scratch of the tensor-core projector products and their sticky error flag
struct TcScratch {
  DevBuf b1, part, b2, err;
  unsigned long long wait_ns = 2000000000ull;   // hand-off wait limit of the tensor-core GEMMs
};
int tc_wait_selftest(cpw_b200_ctx* c, unsigned long long limit_ns, cudaStream_t st);
// an A operand of the int8 tensor-core (Ozaki) complex GEMM split into int8 tiles with its row
// scales (oz.cu); kept and reused for products with the same A
struct OzOperand {
  DevBuf tiles, e;
  int M = 0, K = 0, s = 0, nkb = 0, tiles_m = 0;
  bool conj = false, ready = false;
};
// work space of the int8 tensor-core GEMM and its sticky error flag
struct OzScratch {
  OzOperand aop;
  DevBuf b, eb, part, err;
  bool err_init = false;
};
int oz_prepare_a(OzOperand& op, bool conjA, int M, int K, const void* A, long long lda, int slices, cudaStream_t st);
// triangular structure an int8 product may exploit (oz.cu)
enum OzTri : int {
  kOzFull = 0,
  kOzLowerOut = 1,   // only the lower triangle of C (M = N) is wanted: tiles strictly above the diagonal are written as zeros
  kOzUpperB = 2,     // B (K = N) is upper triangular: column block j reads only the first K rows it can reach
};
int oz_gemm_prepared(OzScratch& w, const OzOperand& op, int N, const void* B, long long ldb, double alpha,
                     bool accumulate, void* C, long long ldc, unsigned long long wait_ns, cudaStream_t st,
                     int tri = kOzFull);
// C = alpha op(A) B (+ C) with op(A) = A or A^H, complex128 column-major, FP64-accurate on the
// int8 tensor cores with `slices` 7-bit slices per operand (oz.cu)
int oz_zgemm(OzScratch& w, bool conjA, int M, int N, int K, const void* A, long long lda, const void* B, long long ldb,
             double alpha, bool accumulate, void* C, long long ldc, int slices, unsigned long long wait_ns,
             cudaStream_t st, int tri = kOzFull);
int oz_read_error(OzScratch& w);
int tc_error_flag(TcScratch& t);
int tc_read_error(TcScratch& t);
int tc_prepare_projectors(cpw_b200_ctx* c);
int tc_prepare_operands(int m, int na, const void* anl, const void* anld, DevBuf& a1buf, DevBuf& a2buf,
                        long long* nkb1_out, long long* nkb2_out, cudaStream_t st);
int tc_nl_apply_ops(TcScratch& t, int m, int na, long long nkb1, long long nkb2, const float* a1, const float* a2,
                    int nb, const void* psi, long long ldpsi, void* hpsi, long long ldh, cudaStream_t st,
                    cudaEvent_t t0, cudaEvent_t t1, cudaEvent_t t2, int splits = 0);
int tc_nl_apply(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, void* hpsi, long long ldh, cudaStream_t st,
                cudaEvent_t t0, cudaEvent_t t1, cudaEvent_t t2);
int tc_check_error(cpw_b200_ctx* c);
int tc_zgemm_nn(cpw_b200_ctx* c, int m, int n, int kk, const void* a, long long lda, const void* b, long long ldb,
                void* cm, long long ldc, cudaStream_t st, bool accumulate = false);
int density_device(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, const double* occ, void* rho,
                   cudaStream_t st);
int structure_grad_device(cpw_b200_ctx* c, const void* g, int natom, const int* atom_type, const double* tau,
                          int ntype, const void* vgt, double* dedtau, cudaStream_t st);
int stress_inputs_device(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, const double* occ, double* w,
                         void* y, cudaStream_t st);
int nl_grad_device(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, const double* occ,
                   const int* proj_atom, int natom, double* dedtau, cudaStream_t st);
}  // namespace cpwb

struct cpw_b200_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  // drop-in host path: copy streams and per-chunk events of the pipelined transfer
  cudaStream_t s_in = nullptr, s_out = nullptr;
  std::vector<cudaEvent_t> ev_pipe;
  // drop-in host path, FP64 projectors: projections of the band chunks on their own stream
  // and cuBLAS handle (own workspace), so that they leave the chunk's critical path
  cudaStream_t s_nl = nullptr;
  cublasHandle_t blas_nl = nullptr;
  std::vector<cudaEvent_t> ev_nl;
  cudaEvent_t ov_ev[2] = {nullptr, nullptr};   // device H|psi>: projection on s_nl beside the local kernels
  cublasHandle_t blas = nullptr;
  int precision = 0;            // 0: FP64; 1: FP32 local + FP64 projector GEMMs; 2: 1 with split-TF32 tensor-core projectors
  size_t slab_budget = 512ull << 20;

  // basis of the current k-point
  bool have_basis = false;
  int mtxd = 0;
  int ident = 0;                // leading dimension id of the reference box (kmscr(7))
  cpwb::LocalPlan plan{};
  cpwb::DevBuf plane_start, pw_idx, pw_pos, ekpg, kgvb;   // kgvb: (3, mtxd) G of the basis
  cpwb::DevBuf tw64[3], tw32[3];

  // local potential on the box, [z][y][x] scaled by 1/N
  bool have_pot = false;
  int pot_n[3] = {0, 0, 0};
  cpwb::DevBuf v64, v32;

  // KB projectors (column-major mtxd x nanl) pre-multiplied by xnlkb in anld
  int nanl = 0;
  cpwb::DevBuf anl, anld, proj;
  std::vector<double> xnl_h;    // host copy of xnlkb
  // mixed precision: split-TF32 operands of the tensor-core projector GEMMs
  cpwb::DevBuf tc_a1, tc_a2, tc_ga, tc_gb;
  cpwb::TcScratch tcs;
  cpwb::OzScratch ozs;          // int8 tensor-core GEMMs of the eigensolver's basis products
  // projector products on the int8 tensor cores: nl_slices > 0 slices per operand (0: the
  // precision form's default), X (for X^H psi) and X D (for hpsi += X D P) split once per set
  int nl_slices = 0;
  cpwb::OzOperand oz_x, oz_xd;
  cpwb::OzOperand oz_gs[3];     // eigensolver: converged block of a Gram-Schmidt call, split once
  bool oz_nl_ready = false;
  long long tc_k1p = 0, tc_k2p = 0;     // K blocks (32 reals) of the projection and expansion operands
  bool tc_ready = false;

  // two-component spinors (hk_psi_spin_c16): nsp potential combinations scaled by 1/N
  // ([V] or [V1+V2, V1-V2] or [V1+V2, V1-V2, V3, -V4]), the spinor projectors (2 mtxd rows)
  // and the component views of the basis (doubled plane-wave indices and kinetic diagonal)
  int nsp = 0;
  cpwb::DevBuf sp_v64[4], sp_v32[4];
  int nanl_sp = 0;
  cpwb::DevBuf anl_sp, anld_sp, sp_idx2, sp_ek2;

  // poll limit of the eigensolver's cooperative grid barrier (bounded device wait)
  long long grid_polls = 1LL << 24;
  // eigensolver device buffers and cuSOLVER handle, kept between calls (ditsp.cu)
  cpwb::DevBuf ditsp_pool[24];
  void* ditsp_sol = nullptr;

  cpwb::StageTimer timer;

  // slab for the band chunk and staging for host-array entry points
  cpwb::DevBuf slab, h_in, h_out;

  // host shadows used by the drop-in to decide what to re-upload (the projectors are compared by
  // content: the reference recomputes anlga without any obligation to raise lnewanl)
  std::vector<int> sh_isort, sh_kgv, sh_kmscr;
  std::vector<double> sh_ekpg, sh_vscr, sh_anl, sh_xnl;
  int sh_mtxd = -1, sh_nanl = -1;
};

namespace cpwb {
int ctx_set_basis(cpw_b200_ctx* c, int mtxd, const int* isort, const int* kgv, int ng, const double* ekpg,
                  const int* kmscr);
int ctx_set_potential(cpw_b200_ctx* c, const double* vscr, long long nscr);
int ctx_set_projectors(cpw_b200_ctx* c, int nanl, const double* anlga, int ld, const double* xnlkb, bool on_device);
void ditsp_release(cpw_b200_ctx* c);
int ctx_set_potential_spin(cpw_b200_ctx* c, const double* vscr_sp, long long mxdscr, int nsp);
int ctx_set_projectors_spin(cpw_b200_ctx* c, int nanl, const double* anlsp, long long ld, const double* xnlkb);
int ctx_hkpsi_kin_device(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, void* hpsi, long long ldh,
                         bool ladd, int nspin, cudaStream_t st);
int ctx_hkpsi_loc_general(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, void* hpsi, long long ldh,
                          bool ladd, int nspin, cudaStream_t st);
int ctx_hkpsi_spin_device(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, void* hpsi, long long ldh,
                          cudaStream_t st);
int ctx_proj_nl_kb(cpw_b200_ctx* c, const double* rkpt, int ntype, const int* natom, const double* rat, int mxdatm,
                   const double* adot, const int* nqnl, const double* delqnl, const double* vkb, int mxdlqp,
                   const int* nkb, int nanl, double* xnlkb_out, void* anlga_out, long long ld_out);
int ctx_proj_nl_kb_der(cpw_b200_ctx* c, int nder, const double* rkpt, int ntype, const int* natom, const double* rat,
                       int mxdatm, const double* adot, const int* nqnl, const double* delqnl, const double* vkb,
                       int mxdlqp, const int* nkb, int nanl, double* xnlkb_out, void* anlga, long long ld,
                       long long mxdanl, void* danlgadrk, void* d2anlgadrk2);
int hamilt_kb_device(cpw_b200_ctx* c, int mtxd, const double* hdiag, const int* isort, const double* qmod, int ng,
                     const int* kgv, const double* phase, const double* conj, const int* inds, const int* kmax,
                     const int* indv, const double* ek, const double* sfact, const double* veff, const int* nqnl,
                     const double* delqnl, const double* vkb, const int* nkb, int ntype, const double* adot,
                     void* hamk, long long ldh, int mxdtyp, int mxdgve, int mxdnst, int mxdcub, int mxdlqp,
                     int mxddim);
int ctx_hkpsi_device(cpw_b200_ctx* c, int nb, const void* psi, long long ldpsi, void* hpsi, long long ldh,
                     cudaStream_t st, bool with_kinetic, bool with_nl);
}  // namespace cpwb
