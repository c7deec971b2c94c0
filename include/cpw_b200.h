/*
 * cpw_b200.h -- C ABI of the B200-native H|psi> operator and block eigensolver
 * for cpw2000 (plain pointers and sizes; no torch or CUDA types in signatures).
 *
 * Two layers:
 *
 *  1. Drop-ins with the reference's Fortran argument lists, every argument by
 *     reference as gfortran passes it (LOGICAL is a 4-byte int, 0 = .FALSE.),
 *     complex(8) arrays as interleaved (re, im) doubles, column-major with the
 *     reference's leading dimensions, 1-based isort into kgv(3, mxdgve):
 *       cpw_b200_hk_psi_c16  / hk_psi_c16_    replaces Src/hk_psi/reference/hk_psi_c16.f90:28-32
 *       cpw_b200_hk_psi_nl_c16 / hk_psi_nl_c16_ replaces Src/cpw_lib/hk_psi_nl_c16.f90:23-24
 *       cpw_b200_hk_psi_spin_c16 / hk_psi_spin_c16_ replaces Src/hk_psi/reference/hk_psi_spin_c16.f90:1-316
 *       cpw_b200_ditsp_c16   / ditsp_c16_     replaces Src/ditsp/ditsp_c16.f90:20-27
 *     The cpw_b200_* forms return a status (0 = success) and never stop the
 *     program; the trailing-underscore forms are link-time substitutes for the
 *     Fortran symbols and, like the reference, print the message and stop the
 *     program on an error (exit status 1).
 *
 *  2. A context API for callers that keep data on the device: the per-k-point
 *     inputs are set once (basis, potential, projectors) and H|psi> is applied
 *     to device-resident column-major complex128 blocks on a caller stream.
 *
 * Threading: a context is not re-entrant; one context per host thread. The
 * drop-ins use one process-wide context on the current CUDA device and are
 * synchronous (results are in the host arrays on return), as the reference's
 * routines are.
 */
#ifndef CPW_B200_H
#define CPW_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define CPW_B200_OK 0
#define CPW_B200_BAD_ARG 1       /* invalid dimension or argument (the reference stops) */
#define CPW_B200_WRAP 2          /* basis wraps around the FFT box (hk_psi_c16.f90:161-172) */
#define CPW_B200_UNSUPPORTED 3   /* FFT length not a product of two radices <= 16, or too large */
#define CPW_B200_NOT_READY 4     /* context: basis / potential not set */
#define CPW_B200_NOT_CONVERGED 5 /* eigensolver did not reach epspsi; ifail holds the digits */
#define CPW_B200_CUDA_ERROR (-1)
#define CPW_B200_CUBLAS_ERROR (-2)
#define CPW_B200_CUSOLVER_ERROR (-3)
#define CPW_B200_TIMEOUT (-4)

/* ---- precision modes ---- */
#define CPW_B200_FP64 0  /* plain FP64 everywhere (the drop-in default) */
#define CPW_B200_MIXED 1 /* FP32 FFT/V_loc, FP64 projector GEMMs, FP64 subspace steps */
/* MIXED with the projector products as split-TF32 (hi.hi + hi.lo + lo.hi) tcgen05 GEMMs with FP32
 * accumulation in tensor memory: ~1e-6 relative error in the projector term; opt-in, set before the
 * projectors (they are prepared in the split layouts at set_projectors). */
#define CPW_B200_MIXED_TC 2

typedef struct cpw_b200_ctx cpw_b200_ctx;

/* Message of the last failing call on this host thread ("" if none). */
const char* cpw_b200_last_error(void);
/* Library ABI version (major*10000 + minor*100 + patch). */
int cpw_b200_version(void);

/* ---- context API ---- */
int cpw_b200_create(cpw_b200_ctx** ctx, int device);
int cpw_b200_destroy(cpw_b200_ctx* ctx);
/* The context's own CUDA stream (cudaStream_t as void*). */
void* cpw_b200_stream(cpw_b200_ctx* ctx);
/* Waits for all work on the device; returns CPW_B200_TIMEOUT if a bounded
 * device-side wait of an earlier kernel gave up (its outputs are then invalid). */
int cpw_b200_synchronize(cpw_b200_ctx* ctx);
int cpw_b200_set_precision(cpw_b200_ctx* ctx, int mode);
/* Device bytes the FFT slab of one band chunk may use (default 512 MiB). */
int cpw_b200_set_slab_budget(cpw_b200_ctx* ctx, long long bytes);

/* Bounded device waits (failure detection). Every wait of this library's kernels
 * on another party gives up after a limit, records the failure and lets the
 * kernel return; the host then reports CPW_B200_TIMEOUT (from
 * cpw_b200_synchronize for the tensor-core GEMMs, from the eigensolver call for
 * its cooperative Gram-Schmidt kernel) and the context stays usable.
 * set_wait_limits: the time limit of the tensor-core GEMMs' hand-off mbarrier
 *   waits (default 2 s) and the poll limit of the Gram-Schmidt grid barrier
 *   (default 2^24, ~1 s); a negative value restores the default. The waits for
 *   copies and tensor-core work already issued, before a kernel exits, keep
 *   their 2 s limit.
 * wait_selftest: no counterpart in the reference. Launches one kernel that
 *   waits, with the GEMMs' bounded wait, on an mbarrier nothing arrives at, for
 *   at most limit_ns (<= 2 s); the next cpw_b200_synchronize returns
 *   CPW_B200_TIMEOUT. A test of the failure path that faults no GPU. */
int cpw_b200_set_wait_limits(cpw_b200_ctx* ctx, long long mbarrier_ns, long long grid_polls);
int cpw_b200_wait_selftest(cpw_b200_ctx* ctx, long long limit_ns, void* stream);

/* Projector products P = X^H psi and hpsi += X D P (hk_psi_nl_c16.f90:82-96) of
 * the context's H|psi> on the int8 tensor cores with `slices` 7-bit slices per
 * operand (1..8; the split of X and X D is kept until the projectors change),
 * in any precision form; 0 restores the form's default (cuBLAS FP64 ZGEMMs in
 * FP64 and MIXED, split-TF32 tensor-core GEMMs in MIXED_TC). 7 slices give
 * FP64-level products (~2^-48 of the row maxima); 4 give ~2^-27, without the
 * bias of FP32 accumulation (the integer sums are exact). */
int cpw_b200_set_projector_slices(cpw_b200_ctx* ctx, int slices);

/* FP64-accurate complex GEMM on the int8 tensor cores (no counterpart in the
 * reference, whose ZGEMMs are BLAS calls): C = alpha op(A) B (+ C when
 * accumulate != 0), op(A) = A (transa 'N', A m x k) or A^H (transa 'C', A k x
 * m), B k x n; device complex128 column-major arrays, alpha real. Each operand
 * row is split into `slices` (1..8) 7-bit integer slices under a power-of-two
 * row scale (the Ozaki scheme); with 7 slices an entry's error is below ~2^-48
 * k max|a| max|b|. Asynchronous on `stream` (NULL = the context stream); a
 * bounded wait that gave up is reported by cpw_b200_synchronize. */
int cpw_b200_zgemm_i8(cpw_b200_ctx* ctx, int transa, int m, int n, int k, const void* a, long long lda,
                      const void* b, long long ldb, double alpha, int accumulate, void* c, long long ldc, int slices,
                      void* stream);

/* cpw_b200_zgemm_i8 with a triangular structure it may exploit: tri 0 none;
 * 1 only the lower triangle of C is wanted (m = n; output tiles strictly above
 * the diagonal are written as zeros, the others in full); 2 B is upper
 * triangular (k = n; the products with its zero part are skipped, so entries
 * of B below the diagonal are treated as zero). */
int cpw_b200_zgemm_i8_tri(cpw_b200_ctx* ctx, int transa, int m, int n, int k, const void* a, long long lda,
                          const void* b, long long ldb, double alpha, int accumulate, void* c, long long ldc, int slices,
                          int tri, void* stream);

/* Stage timers (CUDA events around each kernel of a stage, on the stream the
 * kernel runs on). timing_end synchronises and writes per-stage totals in ms
 * and launch counts for stages 0..nstage-1: 0 scatter+inverse xy, 1 inverse z +
 * V_loc + forward z, 2 forward xy + gather, 3 projection X^H psi, 4 expansion
 * hpsi += X D P, 5 eigensolver subspace work. */
int cpw_b200_timing_begin(cpw_b200_ctx* ctx);
int cpw_b200_timing_end(cpw_b200_ctx* ctx, double* ms, long long* launches, int nstage);

/* Basis of one k-point: isort(mtxd) 1-based into kgv(3, ng), ekpg(mtxd) in
 * Hartree, kmscr(7) as the reference (kmscr(4:6) = n1,n2,n3, kmscr(7) = id).
 * Host arrays. (Inputs of hk_psi_c16.f90:28-32 that depend only on k.) */
int cpw_b200_set_kpoint(cpw_b200_ctx* ctx, int mtxd, const int* isort, const int* kgv, int ng,
                        const double* ekpg, const int* kmscr);
/* Screened potential vscr(id*n2*n3) on the FFT box, host array. */
int cpw_b200_set_potential(cpw_b200_ctx* ctx, const double* vscr, long long mxdscr);
/* KB projectors anlga(mxddim, nanl) complex(8) and xnlkb(nanl), host arrays
 * (the outputs of Src/omp/proj_nl_kb_c16.f90). */
int cpw_b200_set_projectors(cpw_b200_ctx* ctx, int nanl, const double* anlga, int mxddim, const double* xnlkb);
/* Same with device pointers (anlga complex128, leading dimension ld). */
int cpw_b200_set_projectors_device(cpw_b200_ctx* ctx, int nanl, const void* anlga, int ld, const void* xnlkb);
/* KB projectors of the context's k-point computed on the device: replaces
 * Src/omp/proj_nl_kb_c16.f90:23-275 (same arguments: rkpt(3) lattice
 * coordinates of k, natom(ntype), rat(3, mxdatm, ntype) lattice coordinates,
 * adot(3,3) metric, nqnl(ntype), delqnl(ntype), vkb(-2:mxdlqp, 0:3, -1:1, ntype)
 * and nkb(0:3, -1:1, ntype) as in the reference; host arrays) followed by
 * cpw_b200_set_projectors, without the host loop and the mtxd x nanl upload.
 * The basis is the one given to cpw_b200_set_kpoint. nanl must equal
 * sum_type natom * sum_{l: nkb(l,0,type) != 0} (2l+1) (the reference's check).
 * xnlkb (host, nanl) may be NULL; anlga (device, complex128, leading dimension
 * ldanl >= mtxd) may be NULL, else it receives a copy of the projectors.
 * Synchronous. */
int cpw_b200_proj_nl_kb_device(cpw_b200_ctx* ctx, const double* rkpt, int ntype, const int* natom,
                               const double* rat, int mxdatm, const double* adot, const int* nqnl,
                               const double* delqnl, const double* vkb, int mxdlqp, const int* nkb, int nanl,
                               double* xnlkb, void* anlga, long long ldanl);

/* KB projectors and their derivatives with respect to the k-point's lattice
 * coordinates, on the device: replaces Src/omp/proj_nl_kb_der_c16.f90:25-417
 * (same inputs as cpw_b200_proj_nl_kb_device, nder = 0, 1 or 2). Outputs are
 * device complex128 arrays in the reference layouts: anlga(ld, mxdanl),
 * danlgadrk(ld, mxdanl, 3) for nder >= 1 and d2anlgadrk2(ld, mxdanl, 3, 3) for
 * nder = 2 (ld >= mtxd, mxdanl >= nanl; the arrays a lower nder does not need
 * may be NULL); xnlkb (host, may be NULL). The basis is the context's k-point;
 * the context's own projectors are not changed. Synchronous. */
int cpw_b200_proj_nl_kb_der_device(cpw_b200_ctx* ctx, int nder, const double* rkpt, int ntype, const int* natom,
                                   const double* rat, int mxdatm, const double* adot, const int* nqnl,
                                   const double* delqnl, const double* vkb, int mxdlqp, const int* nkb, int nanl,
                                   double* xnlkb, void* anlga, long long ld, long long mxdanl, void* danlgadrk,
                                   void* d2anlgadrk2);

/* The small dense Hamiltonian of the start basis on the device: replaces
 * Src/ALFA/hamilt_kb.f90:1-234 (same arguments and layouts, host arrays:
 * hdiag/isort/qmod (mtxd), kgv(3, mxdgve), phase(mxdgve) complex(8),
 * conj(mxdgve), inds(mxdgve) 1-based stars, kmax(3), indv(mxdcub), ek(mxdnst),
 * sfact(mxdtyp, mxdnst) complex(8), veff(mxdnst) complex(8), nqnl/delqnl
 * (mxdtyp), vkb(-2:mxdlqp, 0:3, -1:1, mxdtyp), nkb(0:3, -1:1, mxdtyp), adot).
 * hamk is a device complex128 array (ldh >= mtxd) that receives the full
 * Hermitian matrix (the reference's output, both triangles), ready to be
 * copied to the hamsm argument of the eigensolver. Synchronous. */
int cpw_b200_hamilt_kb_device(cpw_b200_ctx* ctx, int mtxd, const double* hdiag, const int* isort, const double* qmod,
                              int ng, const int* kgv, const double* phase, const double* conj, const int* inds,
                              const int* kmax, const int* indv, const double* ek, const double* sfact,
                              const double* veff, const int* nqnl, const double* delqnl, const double* vkb,
                              const int* nkb, int ntype, const double* adot, void* hamk, long long ldh, int mxdtyp,
                              int mxdgve, int mxdnst, int mxdcub, int mxdlqp, int mxddim);

/* Screened local potential on the FFT mesh, computed on the device: replaces
 * Src/cpw_lib/pot_local.f90:1-190 (same arguments and array layouts, host
 * arrays: veff(mxdnst) complex(8) per star, kmscr(7) in/out (kmscr(4:7) set to
 * n1, n2, n3, id = n1 + idshift), kgv(3, mxdgve), phase(mxdgve) complex(8),
 * conj(mxdgve), inds(mxdgve) 1-based stars; ipr dropped). vscr(id*n2*n3)
 * (host, may be NULL) receives the real potential; vmax/vmin its extrema and
 * cmax the largest imaginary part (each may be NULL). Fails like the
 * reference's stop when cmax > 1e-6. install != 0 also makes it the context's
 * potential without a host round trip (the context's k-point box must be the
 * same mesh). G vectors outside the mesh wrap modulo the mesh. Synchronous. */
int cpw_b200_pot_local(cpw_b200_ctx* ctx, double* vscr, double* vmax, double* vmin, double* cmax,
                       const double* veff, int* kmscr, int idshift, int ng, const int* kgv,
                       const double* phase, const double* conj, int ns, const int* inds, int mxdscr,
                       int mxdgve, int mxdnst, int install);

/* The split operators on device blocks (columns of nspin*mtxd rows, spinor rows
 * interleaved up, down when nspin = 2), on `stream` (NULL = the context stream);
 * ladd != 0 adds to hpsi, else hpsi is overwritten:
 *   cpw_b200_hk_psi_kin_device      replaces Src/omp/hk_psi_kin_c16.f90:22-131
 *                                   (hpsi (+)= ekpg psi);
 *   cpw_b200_hk_psi_loc_c16_device  replaces Src/omp/hk_psi_loc_c16.f90:23-362
 *                                   (local potential alone: the context's vscr when
 *                                   nspin = 1, its spin potential when nspin = 2). */
int cpw_b200_hk_psi_kin_device(cpw_b200_ctx* ctx, int neig, const void* psi, long long ldpsi, void* hpsi,
                               long long ldh, int ladd, int nspin, void* stream);
int cpw_b200_hk_psi_loc_c16_device(cpw_b200_ctx* ctx, int neig, const void* psi, long long ldpsi, void* hpsi,
                                   long long ldh, int ladd, int nspin, void* stream);

/* Spinor form on a context (the k-point from cpw_b200_set_kpoint): the nsp
 * potential columns vscr_sp(mxdscr, nsp) (host), the spinor projectors
 * anlsp(ld >= 2*mtxd, nanlsp) and xnlkbsp (host), then hpsi_sp = H psi_sp for
 * neig device-resident spinors (complex128, ld >= 2*mtxd, rows interleaved up,
 * down) on `stream` (NULL = the context stream). MIXED contexts run the local
 * part in FP32; the projector products are FP64 in every form. */
int cpw_b200_set_potential_spin(cpw_b200_ctx* ctx, const double* vscr_sp, long long mxdscr, int nsp);
int cpw_b200_set_projectors_spin(cpw_b200_ctx* ctx, int nanlsp, const double* anlsp, long long ld,
                                 const double* xnlkbsp);
int cpw_b200_hk_psi_spin_device(cpw_b200_ctx* ctx, int neig, const void* psi_sp, long long ldpsi, void* hpsi_sp,
                                long long ldh, void* stream);

/* hpsi = H psi for neig device-resident complex128 columns (ld >= mtxd), on
 * `stream` (cudaStream_t; NULL = the context stream). Asynchronous.
 * Same operator as hk_psi_c16.f90:176-231. */
int cpw_b200_hk_psi_device(cpw_b200_ctx* ctx, int neig, const void* psi, long long ldpsi, void* hpsi,
                           long long ldhpsi, void* stream);
/* Local part only, hpsi = V_loc psi (Src/omp/hk_psi_loc_c16.f90 with ladd = .false., nsp = 1). */
int cpw_b200_hk_psi_loc_device(cpw_b200_ctx* ctx, int neig, const void* psi, long long ldpsi, void* hpsi,
                               long long ldhpsi, void* stream);

/* ---- adjoint of H|psi> for fixed wavefunctions (Hellmann-Feynman) ----
 * For E = sum_n occ_n <psi_n|H|psi_n>:
 * density: rho(r) = sum_n occ_n |psi_n(r)|^2 on the box, device doubles laid out
 *   [z][y][x] (n1*n2*n3), psi_n(r) the unscaled backward transform, as the mesh
 *   density of Src/omp/charge_by_fft.f90:185-199; dE/dvscr(r) = rho(r)/(n1 n2 n3).
 * structure_grad: dE/dtau (host natom x 3, lattice coordinates) of sum_r g(r) V(r)
 *   for V(G) = sum_a e^{-2 pi i G.tau_a} v_t(G): g device [z][y][x] box doubles,
 *   vgt device ntype x n1 x n2 x n3 form factors v_t(G) in FFT order, tau host
 *   natom x 3, atom_type host 0-based (local term of Src/ALFA/for_str_local_force.f90).
 * nl_grad: dE/dtau of the Kleinman-Bylander energy for the context's projectors;
 *   proj_atom (host, nanl) is the 0-based atom of each projector column (the KB
 *   term of Src/ALFA/for_str_nl_kb.f90). Forces are minus these derivatives. */
int cpw_b200_density_device(cpw_b200_ctx* ctx, int neig, const void* psi, long long ldpsi, const double* occ,
                            void* rho, void* stream);
int cpw_b200_structure_grad_device(cpw_b200_ctx* ctx, const void* g, int natom, const int* atom_type,
                                   const double* tau, int ntype, const void* vgt, double* dedtau, void* stream);
int cpw_b200_nl_grad_device(cpw_b200_ctx* ctx, int neig, const void* psi, long long ldpsi, const double* occ,
                            const int* proj_atom, int natom, double* dedtau, void* stream);
/* stress_inputs: the blocks the strain derivative (stress) of sum_n occ_n <psi_n|H|psi_n> needs
 *   besides the density (Src/ALFA/for_str_kinetic_stress.f90, for_str_nl_kb.f90:364-376):
 *   w (device, mtxd doubles) = sum_n occ_n |psi(i,n)|^2 and y (device, mtxd x nanl
 *   complex128, ld mtxd) = psi diag(occ) P^H diag(xnlkb) with P = X^H psi for the context's
 *   projectors X; a change dX of the projectors changes the KB energy by 2 Re sum conj(dX) y. */
int cpw_b200_stress_inputs_device(cpw_b200_ctx* ctx, int neig, const void* psi, long long ldpsi, const double* occ,
                                  double* w, void* y, void* stream);

/* ---- drop-ins with the reference argument lists ---- */

/* Src/hk_psi/reference/hk_psi_c16.f90:28-32. lnewanl is only read, never
 * written (callers pass literals, e.g. Src/ALFA/berry_derivative.f90:229):
 * lnewanl != 0 makes the library re-upload anlga/xnlkb at once. The k-point
 * arrays, vscr and anlga/xnlkb are compared by content with the previous
 * call's (host shadows) and re-uploaded only when they changed; vscr and the
 * projectors are compared while the device already computes with the
 * previous call's copies, and a call whose inputs changed computes again. */
int cpw_b200_hk_psi_c16(const int* mtxd, const int* neig, const double* psi, double* hpsi, int* lnewanl,
                        const int* ng, const int* kgv, const double* ekpg, const int* isort, const double* vscr,
                        const int* kmscr, const double* anlga, const double* xnlkb, const int* nanl,
                        const int* mxddim, const int* mxdbnd, const int* mxdanl, const int* mxdgve,
                        const int* mxdscr);
void hk_psi_c16_(const int* mtxd, const int* neig, const double* psi, double* hpsi, int* lnewanl, const int* ng,
                 const int* kgv, const double* ekpg, const int* isort, const double* vscr, const int* kmscr,
                 const double* anlga, const double* xnlkb, const int* nanl, const int* mxddim, const int* mxdbnd,
                 const int* mxdanl, const int* mxdgve, const int* mxdscr);

/* Src/hk_psi/reference/hk_psi_spin_c16.f90: H|psi> of two-component spinors,
 * psi_sp/hpsi_sp complex(8)(2*mxddim, mxdbnd) with the up component of plane
 * wave i at row 2i-1 and the down component at row 2i (1-based), vscr_sp
 * real(8)(mxdscr, mxdnsp) with nsp = 1, 2 or 4 columns (1, sigma_z, sigma_x,
 * sigma_y), anlsp complex(8)(2*mxddim, mxdasp) spinor KB projectors. The
 * k-point arrays, vscr_sp, anlsp and xnlkbsp are compared by content with the
 * previous call's and re-uploaded when they changed; lnewanl (only read) != 0
 * forces the projector upload. */
int cpw_b200_hk_psi_spin_c16(const int* mtxd, const int* neig, const double* psi_sp, double* hpsi_sp,
                             int* lnewanl, const int* ng, const int* kgv, const double* ekpg, const int* isort,
                             const double* vscr_sp, const int* kmscr, const int* nsp, const double* anlsp,
                             const double* xnlkbsp, const int* nanlsp, const int* mxddim, const int* mxdbnd,
                             const int* mxdasp, const int* mxdgve, const int* mxdscr, const int* mxdnsp);
void hk_psi_spin_c16_(const int* mtxd, const int* neig, const double* psi_sp, double* hpsi_sp, int* lnewanl,
                      const int* ng, const int* kgv, const double* ekpg, const int* isort, const double* vscr_sp,
                      const int* kmscr, const int* nsp, const double* anlsp, const double* xnlkbsp,
                      const int* nanlsp, const int* mxddim, const int* mxdbnd, const int* mxdasp,
                      const int* mxdgve, const int* mxdscr, const int* mxdnsp);

/* Src/cpw_lib/hk_psi_nl_c16.f90:23-24: hpsi = [hpsi if ladd] + anlga xnlkb anlga^H psi. */
int cpw_b200_hk_psi_nl_c16(const int* mtxd, const int* neig, const double* psi, double* hpsi, const double* anlga,
                           const double* xnlkb, const int* nanl, const int* ladd, const int* mxddim,
                           const int* mxdbnd, const int* mxdanl);
void hk_psi_nl_c16_(const int* mtxd, const int* neig, const double* psi, double* hpsi, const double* anlga,
                    const double* xnlkb, const int* nanl, const int* ladd, const int* mxddim, const int* mxdbnd,
                    const int* mxdanl);

/* Block iterative eigensolver on device-resident psi/hpsi (complex128, ldpsi >= mtxd,
 * mxdbnd columns), restating Src/ditsp/ditsp_c16.f90 (start/loop/ritz, block
 * Gram-Schmidt, zheevd subspace eigensolve, Jacobi relaxation). hamsm is the host
 * complex(8) (mxdsml, mxdsml) leading block of H, hdiag the host diagonal, ei
 * host output (mxdbnd). *neig may grow to the degeneracy-closed count. Returns
 * CPW_B200_NOT_CONVERGED with *ifail = number of accurate digits when epspsi is
 * not reached in icmax outer iterations. ihkpsum (may be NULL) receives the
 * number of H|psi> band applications. Synchronous. itlog (may be NULL) is a host
 * array of itlog_rows rows of (4 + mxdbnd) doubles; after outer iteration ic
 * row ic-1 holds the elapsed seconds, xmax, nconv, the H|psi> products so far
 * and the current Ritz values (the time-to-eigenvalue trace). */
int cpw_b200_ditsp_device(cpw_b200_ctx* ctx, int ipr, int* ifail, int icmax, int iguess, double epspsi, int* neig,
                          int mtxds, void* psi, long long ldpsi, void* hpsi, double* ei, const double* hamsm,
                          int mxdsml, const double* hdiag, int mxdbnd, long long* ihkpsum, void* stream,
                          double* itlog, int itlog_rows);

/* Src/ditsp/ditsp_c16.f90:20-27 with host arrays (psi, hpsi complex(8) (mxddim, mxdbnd)).
 * lnewanl is only read, as in cpw_b200_hk_psi_c16 (the projectors are also compared by content). */
int cpw_b200_ditsp_c16(const int* ipr, int* ifail, const int* icmax, const int* iguess, const double* epspsi,
                       int* lnewanl, int* neig, const int* mtxd, const int* mtxds, double* psi, double* hpsi,
                       double* ei, const double* ekpg, const int* isort, const double* vscr, const int* kmscr,
                       const int* ng, const int* kgv, const double* anlga, const double* xnlkb, const int* nanl,
                       const double* hamsm, const double* hdiag, const int* mxddim, const int* mxdsml,
                       const int* mxdbnd, const int* mxdgve, const int* mxdscr, const int* mxdanl);
void ditsp_c16_(const int* ipr, int* ifail, const int* icmax, const int* iguess, const double* epspsi, int* lnewanl,
                int* neig, const int* mtxd, const int* mtxds, double* psi, double* hpsi, double* ei,
                const double* ekpg, const int* isort, const double* vscr, const int* kmscr, const int* ng,
                const int* kgv, const double* anlga, const double* xnlkb, const int* nanl, const double* hamsm,
                const double* hdiag, const int* mxddim, const int* mxdsml, const int* mxdbnd, const int* mxdgve,
                const int* mxdscr, const int* mxdanl);

/* ---- batched k-points ----
 * No counterpart in the reference, which applies H one k-point at a time
 * (Src/cpw_lib/cpw_scf.f90:488 -> h_kb_dia -> ditsp_c16 -> hk_psi_c16). A batch
 * holds the bases of nk k-points of one crystal (one FFT box, the context's
 * potential, one projector set per k-point) and applies
 * hpsi_k = H_k psi_k (hk_psi_c16.f90:28-241 per k) to all of them in one call:
 * one launch per local stage over the bands of every k-point (uneven plane-wave
 * and band counts), then the projector products of each k-point. The first
 * call with a given set of arrays and band counts times a small set of launch
 * shapes (autotuning), runs the fastest and captures it as a CUDA graph; later
 * calls with the same arrays and counts replay the graph. The precision is the
 * context's at creation (FP64, MIXED or MIXED_TC); the potential is the
 * context's (cpw_b200_set_potential), set before the first call.
 *
 * create: mtxd[k], isort[k] (1-based into kgv, reference layout), ekpg[k] are
 *   host arrays per k-point; kgv(3, ng) and kmscr(7) are shared. The context
 *   keeps k-point 0 as its own basis.
 * set_projectors: host anlga(ld, nanl) complex128 column-major (first mtxd[ik]
 *   rows used) and xnlkb(nanl) of k-point ik (proj_nl_kb_c16.f90 output).
 * hk_psi_device: per k-point device blocks psi[k], hpsi[k] (complex128,
 *   column-major, leading dimensions ldpsi[k], ldh[k] >= mtxd[k]) of nb[k]
 *   bands; stream: cudaStream_t the call is ordered after and before.
 * synchronize: waits for the batch's work; CPW_B200_TIMEOUT if a bounded wait
 *   in a tensor-core kernel gave up.
 * info: out[0..n) = {tuned, chunk bands, kernel B grouping, projection split
 *   setting, tuned call time in us, candidates timed, graph replays, captures}. */
typedef struct cpw_b200_kbatch cpw_b200_kbatch;
int cpw_b200_kbatch_create(cpw_b200_ctx* ctx, int nk, const int* mtxd, const int* const* isort, const int* kgv,
                           int ng, const double* const* ekpg, const int* kmscr, cpw_b200_kbatch** out);
int cpw_b200_kbatch_destroy(cpw_b200_kbatch* b);
int cpw_b200_kbatch_set_projectors(cpw_b200_kbatch* b, int ik, int nanl, const void* anlga, long long ld,
                                   const double* xnlkb);
int cpw_b200_kbatch_hk_psi_device(cpw_b200_kbatch* b, const int* nb, void* const* psi, const long long* ldpsi,
                                  void* const* hpsi, const long long* ldh, void* stream);
int cpw_b200_kbatch_synchronize(cpw_b200_kbatch* b);
int cpw_b200_kbatch_info(cpw_b200_kbatch* b, long long* out, int n);

/* ---- allocation-free local H|psi> ----
 * No counterpart in the reference. For callers that cannot call cudaMalloc
 * (a caller-owned memory pool or fixed device-memory budget, a host code that
 * owns every device buffer and forbids the library to grow the device heap):
 * hpsi = V_loc psi (+ ekpg psi when ekpg is not NULL), the local part of
 * hk_psi_c16, FP64, on `stream` (cudaStream_t; NULL = legacy default stream).
 * Every pointer except kmscr is device memory owned by the caller: psi/hpsi
 * complex128 column-major (ld >= mtxd), kgvb(3, mtxd) = kgv(:, isort(i)) of
 * the basis, ekpg(mtxd) or NULL, vscr in the reference layout holding at
 * least kmscr(7)*kmscr(5)*kmscr(6) doubles (id*n2*n3; not checked: a shorter
 * buffer is read out of bounds); kmscr(7) is host memory. The call allocates nothing: its work space (FFT
 * slab of a band chunk, plane lists, twiddles, repacked potential) is one
 * fixed device array of CPW_B200_NOALLOC_SCRATCH_BYTES held by every GPU that
 * loads the library until the process exits. Sizes whose set-up data or one
 * band's FFT slab do not fit are rejected with CPW_B200_BAD_ARG and a message.
 * All calls share the array: calls that overlap on the GPU race, so serialise
 * them. Each call reads the sphere extent of the basis back to the host, so
 * it returns only after the work queued before it on `stream` has finished.
 * The first call on a device looks up the array's address with that device
 * current; make it before any stream capture. The address is kept for the
 * life of the process: do not call this on a device after cudaDeviceReset. */
#define CPW_B200_NOALLOC_SCRATCH_BYTES (64LL << 20)
int cpw_b200_hk_psi_loc_noalloc(int mtxd, int neig, const void* psi, long long ldpsi, void* hpsi, long long ldhpsi,
                                const int* kgvb, const double* ekpg, const double* vscr, const int* kmscr,
                                void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CPW_B200_H */
