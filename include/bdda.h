/*
 * bdda.h -- C ABI of libbdda.so, the B200 (sm_100a) hot path of block-DDA:
 * the Goodman doubled-grid FFT matrix-vector product and the block Krylov
 * solvers built on it.
 *
 * Conventions
 *  - Every device buffer is allocated by the caller; the library never
 *    allocates or frees device memory.  Sizes come from the *_bytes queries.
 *  - All calls are stream-ordered on the given stream (a cudaStream_t passed
 *    as void*; NULL = legacy default stream).  Solver entry points read the
 *    residual back every iteration and therefore synchronise that stream.
 *  - Complex arrays are interleaved (re, im): c128 = 2 x double, c64 = 2 x float.
 *  - The plan tables and Green's spectra must be 16-byte aligned (they are
 *    staged into shared memory with 16-byte asynchronous copies).
 *  - Block vectors are row-major (3*N_occ, L): row 3m+c is component c of
 *    occupied dipole m, the L columns are orientations (reference layout,
 *    bl_krylov/bl_krylov.py:27-55).  Full-cuboid vectors are (3*Nc, L) with
 *    cells in C order (x slowest, z fastest), mvp_fft/mvp_fft.py:151-152.
 *  - Return value: a BDDA_* status code.
 *
 * Reference interfaces replaced (block-DDA_Py v0.3.0, paths in that project):
 *  mvp_fft/mvp_fft.py:13   build_interaction_tensor -> bdda_green_build (+ export)
 *  mvp_fft/mvp_fft.py:97   fft_init                 -> bdda_green_build
 *  mvp_fft/mvp_fft.py:122  fft_mvp                  -> bdda_fft_mvp
 *  bl_krylov/bl_krylov.py:5   _build_scatter_index  -> bdda_occupancy_map
 *  bl_krylov/bl_krylov.py:27  _block_mvp            -> bdda_block_mvp
 *  bl_krylov/bl_krylov.py:58  bl_cocg_rq_jacobi_mvp_fft  -> bdda_cocg_rq
 *  bl_krylov/bl_krylov.py:121 bl_bicgstab_jacobi_mvp_fft -> bdda_bicgstab
 *  bl_dda/scatterer.py:135-161 set_interaction_matrix (diag_A, B) -> bdda_polarizability, bdda_incident_rhs
 *  bl_dda/scatterer.py:182-227 E, C_abs, C_ext, S_fw, S_bk       -> bdda_observables
 *  bl_dda/scatterer.py:135-227 set_interaction_matrix + solve_matrix_equation + compute_* -> bdda_dda_solve
 *  shape_model/gaussian_ellipsoid.py:182-237 near-surface distance + inside test -> bdda_gre_occupancy
 */
#ifndef BDDA_H
#define BDDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bdda_plan bdda_plan;

enum bdda_status {
  BDDA_OK = 0,
  BDDA_NOT_CONVERGED = 1, /* solver ran itermax iterations without err < tol (not an error
                             in the reference, scatterer.py:175-176) */
  BDDA_BREAKDOWN = 2,     /* singular or non-finite L x L system (numpy LinAlgError) */
  BDDA_BAD_ARG = 3,       /* invalid size, pointer or option (reference ValueError) */
  BDDA_NO_WORKSPACE = 4,  /* workspace pointer missing or plan tables not attached */
  BDDA_TIMEOUT = 5,       /* a bounded device-side wait gave up */
  BDDA_CUDA_ERROR = 6     /* a CUDA runtime call failed */
};

enum bdda_solver_kind {
  BDDA_BICGSTAB = 0, /* block-BiCGSTAB, bl_krylov/bl_krylov.py:121 */
  BDDA_COCG_RQ = 1   /* block-COCG-rq,  bl_krylov/bl_krylov.py:58 */
};

enum bdda_precision {
  BDDA_C128 = 0, /* complex128 end to end */
  BDDA_C64 = 1   /* complex64 storage, FP32 arithmetic */
};

const char* bdda_status_string(int status);
int bdda_version(void);

/* ---- plan: grid geometry and FFT factorisation (host object) -------------
 * n = cuboid (Nx, Ny, Nz).  m = cyclic FFT grid; NULL chooses, per axis, the
 * smallest even 7-smooth length >= 2N (= 2N, the reference's doubled grid,
 * whenever 2N is 7-smooth).  Any m >= 2N-1 gives the same product, because
 * only displacements |d| <= N-1 reach the cropped output.
 * replaces the implicit grid of mvp_fft/mvp_fft.py:43-45,155 */
int bdda_plan_create(const int n[3], const int m[3], bdda_plan** out);
void bdda_plan_destroy(bdda_plan* plan);
int bdda_plan_grid(const bdda_plan* plan, int m[3]);
int bdda_plan_radices(const bdda_plan* plan, int axis, int radices[12], int* nstage);
/* Twiddle and digit-reversal tables: the caller gives a device buffer of
 * bdda_plan_table_bytes(); the plan uploads into it and keeps the pointer. */
size_t bdda_plan_table_bytes(const bdda_plan* plan);
int bdda_plan_attach_tables(bdda_plan* plan, void* dev_tables, void* stream);
/* Bounded waits of this plan's pass kernels that ran out (a CTA whose tile
 * copy did not land in time counts one and leaves its pencil unwritten): 0
 * in every correct run.  The counter lives in the table buffer, zeroed by
 * bdda_plan_attach_tables; the solve entry points read it when they finish
 * and return BDDA_TIMEOUT if it is not 0.  Synchronises the stream. */
int bdda_plan_wait_timeouts(const bdda_plan* plan, unsigned int* count, void* stream);

/* Launch shape of the pencil passes (no counterpart in the reference; used by
 * the autotuner).  kind: 0 forward passes (Z, Y), 1 X pass (forward, Green
 * multiply, inverse), 2 inverse passes (Y^-1, Z^-1).  smem_budget bounds the
 * shared memory of one CTA and so selects the widest column tile that fits;
 * threads per CTA is a multiple of 32 up to 512.  Process-wide settings. */
int bdda_tune_set(int prec, int kind, size_t smem_budget, int threads);
int bdda_tune_get(int prec, int kind, size_t* smem_budget, int* threads);
/* Per-pass launch choice for passes of (prec, kind) over an axis of length M
 * at block width L: column tile width lt (2, 4, 8, 16; 0 = the smem_budget rule)
 * and kernel variant (0 = the first specialised kernel compiled for the radix
 * sequence; k in 1..8 = the one of 256 threads compiled for k resident CTAs
 * per SM; k + 16 * (threads / 32) = the one of that CTA size; 512 + either
 * = a complex64 kernel whose jobs take two adjacent columns, used when L is
 * even and the pass's field pointers are 16-byte aligned; 1024 + any of
 * these = the same kernel with the tile's first read done by a bulk tensor
 * copy (TMA), used when the pass's source is dense and 16-byte aligned, the
 * plain kernel otherwise; 2048 + (0 or 1024) + MINB + 16 * (threads / 32) =
 * an X-pass kernel that transforms the axis in two register stages (a
 * 192-point axis as 24 x 8) instead of the plan's radix sequence, with or
 * without the TMA-filled tile; -1 = the generic run-time-radix kernel, -2 =
 * the same with the TMA-filled tile, which a pass without a specialised
 * kernel for its radix sequence runs when no choice is set).
 * lt 16 exists as specialised kernels only.  Process-wide; set by
 * bdda_autotune. */
int bdda_tune_pass(int prec, int kind, int M, int L, int lt, int variant);
int bdda_tune_pass_get(int prec, int kind, int M, int L, int* lt, int* variant);
/* Variant ids (as bdda_tune_pass) of the specialised kernels compiled for the
 * pass (prec, kind) over this plan's axis (0 = x, 1 = y, 2 = z) at tile width
 * lt: up to cap of them into variants, their number into *n. */
int bdda_tune_pass_variants(const bdda_plan* plan, int prec, int kind, int axis, int lt, int* variants, int cap,
                            int* n);
/* Autotuner (no counterpart in the reference; the reference's scipy.fft plans
 * itself).  Runs block MVPs of this plan on the caller's buffers (arguments as
 * bdda_block_mvp; out and work are overwritten), times each pass over every
 * candidate (tile width x kernel variant) with CUDA events, reps timed
 * products per candidate, and keeps the fastest per pass key through
 * bdda_tune_pass.  ms_before / ms_after (nullable): one product before and
 * after.  Synchronises the stream; do not call during stream capture. */
int bdda_autotune(const bdda_plan* plan, int prec, int L, const void* ghat, const int32_t* cell_map,
                  const void* diag, const void* jpre, const void* S, void* out, void* work, int reps,
                  double* ms_before, double* ms_after, void* stream);
/* on != 0 (default): radix sequences and block widths L with a compile-time-
 * specialised kernel use it (FFT passes, Gram products, block updates) */
int bdda_tune_fixed(int on);

/* ---- Green's tensor spectrum ----------------------------------------------
 * A'(r) (mvp_fft/mvp_fft.py:77-84) on the cyclic grid, 6 unique components
 * (xx, xy, xz, yy, yz, zz), forward FFT over the three axes.  Stored in the
 * library's own order (x-pencil major, spectra digit-reversed).
 * replaces mvp_fft/mvp_fft.py:13 build_interaction_tensor + :97 fft_init */
size_t bdda_green_bytes(const bdda_plan* plan, int prec);
size_t bdda_green_build_workspace_bytes(const bdda_plan* plan);
int bdda_green_build(const bdda_plan* plan, double lf, double k, void* ghat_c128, void* work,
                     void* stream);
/* Real-space tensor A'(r) in natural order (Mx, My, Mz, 3, 3) c128, origin and
 * non-physical displacements zero: the reference's array when m = 2n.
 * replaces mvp_fft/mvp_fft.py:13 build_interaction_tensor */
int bdda_green_real(const bdda_plan* plan, double lf, double k, void* full_c128, void* stream);
/* c128 -> c64 rounding copy for the FP32 product */
int bdda_green_convert(const bdda_plan* plan, const void* ghat_c128, void* ghat_c64, void* stream);
/* Library order <-> natural (Mx, My, Mz, 3, 3) c128 (the reference's Au_til
 * layout when m = 2n).  Import reads the upper triangle. */
int bdda_green_export(const bdda_plan* plan, const void* ghat_c128, void* full_c128, void* stream);
int bdda_green_import(const bdda_plan* plan, const void* full_c128, void* ghat_c128, void* stream);

/* ---- matrix-vector products ------------------------------------------------ */
size_t bdda_mvp_workspace_bytes(const bdda_plan* plan, int prec, int L);
/* cell_map[cell] = m for address[m] = cell, -1 elsewhere (Nc int32).
 * replaces bl_krylov/bl_krylov.py:5 _build_scatter_index */
int bdda_occupancy_map(const bdda_plan* plan, const int64_t* address, int n_occ,
                       int32_t* cell_map, void* stream);
/* Y_full = A_off P_full on the full cuboid, (3 Nc, L).
 * replaces mvp_fft/mvp_fft.py:122 fft_mvp */
int bdda_fft_mvp(const bdda_plan* plan, int prec, int L, const void* ghat, const void* P_full,
                 void* Y_full, void* work, void* stream);
/* out = jpre * (diag * S + gather(A_off scatter(S))), S and out (3 N_occ, L).
 * replaces bl_krylov/bl_krylov.py:27 _block_mvp */
int bdda_block_mvp(const bdda_plan* plan, int prec, int L, const void* ghat,
                   const int32_t* cell_map, const void* diag, const void* jpre, const void* S,
                   void* out, void* work, void* stream);

/* Block MVP with no scratch argument (no counterpart in the reference).  For
 * callers that cannot allocate device memory -- a plugin whose host
 * application's allocator owns all device memory, or a latency-critical path
 * that cannot take the synchronisation cudaMalloc / cudaFree may imply.  Same
 * product and arguments as bdda_block_mvp minus `work`; the scratch field
 * buffer is a static 64 MiB device array (bdda_block_mvp_noalloc_max_bytes())
 * that every GPU loading the library holds until exit.  Returns BDDA_BAD_ARG
 * when bdda_mvp_workspace_bytes(plan, prec, L) exceeds it
 * (bdda_block_mvp_noalloc_fits() tells in advance).  All calls on a device
 * share the array: calls that overlap on the GPU race, so serialise them.
 * Nothing in it needs to start at zero.  The first call on a device looks up
 * the array's address with that device current; make it before any stream
 * capture.  That address is kept until exit: do not cudaDeviceReset a device
 * after calling this entry point on it.  It allocates nothing (cudaMalloc, cudaFree and allocating library
 * routines are never called; profiling, off by default, creates CUDA events). */
size_t bdda_block_mvp_noalloc_max_bytes(void);
int bdda_block_mvp_noalloc_fits(const bdda_plan* plan, int prec, int L);
int bdda_block_mvp_noalloc(const bdda_plan* plan, int prec, int L, const void* ghat,
                           const int32_t* cell_map, const void* diag, const void* jpre, const void* S,
                           void* out, void* stream);

/* ---- block Krylov solvers -----------------------------------------------------
 * Solve A X = B with Jacobi left preconditioning, M = diag(A): iterate on
 * M^-1 A X = M^-1 B until ||R||_F / ||M^-1 B||_F < tol (a single global
 * Frobenius criterion over the L columns, bl_krylov.py:106,177) or itermax
 * iterations.  diag (3 N_occ) c128 is DIAG_A; B, X0 (nullable = zero start)
 * and X are (3 N_occ, L) c128.  prec selects the storage/arithmetic of the
 * Krylov vectors and of the product (ghat must be in that precision); the
 * L x L Gram matrices, solves and QR factors are always FP64.
 * iter_fin is the 0-based index of the last iteration, err_fin its relative
 * residual (reference semantics); history (nullable, itermax doubles, host)
 * receives the residual of every iteration.  L <= 64.
 * Returns BDDA_OK (converged), BDDA_NOT_CONVERGED (itermax reached, or the
 * iteration produced non-finite values: err_fin is then NaN/Inf), or
 * BDDA_BREAKDOWN (exactly singular L x L system: numpy's LinAlgError).
 * The stream is synchronised once per iteration to read the residual. */
size_t bdda_solver_workspace_bytes(const bdda_plan* plan, int solver, int prec, int L, int n_occ);
int bdda_solve(const bdda_plan* plan, int solver, int prec, int L, int n_occ, const void* ghat,
               const int32_t* cell_map, const void* diag, const void* B, const void* X0, double tol,
               int itermax, void* X, int* iter_fin, double* err_fin, double* history, void* work,
               size_t work_bytes, void* stream);
/* replaces bl_krylov/bl_krylov.py:121 bl_bicgstab_jacobi_mvp_fft */
int bdda_bicgstab(const bdda_plan* plan, int prec, int L, int n_occ, const void* ghat,
                  const int32_t* cell_map, const void* diag, const void* B, const void* X0,
                  double tol, int itermax, void* X, int* iter_fin, double* err_fin,
                  double* history, void* work, size_t work_bytes, void* stream);
/* replaces bl_krylov/bl_krylov.py:58 bl_cocg_rq_jacobi_mvp_fft */
int bdda_cocg_rq(const bdda_plan* plan, int prec, int L, int n_occ, const void* ghat,
                 const int32_t* cell_map, const void* diag, const void* B, const void* X0,
                 double tol, int itermax, void* X, int* iter_fin, double* err_fin,
                 double* history, void* work, size_t work_bytes, void* stream);

/* ---- FP32 Krylov with FP64 refinement (no counterpart in the reference) ----------
 * Products and Krylov vectors in complex64 (ghat_c64), the solution and the
 * true residual r = M^-1 (B - A X) in complex128 (ghat_c128); FP64 Gram
 * matrices and small solves.  Converged when ||r||_F / ||M^-1 B||_F < tol.
 *  - max_outer > 0: restarted refinement, at most max_outer corrections;
 *    each solves M^-1 A D = r in FP32 with the chosen block solver to the
 *    relative tolerance max(inner_tol, 0.3 tol / err) and sets X += D.  A
 *    correction that raises the true residual is undone and ends the solve.
 *  - max_outer < 0 with BDDA_BICGSTAB: one block-BiCGSTAB recursion in FP32
 *    with FP64 reliable updates: X accumulates in FP64 and R is replaced by
 *    the true FP64 residual whenever the recursive residual fell by the
 *    factor inner_tol since the last replacement and before convergence is
 *    declared.  No restarts; suited to small L (the FP32 recursion's
 *    attainable accuracy drops with the block width).
 * itermax caps the FP32 iterations in total.  iter_fin = that count - 1;
 * err_fin = the true relative residual of the returned X; history
 * (nullable, itermax doubles) = per-iteration residual relative to
 * ||M^-1 B||.  Returns BDDA_OK when err_fin < tol, else BDDA_NOT_CONVERGED
 * (or BDDA_BREAKDOWN as bdda_solve). */
size_t bdda_refine_workspace_bytes(const bdda_plan* plan, int L, int n_occ);
int bdda_refine_solve(const bdda_plan* plan, int solver, int L, int n_occ, const void* ghat_c128,
                      const void* ghat_c64, const int32_t* cell_map, const void* diag, const void* B,
                      const void* X0, double tol, int itermax, double inner_tol, int max_outer, void* X,
                      int* iter_fin, double* err_fin, double* history, void* work, size_t work_bytes,
                      void* stream);

/* ---- complex128 Krylov with complex64 products (no counterpart in the
 * reference) ------------------------------------------------------------------
 * The block solver of `solver` with X, the residual, every Krylov vector,
 * Gram product and L x L step in complex128, and the products inside the
 * iteration in complex64 (ghat_c64 from bdda_green_convert).  BiCGSTAB
 * replaces its recursive residual by the true one ||M^-1 (B - A X)|| /
 * ||M^-1 B|| (complex128 product) after every replace_drop-fold drop and
 * before it stops, and finishes with complex128 products once the true
 * residual is below switch_ratio * tol (bdda_tune_mixed); a recursion that
 * diverges is abandoned for complex128 products, warm-started from the X of
 * its smallest residual when that is below 1.  COCG-rq's
 * recursion runs to tol / 2 and the true residual then decides.  The solver
 * restarts from X (exact product) while the true residual is not below tol,
 * up to max_outer rounds.  err_fin is the final residual (the true one, or
 * after a switch the complex128 recursion's); iter_fin counts the iterations
 * of all rounds. */
size_t bdda_mixed_workspace_bytes(const bdda_plan* plan, int L, int n_occ);
/* Process-wide settings of bdda_mixed_solve's BiCGSTAB (and of the batched
 * solver's mode MIXED for replace_drop and diverge_factor): replace_drop in
 * (0, 1), default 0.1; switch_ratio >= 0, default 0 (complex64 products to
 * the end); diverge_factor > 1, default 10: the recursion counts as
 * diverged once its residual exceeds its smallest value so far by this
 * (in the one-problem solver: in its first 8 iterations before any residual
 * replacement, the first iteration's residual instead, which block
 * BiCGSTAB's early rise can exceed tenfold; a recursion whose smallest
 * residual has not halved in 60 iterations counts as stalled, with the same
 * complex128 fallback). */
int bdda_tune_mixed(double replace_drop, double switch_ratio, double diverge_factor);
int bdda_tune_mixed_get(double* replace_drop, double* switch_ratio, double* diverge_factor);
/* Small one-problem solves (padded grid points x L <= 64 Mi, itermax <= 4096,
 * plain complex128 / complex64 forms) run their iterations as a CUDA graph
 * "while" node: one iteration is captured as the body and the loop condition
 * is set on the device at the residual test, so a solve is one graph launch
 * and one read-back instead of ~20 launches and a synchronisation per
 * iteration.  on = 0 uses the host-driven loop everywhere (process-wide). */
int bdda_tune_solver_graphs(int on);
int bdda_mixed_solve(const bdda_plan* plan, int solver, int L, int n_occ, const void* ghat_c128,
                     const void* ghat_c64, const int32_t* cell_map, const void* diag, const void* B,
                     const void* X0, double tol, int itermax, int max_outer, void* X, int* iter_fin,
                     double* err_fin, double* history, void* work, size_t work_bytes, void* stream);

/* ---- batched solve (no counterpart in the reference, which solves one problem
 * per call: scatterer.py:169-171 inside the loops of run_dda.py:56-65) --------
 * Many independent block-BiCGSTAB problems -- particles, wavelengths,
 * orientation blocks, each with its own plan (grid), Green's spectrum,
 * occupancy map, Jacobi diagonal and right-hand sides -- advance together:
 * every step of an iteration is one persistent launch over a device work list
 * of the problems still iterating, each problem's convergence test runs on
 * the device, and the iteration is replayed as a CUDA graph (use_graph != 0).
 * Per problem the result is that of bdda_bicgstab (mode C128 / C64) or of
 * bdda_mixed_solve (mode MIXED, at most max_outer rounds).  All problems share L, which
 * is 8, 16, 32 or 64; at most 1024 problems per call. */
typedef struct bdda_batch_problem {
  const bdda_plan* plan;      /* the problem's grid, tables attached */
  int n_occ;                  /* occupied dipoles */
  const void* ghat;           /* complex128 spectrum (modes C128 and MIXED) */
  const void* ghat_c64;       /* complex64 spectrum (modes C64 and MIXED) */
  const int32_t* cell_map;    /* bdda_occupancy_map of the problem */
  const void* diag;           /* complex128 [3 n_occ], DIAG_A */
  const void* B;              /* complex128 [3 n_occ][L] */
  const void* X0;             /* complex128 [3 n_occ][L] warm start, or NULL */
  void* X;                    /* complex128 [3 n_occ][L] output */
} bdda_batch_problem;

enum bdda_batch_mode {
  BDDA_BATCH_C128 = 0,        /* complex128 solves */
  BDDA_BATCH_C64 = 1,         /* complex64 vectors and products, FP64 Gram / L x L */
  BDDA_BATCH_MIXED = 2        /* complex128 vectors, complex64 products (bdda_mixed_solve) */
};

/* Device workspace of one batched call (0: bad arguments). */
size_t bdda_batch_workspace_bytes(const bdda_batch_problem* problems, int nprob, int mode, int L, int itermax);
/* status[i], iter_fin[i], err_fin[i] (host arrays of nprob) receive each
 * problem's outcome as bdda_bicgstab reports it; history (host, nprob x
 * itermax, nullable) the residual per iteration.  Returns BDDA_OK when every
 * problem converged, else BDDA_BREAKDOWN if one broke down, else
 * BDDA_NOT_CONVERGED; argument and CUDA errors as elsewhere.  Runs on its own
 * stream ordered after `stream`, and synchronises it. */
int bdda_batch_bicgstab(const bdda_batch_problem* problems, int nprob, int mode, int L, double tol, int itermax,
                        int max_outer, int use_graph, int* status, int* iter_fin, double* err_fin, double* history,
                        void* work, size_t work_bytes, void* stream);

/* ---- learned warm start (no counterpart in the reference, whose solvers
 * start from X0 = 0: bl_krylov.py:84-85,146) ------------------------------------
 * A Fourier neural operator maps, per lattice cell and orientation, the
 * occupancy mask, the per-axis chi = (eps - 1)/(eps + 2) and the Jacobi guess
 * J = B / DIAG_A (scaled by its RMS) to a correction of J:
 * X0 = J + scale * y.  lift cin -> width, `layers` Fourier layers (per-mode
 * complex width x width matrices on the `modes` lowest frequencies per axis,
 * plus a pointwise width x width map, GELU), projection width -> proj -> cout.
 * The shipped shapes are cin 13, width 32, cout 6, proj 64; every lattice
 * axis is at least `modes` and at most 512 cells.  One call handles B samples
 * (orientations) of one lattice; activations live in `work`
 * (bdda_fno_workspace_bytes), parameters in one FP32 array
 * (bdda_fno_param_count floats, layout by bdda_fno_offset).  bdda_fno_features
 * also writes the lattice's DFT tables into `work`; the other calls on that
 * workspace use them, so it comes first for each lattice. */
typedef struct bdda_fno_config {
  int cin, width, cout, proj, layers, modes;
} bdda_fno_config;

size_t bdda_fno_param_count(const bdda_fno_config* cfg);
/* what: 0 P, 1 p, 2 R_l, 3 W_l, 4 b_l, 5 Q1, 6 q1, 7 Q2, 8 q2 (float offset) */
size_t bdda_fno_offset(const bdda_fno_config* cfg, int what, int layer);
size_t bdda_fno_workspace_bytes(const bdda_fno_config* cfg, int B, const int n[3]);
/* byte offset in `work` of: 0 features [B][cells][cin], 1 output [B][cells][cout],
 * 2 mask [cells], 3 loss gradient [B][cells][cout], 4 target [B][cells][cout] */
size_t bdda_fno_buffer_offset(const bdda_fno_config* cfg, int B, const int n[3], int which);
/* Features of the L = B orientations of one particle into work; scale (device,
 * L doubles) receives the RMS of each Jacobi-guess column. */
int bdda_fno_features(const bdda_fno_config* cfg, const int n[3], int n_occ, int L, const int32_t* cell_map,
                      const void* diag, const void* B, const double chi[6], double* scale, void* work,
                      size_t work_bytes, void* stream);
/* Forward pass on the features in work (train != 0 keeps what backward needs). */
int bdda_fno_forward(const bdda_fno_config* cfg, int B, const int n[3], const float* params, int train, void* work,
                     size_t work_bytes, void* stream);
/* Masked relative squared error of the output against the solution X
 * (complex128 [3 n_occ][B]): mean over samples of
 * sum |y - (X - J)/scale|^2 / sum |(X - J)/scale|^2 over occupied cells; its
 * gradient w.r.t. the output goes to the work buffer 3.  *loss is written
 * when the stream reaches it. */
int bdda_fno_loss(const bdda_fno_config* cfg, int B, const int n[3], int n_occ, const int32_t* cell_map,
                  const void* diag, const void* Bm, const void* X, const double* scale, double* loss, void* work,
                  size_t work_bytes, void* stream);
/* Gradients of every parameter, ADDED to grads (zero it first); grad_out null
 * means the loss gradient in work. */
int bdda_fno_backward(const bdda_fno_config* cfg, int B, const int n[3], const float* params, const float* grad_out,
                      float* grads, void* work, size_t work_bytes, void* stream);
/* One Adam step (bias-corrected, decoupled weight decay as L2 on the gradient). */
int bdda_fno_adam(float* params, const float* grads, float* m, float* v, size_t n, float lr, float beta1, float beta2,
                  float eps, float weight_decay, int step, void* stream);
/* X0 (complex128 [3 n_occ][L]) = J + scale * output at the occupied cells. */
int bdda_fno_warm_start(const bdda_fno_config* cfg, const int n[3], int n_occ, int L, const int32_t* cell_map,
                        const void* diag, const void* B, const double* scale, void* X0, void* work,
                        size_t work_bytes, void* stream);

/* ---- physics around the solve --------------------------------------------------
 * Homogeneous particle, per-axis index m_p_xyz = (re x, im x, re y, im y, re z, im z):
 * eps_r = m_p^2 / m_m^2, Clausius-Mossotti polarizability with the CR2009
 * correction, diag = 1 / alpha ordered [x0 y0 z0 x1 ...] (3 N_occ c128);
 * eper_r (nullable) receives eps_r in the same order.
 * replaces bl_dda/scatterer.py:137-148 */
int bdda_polarizability(int n_occ, const double m_p_xyz[6], double m_m, double lf, double k, void* diag,
                        void* eper_r, void* stream);
/* B[3n + c, l] = e0[l, c] exp(i k u_inc[l] . pos[n]); pos (N_occ, 3) and
 * u_inc (L, 3) double, e0 (L, 3) c128, all on the device.
 * replaces bl_dda/scatterer.py:153-161 */
int bdda_incident_rhs(int n_occ, int L, double k, const double* pos, const double* u_inc, const void* e0,
                      void* B, void* stream);
/* Per orientation, from the solution X (3 N_occ, L): out (L, 12) doubles =
 * C_abs, C_ext, S_fw_theta (re, im), S_fw_phi, S_bk_theta, S_bk_phi, S_bk.
 * vec (L, 21) doubles = u_inc, u_fw, theta_fw, phi_fw, u_bk, theta_bk, phi_bk
 * (particle frame); e0 (L, 3) c128; eper_r (3 N_occ) c128; absorbing = mean
 * Im eps_r >= 1e-12 (else C_abs = 0, scatterer.py:189).
 * replaces bl_dda/scatterer.py:182-227 */
size_t bdda_observables_workspace_bytes(int L);
int bdda_observables(int n_occ, int L, double k, double lf, int absorbing, const double* pos,
                     const void* eper_r, const void* X, const double* vec, const void* e0, double* out,
                     void* work, void* stream);

/* ---- instrumentation (no counterpart in the reference) -------------------------
 * Number of kernels this library has launched in the process.  With
 * profiling on, every block MVP records CUDA events around its five passes;
 * bdda_profile_read waits for them and returns, over the products of one
 * precision (prec = BDDA_C128 / BDDA_C64, or -1 for all), the summed
 * milliseconds of each pass and the number of products.  Enabling clears
 * earlier records. */
unsigned long long bdda_launch_count(void);
int bdda_profile_enable(int on);
int bdda_profile_read(int prec, double pass_ms[5], long long* n_mvp);

/* ---- one DDA solve: set-up, block solve and observables in one call --------
 * replaces, for one particle and L orientations, set_interaction_matrix
 * (bl_dda/scatterer.py:135-161; the Green's spectrum ghat comes from
 * bdda_green_build), solve_matrix_equation (:164-184, block-BiCGSTAB as the
 * reference or block-COCG-rq) and compute_C_abs / compute_C_ext /
 * compute_PCAS_observable_S_fw / compute_OCBS_observable_S_bk (:187-227).
 * The prologue forms diag_A and the Jacobi-scaled right-hand side M^-1 B
 * directly from the positions and incident vectors (B is never stored); the
 * epilogue accumulates the observables in the pass that writes X.
 * mode: BDDA_BATCH_C128 (ghat_c128), BDDA_BATCH_C64 (ghat_c64) or
 * BDDA_BATCH_MIXED (both; max_outer warm-restarted rounds, as
 * bdda_mixed_solve).  Outputs: X (3N, L) c128; obs (L, 12) doubles on the
 * device = C_abs, C_ext, S_fw_theta (re, im), S_fw_phi (re, im), S_bk_theta
 * (re, im), S_bk_phi (re, im), S_bk (re, im), all zero when the solve did
 * not converge (the reference sets P = E only on convergence); diag_out and
 * eper_out (3N c128, nullable) receive diag_A and eps_r.  Return codes and
 * iter_fin / err_fin / history as bdda_solve (bdda_mixed_solve in the mixed
 * mode). */
typedef struct bdda_dda_problem {
  int n_occ;            /* occupied dipoles N */
  int L;                /* orientations (<= 64) */
  double m_p_xyz[6];    /* particle index per axis: re, im of x, y, z */
  double m_m;           /* medium index */
  double lf;            /* lattice spacing */
  double k;             /* wavenumber in the medium, 2 pi m_m / wl_0 */
  int absorbing;        /* 1: C_abs computed (mean Im eps_r >= 1e-12, scatterer.py:189); 0: C_abs = 0 */
  const double* pos;    /* (N, 3) dipole positions, device */
  const double* vec;    /* (L, 21) per orientation: u_inc, u_fw, theta_fw, phi_fw, u_bk, theta_bk, phi_bk */
  const void* e0;       /* (L, 3) c128 incident polarisation vectors, device */
} bdda_dda_problem;
size_t bdda_dda_workspace_bytes(const bdda_plan* plan, int mode, int L, int n_occ);
int bdda_dda_solve(const bdda_plan* plan, const bdda_dda_problem* prob, int solver, int mode, const void* ghat_c128,
                   const void* ghat_c64, const int32_t* cell_map, const void* X0, double tol, int itermax,
                   int max_outer, void* X, void* diag_out, void* eper_out, double* obs, int* iter_fin,
                   double* err_fin, double* history, void* work, size_t work_bytes, void* stream);

/* ---- GRE lattice occupancy (shape_model/gaussian_ellipsoid.py:182-237) -------
 * replaces find_nearest_distance_from_the_GRE_surf (:182-192, a k-d tree
 * query) and extract_lattice_address_in_GRE_volume (:195-237).  Cell (i,j,k)
 * of the nx x ny x nz lattice sits at (xs[i], ys[j], zs[k]) (the reference's
 * axis arrays); near[c] = 1 when some surface point lies closer than thr
 * (distance evaluated as the reference, sqrt((dx^2 + dy^2) + dz^2), each
 * operation rounded); inside[c] = 1 when near cells lie strictly before and
 * strictly after c along all three axes.  c = (i ny + j) nz + k.  The npts
 * surface points (x, y, z doubles) must be sorted by bin of a uniform grid
 * of nbx x nby x nbz bins of edge h >= thr whose corner is (ox, oy, oz):
 * bin b = (bx nby + by) nbz + bz, bx = floor((x - ox) / h); points of bin b
 * are pts[bin_start[b] .. bin_start[b+1]).  All arrays are device memory;
 * work holds bdda_gre_occupancy_workspace_bytes(). */
size_t bdda_gre_occupancy_workspace_bytes(int nx, int ny, int nz);
int bdda_gre_occupancy(int nx, int ny, int nz, const double* xs, const double* ys, const double* zs, int npts,
                       const double* pts, const int32_t* bin_start, int nbx, int nby, int nbz, double ox,
                       double oy, double oz, double h, double thr, uint8_t* near, uint8_t* inside, void* work,
                       size_t work_bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* BDDA_H */
