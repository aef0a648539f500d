// Block Krylov solvers on the device: block-BiCGSTAB and block-COCG-rq with
// Jacobi (diagonal) left preconditioning, built on the fused block MVP.
//
// The host loop launches kernels only; every coefficient (alpha, beta, zeta,
// xi, tau) lives in device memory.  Once per iteration a 16-byte status
// (relative residual, breakdown flag) is read back to decide termination,
// exactly where the reference tests ``err < tol`` (bl_krylov.py:110,181).
// For small problems, where that read-back and the launches would dominate,
// the plain solves instead capture one iteration as the body of a CUDA graph
// "while" node: a one-thread kernel at the test point records the residual and
// sets the loop condition on the device, so the whole solve is one graph
// launch and one read-back.
#include <cmath>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <utility>

#include "bdda_blas.cuh"
#include "bdda_internal.h"
#include "bdda_small.cuh"
#include "bdda_steps.cuh"
#include "bdda_dda.cuh"

namespace bdda {

struct Layout {
  size_t field, vec[8], diag, jpre, partial, small, state, hist, total;
};

// Residual history slots of the graph-driven loop (longer solves run the
// host-driven loop), and the largest product work (padded grid points x L)
// for which it is used: above it an iteration is long enough that the launches
// and the read-back do not matter.
constexpr int kGraphHistCap = 4096;
constexpr double kGraphMaxWork = 64.0 * 1024 * 1024;

constexpr int kVecs = 8;

static size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

static Layout layout(const bdda_plan* p, int prec, int L, int n_occ) {
  Layout o;
  const size_t cb = cplx_bytes(prec);
  const size_t vbytes = (size_t)3 * n_occ * L * cb;
  size_t off = 0;
  o.field = off; off = al(off + bdda_mvp_workspace_bytes(p, prec, L));
  for (int v = 0; v < kVecs; ++v) { o.vec[v] = off; off = al(off + vbytes); }
  o.diag = off; off = al(off + (size_t)3 * n_occ * cb);
  o.jpre = off; off = al(off + (size_t)3 * n_occ * cb);
  o.partial = off; off = al(off + (size_t)kRedBlocks * 2 * kMaxL * kMaxL * sizeof(double2));
  o.small = off; off = al(off + (size_t)kSmallMats * kMaxL * kMaxL * sizeof(double2) + 64 * sizeof(int));
  o.state = off; off = al(off + sizeof(SolverState));
  o.hist = off; off = al(off + kGraphHistCap * sizeof(double));
  o.total = off;
  return o;
}

// ---- elementwise set-up kernels -------------------------------------------------
// jpre = 1/diag and Bj = B * jpre in complex128 (bl_krylov.py:84-87,146-149),
// then stored in the working precision
template <typename T>
__global__ void prepare_kernel(const double2* diag, const double2* B, int64_t nrow, int L, T* diagT,
                               T* jpreT, T* Bj) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nrow * L;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / L;
    const double2 d = diag[r];
    const double2 j = zdiv(make_double2(1.0, 0.0), d);
    if (Bj) Bj[i] = from_d2<T>(zmul(B[i], j));
    if (i % L == 0) {
      diagT[r] = from_d2<T>(d);
      jpreT[r] = from_d2<T>(j);
    }
  }
}

template <typename T>
__global__ void convert_in_kernel(const double2* in, T* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = from_d2<T>(in[i]);
}

template <typename T>
__global__ void convert_out_kernel(const T* in, double2* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = to_d2(in[i]);
}

// ---- one-CTA step kernels (bodies in bdda_steps.cuh) ----------------------------
__global__ void norm_kernel(const double* partial, int nblk, SolverState* st, int set_bnorm) {
  norm_body(partial, nblk, st, set_bnorm);
}

// BiCGSTAB: LU(RV), alpha = RV^-1 (R0^H R)   (bl_krylov.py:166-167)
__global__ void bicg_alpha_kernel(SmallPtrs s, int L, SolverState* st) {
  extern __shared__ double2 sm[];
  bicg_alpha_body(s, L, st, sm);
}

// BiCGSTAB: zeta = tr(Z^H T) / tr(Z^H Z); beta = RV^-1 (-R0^H Z)   (bl_krylov.py:173,184)
__global__ void bicg_zeta_beta_kernel(SmallPtrs s, int L, const double* dot_partial, int nblk,
                                      SolverState* st) {
  extern __shared__ double2 sm[];
  bicg_zeta_beta_body(s, L, dot_partial, nblk, st, sm);
}

// CholeskyQR step: R = chol(G [+ shift I]), rinv = R^-1, tau <- R tau (tau = R on the first step)
__global__ void cholqr_step_kernel(SmallPtrs s, int L, int first, double shift_coef, SolverState* st) {
  extern __shared__ double2 sm[];
  double2* g = sm;
  double2* x = sm + L * L;
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  block_copy(g, s.g2, L * L);
  __syncthreads();
  if (first && shift_coef > 0.0) {
    if (threadIdx.x == 0) {
      double tr = 0.0;
      for (int i = 0; i < L; ++i) tr += g[i * L + i].x;
      const double sh = shift_coef * tr;
      for (int i = 0; i < L; ++i) g[i * L + i].x += sh;
    }
    __syncthreads();
  }
  chol_upper(g, L, &bad);
  tri_upper_inv(g, L, x);
  block_copy(s.rinv, x, L * L);
  // tau <- R tau
  if (first) {
    block_copy(s.tau, g, L * L);
  } else {
    block_copy(x, s.tau, L * L);
    __syncthreads();
    small_matmul<false>(g, x, s.tmp, L);
    block_copy(s.tau, s.tmp, L * L);
  }
  __syncthreads();
  if (threadIdx.x == 0 && bad == 1) atomicExch(&st->bad, 1);
  if (threadIdx.x == 0 && bad == 2) atomicCAS(&st->bad, 0, 2);
}

// COCG: alpha = (S^T AS)^-1 (Q^T Q); alphaxi = alpha xi   (bl_krylov.py:101-102)
__global__ void cocg_alpha_kernel(SmallPtrs s, int L, SolverState* st) {
  extern __shared__ double2 sm[];
  double2* a = sm;
  double2* b = sm + L * L;
  double2* c = sm + 2 * L * L;
  __shared__ int piv[kMaxL];
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  block_copy(a, s.g2, L * L);
  block_copy(b, s.qq, L * L);
  __syncthreads();
  lu_factor(a, L, piv, &bad);
  if (!bad) lu_solve(a, piv, L, b, L);
  block_copy(c, s.xi, L * L);
  __syncthreads();
  small_matmul<false>(b, c, a, L);
  for (int e = threadIdx.x; e < L * L; e += blockDim.x) {
    s.alpha[e] = b[e];
    s.negalpha[e] = make_double2(-b[e].x, -b[e].y);
    s.alphaxi[e] = a[e];
  }
  __syncthreads();
  if (threadIdx.x == 0 && bad == 1) atomicExch(&st->bad, 1);
  if (threadIdx.x == 0 && bad == 2) atomicCAS(&st->bad, 0, 2);
  flag_nonfinite(b, L * L, st);
}

// COCG: xi <- tau xi; err = ||xi||_F / ||M^-1 B||_F   (bl_krylov.py:105-106)
__global__ void cocg_xi_kernel(SmallPtrs s, int L, SolverState* st, int init) {
  extern __shared__ double2 sm[];
  double2* t = sm;
  double2* x = sm + L * L;
  double2* y = sm + 2 * L * L;
  block_copy(t, s.tau, L * L);
  if (init) {
    block_copy(y, s.tau, L * L);   // xi = tau of the initial QR
  } else {
    block_copy(x, s.xi, L * L);
    __syncthreads();
    small_matmul<false>(t, x, y, L);
  }
  __syncthreads();
  block_copy(s.xi, y, L * L);
  double acc = 0.0;
  for (int e = threadIdx.x; e < L * L; e += blockDim.x) acc += y[e].x * y[e].x + y[e].y * y[e].y;
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int i = 0; i < (int)blockDim.x; ++i) tot += red[i];
    st->err = sqrt(tot) / st->bnorm;
    if (!isfinite(st->err)) atomicCAS(&st->bad, 0, 2);
  }
}

// COCG: beta = (Q^T Q)^-1 (tau^T (Qn^T Qn)); Q^T Q <- Qn^T Qn   (bl_krylov.py:113-115)
__global__ void cocg_beta_kernel(SmallPtrs s, int L, SolverState* st) {
  extern __shared__ double2 sm[];
  double2* a = sm;
  double2* b = sm + L * L;
  double2* c = sm + 2 * L * L;
  __shared__ int piv[kMaxL];
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  block_copy(a, s.qq, L * L);
  block_copy(b, s.tau, L * L);
  block_copy(c, s.g2, L * L);
  __syncthreads();
  small_matmul<true>(b, c, s.tmp, L);   // tau^T (Qn^T Qn)
  block_copy(b, s.tmp, L * L);
  __syncthreads();
  lu_factor(a, L, piv, &bad);
  if (!bad) lu_solve(a, piv, L, b, L);
  block_copy(s.beta, b, L * L);
  block_copy(s.qq, c, L * L);
  __syncthreads();
  if (threadIdx.x == 0 && bad == 1) atomicExch(&st->bad, 1);
  if (threadIdx.x == 0 && bad == 2) atomicCAS(&st->bad, 0, 2);
}

// ---- host driver ----------------------------------------------------------------
template <typename T>
struct Ctx {
  const bdda_plan* plan;
  int L;
  int64_t n;         // rows = 3 N_occ
  const T* ghat;
  const int32_t* cell_map;
  T* field;
  T* vec[kVecs];
  T* diag;
  T* jpre;
  double2* partial;
  SmallPtrs sp;
  SolverState* st;
  cudaStream_t stream;
  size_t sm2, sm3;   // dynamic smem of the small kernels (2 or 3 L x L matrices)
  // complex128 vectors with complex64 products (the mixed form): the product
  // inside the iteration runs on these buffers; null = complex128 products
  const float2* ghat32 = nullptr;
  float2 *diag32 = nullptr, *jpre32 = nullptr;
  bool diverged = false;   // set when the complex64-product recursion blew up
  T* xbest = nullptr;      // mixed form: X at the smallest residual so far (or null)
  double best = INFINITY;  // that residual
  bool replaced = false;   // a residual replacement has happened
  double* hist_dev = nullptr;   // graph-driven loop: per-iteration residuals (kGraphHistCap)
  bool watch = false;      // apply the divergence test to complex128 products too
};

// The product in the vectors' own precision.
template <typename T>
static int mvp_exact(Ctx<T>& c, const T* in, T* out) {
  return block_mvp_impl<T>(c.plan, c.L, c.ghat, c.cell_map, c.diag, c.jpre, in, out, c.field, c.stream);
}

// The product inside the iteration: complex64 arithmetic when the context
// carries complex64 buffers; the input is rounded to complex64 as the Z pass
// gathers it and the output widened as the Z^-1 pass writes it.
template <typename T>
static int mvp(Ctx<T>& c, const T* in, T* out) {
  if constexpr (std::is_same<T, double2>::value) {
    if (c.ghat32)
      return block_mvp_wide(c.plan, c.L, c.ghat32, c.cell_map, c.diag32, c.jpre32, in, out,
                            reinterpret_cast<float2*>(c.field), c.stream);
  }
  return mvp_exact(c, in, out);
}

template <typename T>
static int gram2(Ctx<T>& c, bool conj, const T* A, const T* B0, const T* B1, double2* out) {
  GramArgs g;
  g.n = c.n; g.L = c.L; g.nB = B1 ? 2 : 1; g.A = A; g.B[0] = B0; g.B[1] = B1; g.partial = c.partial;
  return gram<T>(g, conj, out, c.stream);
}

template <typename T>
static int upd(Ctx<T>& c, T* out, const T* Y0, const double2* a0, const T* Y1, const double2* a1,
               const T* X1, const T* X2, const double2* c2, const double2* M, bool norm) {
  UpdateArgs u;
  u.n = c.n; u.L = c.L;
  u.Y0 = Y0; u.a0 = a0; u.Y1 = Y1; u.a1 = a1; u.X1 = X1; u.X2 = X2; u.c2 = c2; u.M = M;
  u.out = out;
  u.norm_partial = norm ? reinterpret_cast<double*>(c.partial) : nullptr;
  return update<T>(u, c.stream);
}

template <typename T>
static int read_state(Ctx<T>& c, double* err, int* bad) {
  SolverState h;
  BDDA_CUDA_TRY(cudaMemcpyAsync(&h, c.st, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
  BDDA_CUDA_TRY(cudaStreamSynchronize(c.stream));
  *err = h.err;
  *bad = h.bad;
  return BDDA_OK;
}

#define TRY(expr)                 \
  do {                            \
    int s_ = (expr);              \
    if (s_ != BDDA_OK) return s_; \
  } while (0)

// Residual replacement in the mixed form: when the recursive residual has
// dropped by this factor below its largest value since the last replacement
// (or below tol), it is recomputed from X with the complex128 product.
// Once the true residual is below g_mixed_switch * tol the remaining
// iterations use complex128 products: near tol the complex64 rounding of the
// products, not the Krylov space, limits the recursion (0 = never switch).
// Both set by bdda_tune_mixed.
static double g_replace_drop = 1e-1;
static double g_mixed_switch = 0.0;

double mixed_replace_drop() { return g_replace_drop; }
// ... and it is abandoned as diverged once the residual exceeds its smallest
// value so far by this factor (block-BiCGSTAB on strongly scattering
// particles can amplify the complex64 rounding of the products without bound;
// bdda_tune_mixed).  The fallback continues from the best X so far, so an
// early call costs little: on a sweep of 48 strongly scattering problems
// (m = 1.53) a factor of 10 took the mixed form from 11.3 to 16.2
// orientations/s (complex128: 17.1), against 1000 before.  In the first
// kEarlyHump iterations the reference is the first iteration's residual
// (below).
static double g_diverge_factor = 10.0;
constexpr int kEarlyHump = 8;
// ... and also abandoned once its smallest residual has not halved for
// kStallIters iterations: on strongly scattering particles the complex64
// recursion can stall between 1e-4 and 4e-4 without a 10-fold rise (two of
// the 144 sweep problems ran 500 iterations that way); the complex128
// fallback then continues from the best X.
constexpr int kStallIters = 60;

double mixed_diverge_factor() { return g_diverge_factor; }

// Block-BiCGSTAB (bl_krylov.py:121-187).  vec: 0 X, 1 R, 2 P, 3 R0, 4 V, 5 T, 6 Z, 7 Bj
template <typename T>
static int bicgstab_core(Ctx<T>& c, bool has_x0, double tol, int itermax, int* iter_fin,
                         double* err_fin, double* hist) {
  T *X = c.vec[0], *R = c.vec[1], *P = c.vec[2], *R0 = c.vec[3], *V = c.vec[4], *Tt = c.vec[5],
    *Z = c.vec[6], *Bj = c.vec[7];
  const int L = c.L;
  double* dot_partial = reinterpret_cast<double*>(c.partial) + 2 * (size_t)kMaxL * kMaxL * kRedBlocks;
  // R = M^-1 B and ||M^-1 B|| (bl_krylov.py:149-153)
  TRY(upd<T>(c, R, Bj, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, true));
  norm_kernel<<<1, 256, 0, c.stream>>>(reinterpret_cast<double*>(c.partial), kRedBlocks, c.st, 1);
  count_launch();
  BDDA_CUDA_TRY(cudaGetLastError());
  if (has_x0) {   // R = M^-1 (B - A X0), with the exact product
    TRY(mvp_exact<T>(c, X, V));
    TRY(upd<T>(c, R, Bj, nullptr, V, c.sp.r, nullptr, nullptr, nullptr, nullptr, false));
  }
  TRY(upd<T>(c, P, R, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, false));
  TRY(upd<T>(c, R0, R, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, false));
  *iter_fin = 0;
  *err_fin = INFINITY;
  double err = INFINITY;
  double rmax = 0.0;        // largest residual since the last replacement
  double rmin = INFINITY;   // smallest residual so far
  double rfirst = INFINITY; // residual after the first iteration
  double rstall = INFINITY; // residual at the last halving of the smallest one
  int kstall = 0;           // iteration of that halving
  for (int k = 0; k < itermax; ++k) {
    TRY(mvp<T>(c, P, V));                                   // V = M^-1 A P
    TRY(gram2<T>(c, true, R0, V, R, c.sp.g2));              // R0^H V, R0^H R
    bicg_alpha_kernel<<<1, 256, c.sm2, c.stream>>>(c.sp, L, c.st);
    count_launch();
    BDDA_CUDA_TRY(cudaGetLastError());
    TRY(upd<T>(c, Tt, R, nullptr, nullptr, nullptr, V, nullptr, nullptr, c.sp.negalpha, false));  // T = R - V alpha
    TRY(mvp<T>(c, Tt, Z));                                  // Z = M^-1 A T
    TRY(gram2<T>(c, true, R0, Z, nullptr, c.sp.g2));        // R0^H Z
    DotArgs d;
    d.n = c.n * L; d.A = Z; d.B = Tt; d.partial = dot_partial;
    TRY(dots<T>(d, c.stream));                              // tr(Z^H T), tr(Z^H Z)
    bicg_zeta_beta_kernel<<<1, 256, c.sm2, c.stream>>>(c.sp, L, dot_partial, kRedBlocks, c.st);
    count_launch();
    BDDA_CUDA_TRY(cudaGetLastError());
    TRY(upd<T>(c, X, X, nullptr, Tt, &c.st->zeta, P, nullptr, nullptr, c.sp.alpha, false));  // X += P alpha + zeta T
    TRY(upd<T>(c, R, Tt, nullptr, Z, &c.st->negzeta, nullptr, nullptr, nullptr, nullptr, true));  // R = T - zeta Z
    norm_kernel<<<1, 256, 0, c.stream>>>(reinterpret_cast<double*>(c.partial), kRedBlocks, c.st, 0);
    count_launch();
    BDDA_CUDA_TRY(cudaGetLastError());
    int bad = 0;
    TRY(read_state(c, &err, &bad));
    if (bad == 1) return BDDA_BREAKDOWN;
    if (bad != 2 && c.ghat32 && (err < tol || err < g_replace_drop * rmax || err < g_mixed_switch * tol)) {
      // complex64 products: replace the recursive residual by the true one
      // (complex128 product; Z is free until the next iteration), so the
      // drift of the recursion stays at the level of the current residual
      TRY(mvp_exact<T>(c, X, Z));
      TRY(upd<T>(c, R, Bj, nullptr, Z, c.sp.r, nullptr, nullptr, nullptr, nullptr, true));
      norm_kernel<<<1, 256, 0, c.stream>>>(reinterpret_cast<double*>(c.partial), kRedBlocks, c.st, 0);
      count_launch();
      BDDA_CUDA_TRY(cudaGetLastError());
      TRY(read_state(c, &err, &bad));
      rmax = err;
      // keep X for a warm fallback when its true residual is the smallest so far
      if (c.xbest && bad == 0 && err < c.best) {
        BDDA_CUDA_TRY(cudaMemcpyAsync(c.xbest, X, (size_t)c.n * L * sizeof(T), cudaMemcpyDeviceToDevice,
                                      c.stream));
        c.best = err;
      }
      c.replaced = true;
      if (err < g_mixed_switch * tol) c.ghat32 = nullptr;   // complex128 products from here on
    }
    // before the first replacement, X is kept at every new minimum of the
    // recursive residual (a divergence can come first); after it, only at
    // replacements, so the copies do not run every iteration
    if (c.xbest && c.ghat32 && !c.replaced && bad == 0 && err < c.best) {
      BDDA_CUDA_TRY(cudaMemcpyAsync(c.xbest, X, (size_t)c.n * L * sizeof(T), cudaMemcpyDeviceToDevice, c.stream));
      c.best = err;
    }
    rmax = err > rmax ? err : rmax;
    rmin = err < rmin ? err : rmin;
    if (k == 0) rfirst = err;
    if (err < 0.5 * rstall) {
      rstall = err;
      kstall = k;
    }
    if (hist) hist[k] = err;
    *iter_fin = k;
    *err_fin = err;
    if (bad == 2) return BDDA_NOT_CONVERGED;   // NaN/Inf reached: stop, reported as not converged
    if (err < tol) return BDDA_OK;
    // divergence: a rise by the factor above the smallest residual; during
    // the first kEarlyHump iterations before any replacement, above the first
    // iteration's residual instead, because block BiCGSTAB's early hump rises
    // well above its first minimum in exact arithmetic too (10.5-fold within
    // five iterations on the x=20 particle for one orientation set, in
    // complex128 as in the mixed form)
    const double ref = (c.replaced || k >= kEarlyHump) ? rmin : rfirst;
    if (((c.ghat32 || c.watch) && err > g_diverge_factor * ref) || (c.ghat32 && k - kstall >= kStallIters)) {
      c.diverged = true;
      return BDDA_NOT_CONVERGED;
    }
    // P = R + (P - zeta V) beta
    TRY(upd<T>(c, P, R, nullptr, nullptr, nullptr, P, V, &c.st->negzeta, c.sp.beta, false));
  }
  return BDDA_NOT_CONVERGED;
}

// Shifted CholeskyQR3: Q R = W with R accumulated into sp.tau; the first step
// adds 11 (n L + L (L+1)) u tr(W^H W) to the diagonal so that it cannot fail
// for numerically rank-deficient W.  Writes sa, sb; Q ends in sa.
template <typename T>
static int cholqr3(Ctx<T>& c, const T* W, T* sa, T* sb, T** qout) {
  const double u = 1.1102230246251565e-16;
  const double shift = 11.0 * ((double)c.n * c.L + (double)c.L * (c.L + 1)) * u;
  const T* in = W;
  T* outs[3] = {sa, sb, sa};
  for (int step = 0; step < 3; ++step) {
    TRY(gram2<T>(c, true, in, in, nullptr, c.sp.g2));
    cholqr_step_kernel<<<1, 256, c.sm2, c.stream>>>(c.sp, c.L, step == 0, step == 0 ? shift : 0.0, c.st);
    count_launch();
    BDDA_CUDA_TRY(cudaGetLastError());
    TRY(upd<T>(c, outs[step], nullptr, nullptr, nullptr, nullptr, in, nullptr, nullptr, c.sp.rinv, false));
    in = outs[step];
  }
  *qout = outs[2];
  return BDDA_OK;
}

// Block-COCG-rq (bl_krylov.py:58-118).  vec: 0 X, 1-2-3 rotating Q / QR scratch,
// 4 S, 5 AS, 6 W, 7 Bj
template <typename T>
static int cocg_core(Ctx<T>& c, bool has_x0, double tol, int itermax, int* iter_fin, double* err_fin,
                     double* hist) {
  T *X = c.vec[0], *S = c.vec[4], *AS = c.vec[5], *W = c.vec[6], *Bj = c.vec[7];
  T* rot[3] = {c.vec[1], c.vec[2], c.vec[3]};   // rot[0] holds Q, rot[1..2] are QR scratch
  const int L = c.L;
  // ||M^-1 B|| (bl_krylov.py:87-88); W = M^-1 (B - A X0)
  TRY(upd<T>(c, W, Bj, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, true));
  norm_kernel<<<1, 256, 0, c.stream>>>(reinterpret_cast<double*>(c.partial), kRedBlocks, c.st, 1);
  count_launch();
  BDDA_CUDA_TRY(cudaGetLastError());
  if (has_x0) {
    TRY(mvp_exact<T>(c, X, AS));
    TRY(upd<T>(c, W, Bj, nullptr, AS, c.sp.r, nullptr, nullptr, nullptr, nullptr, false));
  }
  // Q, xi = qr(W)   (bl_krylov.py:92)
  T* q = nullptr;
  TRY(cholqr3<T>(c, W, rot[1], rot[2], &q));
  std::swap(rot[0], rot[1]);               // Q now in rot[0]
  cocg_xi_kernel<<<1, 256, c.sm3, c.stream>>>(c.sp, L, c.st, 1);
  count_launch();
  BDDA_CUDA_TRY(cudaGetLastError());
  TRY(upd<T>(c, S, rot[0], nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, false));
  TRY(gram2<T>(c, false, rot[0], rot[0], nullptr, c.sp.qq));
  *iter_fin = 0;
  *err_fin = INFINITY;
  double err = INFINITY;
  for (int k = 0; k < itermax; ++k) {
    TRY(mvp<T>(c, S, AS));
    TRY(gram2<T>(c, false, S, AS, nullptr, c.sp.g2));
    cocg_alpha_kernel<<<1, 256, c.sm3, c.stream>>>(c.sp, L, c.st);
    count_launch();
    BDDA_CUDA_TRY(cudaGetLastError());
    TRY(upd<T>(c, X, X, nullptr, nullptr, nullptr, S, nullptr, nullptr, c.sp.alphaxi, false));
    TRY(upd<T>(c, W, rot[0], nullptr, nullptr, nullptr, AS, nullptr, nullptr, c.sp.negalpha, false));
    TRY(cholqr3<T>(c, W, rot[1], rot[2], &q));   // Qnew in rot[1], tau in sp.tau
    cocg_xi_kernel<<<1, 256, c.sm3, c.stream>>>(c.sp, L, c.st, 0);
    count_launch();
    BDDA_CUDA_TRY(cudaGetLastError());
    int bad = 0;
    TRY(read_state(c, &err, &bad));
    if (bad == 1) return BDDA_BREAKDOWN;
    if (hist) hist[k] = err;
    *iter_fin = k;
    *err_fin = err;
    if (bad == 2) return BDDA_NOT_CONVERGED;
    if (err < tol) return BDDA_OK;
    TRY(gram2<T>(c, false, rot[1], rot[1], nullptr, c.sp.g2));
    cocg_beta_kernel<<<1, 256, c.sm3, c.stream>>>(c.sp, L, c.st);
    count_launch();
    BDDA_CUDA_TRY(cudaGetLastError());
    TRY(upd<T>(c, S, rot[1], nullptr, nullptr, nullptr, S, nullptr, nullptr, c.sp.beta, false));
    std::swap(rot[0], rot[1]);             // Q <- Qnew
  }
  return BDDA_NOT_CONVERGED;
}

// ---- graph-driven iteration loop ---------------------------------------------------
// The test point of one iteration on the device: record the residual, count
// the iteration, and keep looping while err >= tol, no breakdown or
// non-finite value, and iterations remain.  The loop condition is the graph's
// while-node handle; the counter bounds the loop by itermax whatever happens.
__global__ void loop_check_kernel(SolverState* st, double tol, int itermax, double* hist,
                                  cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int k = st->iter;
  const double err = st->err;
  if (k < kGraphHistCap) hist[k] = err;
  st->iter = k + 1;
  const bool go = st->bad == 0 && !(err < tol) && k + 1 < itermax;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// Non-blocking stream per device for capturing the loop bodies (the caller's
// stream may be the legacy default stream, which cannot be captured).
static cudaStream_t capture_stream() {
  static std::mutex mu;
  static cudaStream_t streams[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!streams[dev] && cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking) != cudaSuccess)
    streams[dev] = nullptr;
  return streams[dev];
}

// Graph-driven loop: one while node whose body is `body(cc, h)` captured on a
// private stream (cc = c with that stream), then one launch on c.stream and
// one read-back.  Returns BDDA_OK / BREAKDOWN / NOT_CONVERGED like the
// host-driven cores; any failure while building the graph returns
// BDDA_CUDA_ERROR before anything ran (the caller then runs the host loop).
template <typename T, typename Body>
static int graph_loop(Ctx<T>& c, double tol, int itermax, int* iter_fin, double* err_fin, double* hist,
                      Body body) {
  cudaStream_t cs = capture_stream();
  if (!cs) return BDDA_CUDA_ERROR;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ex = nullptr;
  cudaGraphConditionalHandle h;
  int status = BDDA_CUDA_ERROR;
  long long n0 = 0, nbody = 0;
  do {
    if (cudaGraphCreate(&g, 0) != cudaSuccess) break;
    if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) break;
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphAddNode(&node, g, nullptr, 0, &np) != cudaSuccess) break;
    cudaGraph_t bodyg = np.conditional.phGraph_out[0];
    Ctx<T> cc = c;
    cc.stream = cs;
    if (cudaStreamBeginCaptureToGraph(cs, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess)
      break;
    n0 = bdda_launch_count();
    const int sb = body(cc, h);
    cudaGraph_t captured = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(cs, &captured);
    nbody = bdda_launch_count() - n0;
    if (sb != BDDA_OK || ec != cudaSuccess) break;
    if (cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) break;
    status = BDDA_OK;
  } while (false);
  if (status != BDDA_OK) {
    cudaGetLastError();
    if (ex) cudaGraphExecDestroy(ex);
    if (g) cudaGraphDestroy(g);
    return BDDA_CUDA_ERROR;
  }
  const cudaError_t el = cudaGraphLaunch(ex, c.stream);
  SolverState hs;
  const cudaError_t ec = el == cudaSuccess ? cudaMemcpyAsync(&hs, c.st, sizeof(hs), cudaMemcpyDeviceToHost, c.stream)
                                           : el;
  const cudaError_t es = ec == cudaSuccess ? cudaStreamSynchronize(c.stream) : ec;
  cudaGraphExecDestroy(ex);
  cudaGraphDestroy(g);
  if (es != cudaSuccess) return BDDA_CUDA_ERROR;
  const int ran = hs.iter < 1 ? 1 : (hs.iter > itermax ? itermax : hs.iter);
  count_launch((int)(nbody * (ran - 1)));   // the body was counted once, at capture
  if (hist) {
    const int nh = ran < kGraphHistCap ? ran : kGraphHistCap;
    BDDA_CUDA_TRY(cudaMemcpy(hist, c.hist_dev, nh * sizeof(double), cudaMemcpyDeviceToHost));
  }
  if (hs.bad == 1) return BDDA_BREAKDOWN;
  *iter_fin = ran - 1;
  *err_fin = hs.err;
  if (hs.bad == 2) return BDDA_NOT_CONVERGED;
  return hs.err < tol ? BDDA_OK : BDDA_NOT_CONVERGED;
}

// Block-BiCGSTAB with the graph-driven loop (plain forms, no complex64 products
// inside complex128 vectors).  Same kernels and order as bicgstab_core.
template <typename T>
static int bicgstab_graph(Ctx<T>& c, bool has_x0, double tol, int itermax, int* iter_fin, double* err_fin,
                          double* hist) {
  T *X = c.vec[0], *R = c.vec[1], *P = c.vec[2], *R0 = c.vec[3], *V = c.vec[4], *Tt = c.vec[5],
    *Z = c.vec[6], *Bj = c.vec[7];
  const int L = c.L;
  double* dot_partial = reinterpret_cast<double*>(c.partial) + 2 * (size_t)kMaxL * kMaxL * kRedBlocks;
  TRY(upd<T>(c, R, Bj, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, true));
  norm_kernel<<<1, 256, 0, c.stream>>>(reinterpret_cast<double*>(c.partial), kRedBlocks, c.st, 1);
  count_launch();
  BDDA_CUDA_TRY(cudaGetLastError());
  if (has_x0) {
    TRY(mvp_exact<T>(c, X, V));
    TRY(upd<T>(c, R, Bj, nullptr, V, c.sp.r, nullptr, nullptr, nullptr, nullptr, false));
  }
  TRY(upd<T>(c, P, R, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, false));
  TRY(upd<T>(c, R0, R, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, false));
  *iter_fin = 0;
  *err_fin = INFINITY;
  return graph_loop<T>(c, tol, itermax, iter_fin, err_fin, hist, [&](Ctx<T>& cc, cudaGraphConditionalHandle h) -> int {
    TRY(mvp<T>(cc, P, V));
    TRY(gram2<T>(cc, true, R0, V, R, cc.sp.g2));
    bicg_alpha_kernel<<<1, 256, cc.sm2, cc.stream>>>(cc.sp, L, cc.st);
    count_launch();
    TRY(upd<T>(cc, Tt, R, nullptr, nullptr, nullptr, V, nullptr, nullptr, cc.sp.negalpha, false));
    TRY(mvp<T>(cc, Tt, Z));
    TRY(gram2<T>(cc, true, R0, Z, nullptr, cc.sp.g2));
    DotArgs d;
    d.n = cc.n * L; d.A = Z; d.B = Tt; d.partial = dot_partial;
    TRY(dots<T>(d, cc.stream));
    bicg_zeta_beta_kernel<<<1, 256, cc.sm2, cc.stream>>>(cc.sp, L, dot_partial, kRedBlocks, cc.st);
    count_launch();
    TRY(upd<T>(cc, X, X, nullptr, Tt, &cc.st->zeta, P, nullptr, nullptr, cc.sp.alpha, false));
    TRY(upd<T>(cc, R, Tt, nullptr, Z, &cc.st->negzeta, nullptr, nullptr, nullptr, nullptr, true));
    norm_kernel<<<1, 256, 0, cc.stream>>>(reinterpret_cast<double*>(cc.partial), kRedBlocks, cc.st, 0);
    loop_check_kernel<<<1, 32, 0, cc.stream>>>(cc.st, tol, itermax, cc.hist_dev, h);
    count_launch(2);
    TRY(upd<T>(cc, P, R, nullptr, nullptr, nullptr, P, V, &cc.st->negzeta, cc.sp.beta, false));
    return cudaGetLastError() == cudaSuccess ? BDDA_OK : BDDA_CUDA_ERROR;
  });
}

// Block-COCG-rq with the graph-driven loop.  The host loop swaps the roles of
// two QR buffers every iteration; a captured body has fixed buffers, so the
// new Q is copied into place instead (one vector copy per iteration, small at
// the sizes this loop runs).
template <typename T>
static int cocg_graph(Ctx<T>& c, bool has_x0, double tol, int itermax, int* iter_fin, double* err_fin,
                      double* hist) {
  T *X = c.vec[0], *S = c.vec[4], *AS = c.vec[5], *W = c.vec[6], *Bj = c.vec[7];
  T *Q = c.vec[1], *Q2 = c.vec[2], *Q3 = c.vec[3];
  const int L = c.L;
  TRY(upd<T>(c, W, Bj, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, true));
  norm_kernel<<<1, 256, 0, c.stream>>>(reinterpret_cast<double*>(c.partial), kRedBlocks, c.st, 1);
  count_launch();
  BDDA_CUDA_TRY(cudaGetLastError());
  if (has_x0) {
    TRY(mvp_exact<T>(c, X, AS));
    TRY(upd<T>(c, W, Bj, nullptr, AS, c.sp.r, nullptr, nullptr, nullptr, nullptr, false));
  }
  T* q = nullptr;
  TRY(cholqr3<T>(c, W, Q2, Q3, &q));   // Q in Q2
  BDDA_CUDA_TRY(cudaMemcpyAsync(Q, Q2, (size_t)c.n * L * sizeof(T), cudaMemcpyDeviceToDevice, c.stream));
  cocg_xi_kernel<<<1, 256, c.sm3, c.stream>>>(c.sp, L, c.st, 1);
  count_launch();
  BDDA_CUDA_TRY(cudaGetLastError());
  TRY(upd<T>(c, S, Q, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, false));
  TRY(gram2<T>(c, false, Q, Q, nullptr, c.sp.qq));
  *iter_fin = 0;
  *err_fin = INFINITY;
  return graph_loop<T>(c, tol, itermax, iter_fin, err_fin, hist, [&](Ctx<T>& cc, cudaGraphConditionalHandle h) -> int {
    TRY(mvp<T>(cc, S, AS));
    TRY(gram2<T>(cc, false, S, AS, nullptr, cc.sp.g2));
    cocg_alpha_kernel<<<1, 256, cc.sm3, cc.stream>>>(cc.sp, L, cc.st);
    count_launch();
    TRY(upd<T>(cc, X, X, nullptr, nullptr, nullptr, S, nullptr, nullptr, cc.sp.alphaxi, false));
    TRY(upd<T>(cc, W, Q, nullptr, nullptr, nullptr, AS, nullptr, nullptr, cc.sp.negalpha, false));
    T* qn = nullptr;
    TRY(cholqr3<T>(cc, W, Q2, Q3, &qn));   // Qnew in Q2, tau in sp.tau
    cocg_xi_kernel<<<1, 256, cc.sm3, cc.stream>>>(cc.sp, L, cc.st, 0);
    loop_check_kernel<<<1, 32, 0, cc.stream>>>(cc.st, tol, itermax, cc.hist_dev, h);
    count_launch(2);
    TRY(gram2<T>(cc, false, Q2, Q2, nullptr, cc.sp.g2));
    cocg_beta_kernel<<<1, 256, cc.sm3, cc.stream>>>(cc.sp, L, cc.st);
    count_launch();
    TRY(upd<T>(cc, S, Q2, nullptr, nullptr, nullptr, S, nullptr, nullptr, cc.sp.beta, false));
    if (cudaMemcpyAsync(Q, Q2, (size_t)cc.n * L * sizeof(T), cudaMemcpyDeviceToDevice, cc.stream) != cudaSuccess)
      return BDDA_CUDA_ERROR;
    return cudaGetLastError() == cudaSuccess ? BDDA_OK : BDDA_CUDA_ERROR;
  });
}

// The host-driven loops are used when the graph-driven one is off
// (bdda_tune_solver_graphs), the problem is large, the history would not fit,
// or profiling records per-pass events.
static int g_solver_graphs = 1;

__global__ void constants_kernel(SmallPtrs s) {
  if (threadIdx.x == 0) s.r[0] = make_double2(-1.0, 0.0);
}

template <typename K>
static int allow_smem(K kern, size_t bytes) {
  BDDA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return BDDA_OK;
}

// Epilogue of the fused entry point: X widened into Xout and the observables
// accumulated in the same pass; a solve that did not converge reports zero
// observables (P = E = 0).
template <typename T>
static int dda_epilogue(const DdaPhys& ph, const T* X, double2* Xout, bool converged, cudaStream_t st) {
  const int L = ph.L;
  dda_epilogue_kernel<T><<<kDdaObsBlocks, dda_epilogue_threads(L), dda_epilogue_smem(L), st>>>(ph, X, Xout,
                                                                                               nullptr);
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch();
  if (converged) {
    observables_finalize_kernel<<<(L + 63) / 64, 64, 0, st>>>(ph.partial, kDdaObsBlocks, L, ph.k, ph.absorbing,
                                                               ph.obs);
    BDDA_CUDA_TRY(cudaGetLastError());
    count_launch();
  } else {
    BDDA_CUDA_TRY(cudaMemsetAsync(ph.obs, 0, (size_t)L * 12 * sizeof(double), st));
  }
  return BDDA_OK;
}

// phys (nullable): the fused DDA entry point; the right-hand side and diagonal
// come from the physics (diag and B unused) and the epilogue adds the observables.
template <typename T>
static int run_solver(int solver, const bdda_plan* p, int L, int n_occ, const void* ghat,
                      const int32_t* cell_map, const double2* diag, const double2* B, const double2* X0,
                      double tol, int itermax, double2* Xout, int* iter_fin, double* err_fin,
                      double* hist, void* work, size_t work_bytes, cudaStream_t st,
                      const DdaPhys* phys = nullptr) {
  const int prec = std::is_same<T, double2>::value ? BDDA_C128 : BDDA_C64;
  const Layout o = layout(p, prec, L, n_occ);
  if (work_bytes < o.total) return BDDA_NO_WORKSPACE;
  unsigned char* w = static_cast<unsigned char*>(work);
  Ctx<T> c;
  c.plan = p;
  c.L = L;
  c.n = 3 * (int64_t)n_occ;
  c.ghat = static_cast<const T*>(ghat);
  c.cell_map = cell_map;
  c.field = reinterpret_cast<T*>(w + o.field);
  for (int v = 0; v < kVecs; ++v) c.vec[v] = reinterpret_cast<T*>(w + o.vec[v]);
  c.diag = reinterpret_cast<T*>(w + o.diag);
  c.jpre = reinterpret_cast<T*>(w + o.jpre);
  c.partial = reinterpret_cast<double2*>(w + o.partial);
  c.sp = small_ptrs(w + o.small);
  c.st = reinterpret_cast<SolverState*>(w + o.state);
  c.hist_dev = reinterpret_cast<double*>(w + o.hist);
  c.stream = st;
  c.sm2 = (size_t)2 * L * L * sizeof(double2);
  c.sm3 = (size_t)3 * L * L * sizeof(double2);
  TRY(allow_smem(bicg_alpha_kernel, c.sm2));
  TRY(allow_smem(bicg_zeta_beta_kernel, c.sm2));
  TRY(allow_smem(cholqr_step_kernel, c.sm2));
  TRY(allow_smem(cocg_alpha_kernel, c.sm3));
  TRY(allow_smem(cocg_xi_kernel, c.sm3));
  TRY(allow_smem(cocg_beta_kernel, c.sm3));
  BDDA_CUDA_TRY(cudaMemsetAsync(c.st, 0, sizeof(SolverState), st));
  constants_kernel<<<1, 32, 0, st>>>(c.sp);
  count_launch();
  if (phys) {
    dda_prologue_kernel<T, false><<<kRedBlocks, 256, 0, st>>>(*phys, c.diag, c.jpre, c.vec[7], nullptr, nullptr);
  } else {
    prepare_kernel<T><<<kRedBlocks, 256, 0, st>>>(diag, B, c.n, L, c.diag, c.jpre, c.vec[7]);
  }
  count_launch();
  BDDA_CUDA_TRY(cudaGetLastError());
  if (X0) {
    convert_in_kernel<T><<<kRedBlocks, 256, 0, st>>>(X0, c.vec[0], c.n * L);
    count_launch();
    BDDA_CUDA_TRY(cudaGetLastError());
  } else {
    BDDA_CUDA_TRY(cudaMemsetAsync(c.vec[0], 0, (size_t)c.n * L * sizeof(T), st));
  }
  const bool graph = g_solver_graphs && !profiling() && itermax <= kGraphHistCap &&
                     (double)grid_points(p) * L <= kGraphMaxWork;
  int status = BDDA_CUDA_ERROR;
  if (graph) {
    status = solver == BDDA_COCG_RQ ? cocg_graph<T>(c, X0 != nullptr, tol, itermax, iter_fin, err_fin, hist)
                                    : bicgstab_graph<T>(c, X0 != nullptr, tol, itermax, iter_fin, err_fin, hist);
  }
  if (status == BDDA_CUDA_ERROR && graph) {   // the graph could not be built: start over on the host loop
    BDDA_CUDA_TRY(cudaMemsetAsync(c.st, 0, sizeof(SolverState), st));
    if (X0) {
      convert_in_kernel<T><<<kRedBlocks, 256, 0, st>>>(X0, c.vec[0], c.n * L);
      count_launch();
      BDDA_CUDA_TRY(cudaGetLastError());
    } else {
      BDDA_CUDA_TRY(cudaMemsetAsync(c.vec[0], 0, (size_t)c.n * L * sizeof(T), st));
    }
  }
  if (!graph || status == BDDA_CUDA_ERROR)
    status = solver == BDDA_COCG_RQ ? cocg_core<T>(c, X0 != nullptr, tol, itermax, iter_fin, err_fin, hist)
                                    : bicgstab_core<T>(c, X0 != nullptr, tol, itermax, iter_fin, err_fin, hist);
  if (status == BDDA_OK || status == BDDA_NOT_CONVERGED) {
    if (phys) {
      TRY(dda_epilogue<T>(*phys, c.vec[0], Xout, status == BDDA_OK, st));
    } else {
      convert_out_kernel<T><<<kRedBlocks, 256, 0, st>>>(c.vec[0], Xout, c.n * L);
      count_launch();
      BDDA_CUDA_TRY(cudaGetLastError());
    }
  }
  return status;
}

// ---- FP32 Krylov with FP64 iterative refinement -----------------------------------
// Outer loop in complex128: r = M^-1 (B - A X) with the FP64 product; inner
// block solve of M^-1 A D = r in complex64 (FP32 product and vectors, FP64
// Gram / small solves); X += D in FP64.  Stops when the true relative
// residual ||r|| / ||M^-1 B|| < tol.
struct RLayout {
  size_t field, v64[4], diag64, jpre64, v32[kVecs], diag32, jpre32, partial, small, st64, st32, total;
};

static RLayout rlayout(const bdda_plan* p, int L, int n_occ) {
  RLayout o;
  const size_t v64 = (size_t)3 * n_occ * L * 16, v32 = (size_t)3 * n_occ * L * 8;
  size_t off = 0;
  o.field = off; off = al(off + bdda_mvp_workspace_bytes(p, BDDA_C128, L));   // shared by both precisions
  for (int v = 0; v < 4; ++v) { o.v64[v] = off; off = al(off + v64); }
  o.diag64 = off; off = al(off + (size_t)3 * n_occ * 16);
  o.jpre64 = off; off = al(off + (size_t)3 * n_occ * 16);
  for (int v = 0; v < kVecs; ++v) { o.v32[v] = off; off = al(off + v32); }
  o.diag32 = off; off = al(off + (size_t)3 * n_occ * 8);
  o.jpre32 = off; off = al(off + (size_t)3 * n_occ * 8);
  o.partial = off; off = al(off + (size_t)kRedBlocks * 2 * kMaxL * kMaxL * sizeof(double2));
  o.small = off; off = al(off + (size_t)kSmallMats * kMaxL * kMaxL * sizeof(double2) + 64 * sizeof(int));
  o.st64 = off; off = al(off + sizeof(SolverState));
  o.st32 = off; off = al(off + sizeof(SolverState));
  o.total = off;
  return o;
}

__global__ void accumulate_kernel(double2* X, const float2* D, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 d = D[i];
    X[i] = make_double2(X[i].x + (double)d.x, X[i].y + (double)d.y);
  }
}

__global__ void negate_accumulate_kernel(double2* X, const float2* D, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 d = D[i];
    X[i] = make_double2(X[i].x - (double)d.x, X[i].y - (double)d.y);
  }
}

template <typename T>
static void fill_ctx(Ctx<T>& c, const bdda_plan* p, int L, int n_occ, const void* ghat, const int32_t* cell_map,
                     unsigned char* w, size_t field, size_t diag, size_t jpre, const size_t* vecs, int nvec,
                     size_t partial, size_t small, size_t state, cudaStream_t st) {
  c.plan = p;
  c.L = L;
  c.n = 3 * (int64_t)n_occ;
  c.ghat = static_cast<const T*>(ghat);
  c.cell_map = cell_map;
  c.field = reinterpret_cast<T*>(w + field);
  for (int v = 0; v < kVecs; ++v) c.vec[v] = v < nvec ? reinterpret_cast<T*>(w + vecs[v]) : nullptr;
  c.diag = reinterpret_cast<T*>(w + diag);
  c.jpre = reinterpret_cast<T*>(w + jpre);
  c.partial = reinterpret_cast<double2*>(w + partial);
  c.sp = small_ptrs(w + small);
  c.st = reinterpret_cast<SolverState*>(w + state);
  c.stream = st;
  c.sm2 = (size_t)2 * L * L * sizeof(double2);
  c.sm3 = (size_t)3 * L * L * sizeof(double2);
}

// Block-BiCGSTAB in complex64 with FP64 reliable updates (residual
// replacement, van der Vorst & Ye): the Krylov vectors and products are FP32,
// the solution X is accumulated in FP64 (X += P alpha + zeta T, the increment
// formed in FP32), and whenever the recursive residual has dropped by the
// factor kReplace since the last replacement -- and before declaring convergence --
// R is replaced by the true residual M^-1 (B - A X) from the FP64 product.
// The Krylov space is kept, so nothing is lost to restarts; convergence is
// judged on the true residual.
static int bicgstab_reliable(Ctx<double2>& c64, Ctx<float2>& c32, bool has_x0, double tol, int itermax,
                             double kReplace, int* iter_fin, double* err_fin, double* hist) {
  double2 *Bj = c64.vec[0], *X = c64.vec[1], *R64 = c64.vec[2], *Tm = c64.vec[3];
  float2 *U = c32.vec[0], *R = c32.vec[1], *P = c32.vec[2], *R0 = c32.vec[3], *V = c32.vec[4],
         *Tt = c32.vec[5], *Z = c32.vec[6];
  const int L = c32.L;
  const int64_t ne = c64.n * L;
  const cudaStream_t st = c64.stream;
  double* dot_partial = reinterpret_cast<double*>(c32.partial) + 2 * (size_t)kMaxL * kMaxL * kRedBlocks;
  // true residual into R64 / R (and its norm into c64.st)
  auto replace = [&](double* err) -> int {
    TRY(mvp<double2>(c64, X, Tm));
    TRY(upd<double2>(c64, R64, Bj, nullptr, Tm, c64.sp.r, nullptr, nullptr, nullptr, nullptr, true));
    norm_kernel<<<1, 256, 0, st>>>(reinterpret_cast<double*>(c64.partial), kRedBlocks, c64.st, 0);
    convert_in_kernel<float2><<<kRedBlocks, 256, 0, st>>>(R64, R, ne);
    count_launch(2);
    int bad = 0;
    TRY(read_state(c64, err, &bad));
    return bad == 2 ? BDDA_NOT_CONVERGED : BDDA_OK;
  };
  TRY(upd<double2>(c64, Tm, Bj, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, true));
  norm_kernel<<<1, 256, 0, st>>>(reinterpret_cast<double*>(c64.partial), kRedBlocks, c64.st, 1);
  count_launch();
  double err = INFINITY;
  if (has_x0) {
    if (replace(&err) != BDDA_OK) return BDDA_NOT_CONVERGED;
  } else {
    BDDA_CUDA_TRY(cudaMemsetAsync(X, 0, (size_t)ne * sizeof(double2), st));
    convert_in_kernel<float2><<<kRedBlocks, 256, 0, st>>>(Bj, R, ne);
    count_launch();
    err = 1.0;
  }
  // the FP32 recursion runs on the residual scaled to the state's norm
  TRY(upd<float2>(c32, P, R, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, true));
  norm_kernel<<<1, 256, 0, st>>>(reinterpret_cast<double*>(c32.partial), kRedBlocks, c32.st, 1);
  count_launch();
  TRY(upd<float2>(c32, R0, R, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, false));
  double last = err;           // true residual at the last replacement (relative to ||M^-1 B||)
  const double base = err;     // ||R|| at the start of the FP32 recursion, relative to ||M^-1 B||
  *iter_fin = 0;
  *err_fin = err;
  if (err < tol) return BDDA_OK;
  double scale = base;         // recursion residual (relative to its start) -> relative to ||M^-1 B||
  for (int k = 0; k < itermax; ++k) {
    TRY(mvp<float2>(c32, P, V));
    TRY(gram2<float2>(c32, true, R0, V, R, c32.sp.g2));
    bicg_alpha_kernel<<<1, 256, c32.sm2, st>>>(c32.sp, L, c32.st);
    count_launch();
    TRY(upd<float2>(c32, Tt, R, nullptr, nullptr, nullptr, V, nullptr, nullptr, c32.sp.negalpha, false));
    TRY(mvp<float2>(c32, Tt, Z));
    TRY(gram2<float2>(c32, true, R0, Z, nullptr, c32.sp.g2));
    DotArgs d;
    d.n = c32.n * L; d.A = Z; d.B = Tt; d.partial = dot_partial;
    TRY(dots<float2>(d, st));
    bicg_zeta_beta_kernel<<<1, 256, c32.sm2, st>>>(c32.sp, L, dot_partial, kRedBlocks, c32.st);
    count_launch();
    // X += P alpha + zeta T: increment in FP32, accumulation in FP64
    TRY(upd<float2>(c32, U, nullptr, nullptr, Tt, &c32.st->zeta, P, nullptr, nullptr, c32.sp.alpha, false));
    accumulate_kernel<<<kRedBlocks, 256, 0, st>>>(X, U, ne);
    count_launch();
    TRY(upd<float2>(c32, R, Tt, nullptr, Z, &c32.st->negzeta, nullptr, nullptr, nullptr, nullptr, true));
    norm_kernel<<<1, 256, 0, st>>>(reinterpret_cast<double*>(c32.partial), kRedBlocks, c32.st, 0);
    count_launch();
    double rr = INFINITY;
    int bad = 0;
    TRY(read_state(c32, &rr, &bad));
    if (bad == 1) return BDDA_BREAKDOWN;
    err = rr * scale;
    *iter_fin = k;
    if (hist) hist[k] = err;
    if (bad == 2) { *err_fin = err; return BDDA_NOT_CONVERGED; }
    if (err < tol || err < kReplace * last) {
      double tr = INFINITY;
      if (replace(&tr) != BDDA_OK) { *err_fin = tr; return BDDA_NOT_CONVERGED; }
      last = tr;
      err = tr;
      if (hist) hist[k] = err;
      // the recursion continues from the true residual: rescale its norm bookkeeping
      TRY(upd<float2>(c32, Tt, R, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, true));
      norm_kernel<<<1, 256, 0, st>>>(reinterpret_cast<double*>(c32.partial), kRedBlocks, c32.st, 1);
      count_launch();
      scale = tr;
      if (tr < tol) { *err_fin = tr; return BDDA_OK; }
    }
    *err_fin = err;
    TRY(upd<float2>(c32, P, R, nullptr, nullptr, nullptr, P, V, &c32.st->negzeta, c32.sp.beta, false));
  }
  // report the true residual of the returned X
  double tr = INFINITY;
  if (replace(&tr) == BDDA_OK) *err_fin = tr;
  return *err_fin < tol ? BDDA_OK : BDDA_NOT_CONVERGED;
}

static int run_refine(int solver, bool restart, const bdda_plan* p, int L, int n_occ, const void* ghat64,
                      const void* ghat32, const int32_t* cell_map, const double2* diag, const double2* B,
                      const double2* X0, double tol, int itermax, double inner_tol, int max_outer, double2* Xout,
                      int* iter_fin, double* err_fin, double* hist, void* work, size_t work_bytes,
                      cudaStream_t st) {
  const RLayout o = rlayout(p, L, n_occ);
  if (work_bytes < o.total) return BDDA_NO_WORKSPACE;
  unsigned char* w = static_cast<unsigned char*>(work);
  Ctx<double2> c64;
  Ctx<float2> c32;
  fill_ctx(c64, p, L, n_occ, ghat64, cell_map, w, o.field, o.diag64, o.jpre64, o.v64, 4, o.partial, o.small,
           o.st64, st);
  fill_ctx(c32, p, L, n_occ, ghat32, cell_map, w, o.field, o.diag32, o.jpre32, o.v32, kVecs, o.partial,
           o.small, o.st32, st);
  TRY(allow_smem(bicg_alpha_kernel, c32.sm2));
  TRY(allow_smem(bicg_zeta_beta_kernel, c32.sm2));
  TRY(allow_smem(cholqr_step_kernel, c32.sm2));
  TRY(allow_smem(cocg_alpha_kernel, c32.sm3));
  TRY(allow_smem(cocg_xi_kernel, c32.sm3));
  TRY(allow_smem(cocg_beta_kernel, c32.sm3));
  double2 *Bj = c64.vec[0], *X = c64.vec[1], *R = c64.vec[2], *Tm = c64.vec[3];
  const int64_t ne = c64.n * L;
  BDDA_CUDA_TRY(cudaMemsetAsync(c64.st, 0, sizeof(SolverState), st));
  BDDA_CUDA_TRY(cudaMemsetAsync(c32.st, 0, sizeof(SolverState), st));
  constants_kernel<<<1, 32, 0, st>>>(c64.sp);
  count_launch();
  prepare_kernel<double2><<<kRedBlocks, 256, 0, st>>>(diag, B, c64.n, L, c64.diag, c64.jpre, Bj);
  prepare_kernel<float2><<<kRedBlocks, 256, 0, st>>>(diag, B, c32.n, L, c32.diag, c32.jpre, c32.vec[7]);
  count_launch(2);
  BDDA_CUDA_TRY(cudaGetLastError());
  if (solver == BDDA_BICGSTAB && max_outer >= 0 && inner_tol > 0.0 && !restart) {
    if (X0) BDDA_CUDA_TRY(cudaMemcpyAsync(X, X0, (size_t)ne * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    const int s2 = bicgstab_reliable(c64, c32, X0 != nullptr, tol, itermax, fmin(inner_tol, 0.5), iter_fin, err_fin, hist);
    if (s2 == BDDA_OK || s2 == BDDA_NOT_CONVERGED)
      BDDA_CUDA_TRY(cudaMemcpyAsync(Xout, X, (size_t)ne * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    return s2;
  }
  // ||M^-1 B||, and the first true residual
  TRY(upd<double2>(c64, Tm, Bj, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, true));
  norm_kernel<<<1, 256, 0, st>>>(reinterpret_cast<double*>(c64.partial), kRedBlocks, c64.st, 1);
  count_launch();
  if (X0) {
    BDDA_CUDA_TRY(cudaMemcpyAsync(X, X0, (size_t)ne * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    TRY(mvp<double2>(c64, X, Tm));
    TRY(upd<double2>(c64, R, Bj, nullptr, Tm, c64.sp.r, nullptr, nullptr, nullptr, nullptr, true));
  } else {
    BDDA_CUDA_TRY(cudaMemsetAsync(X, 0, (size_t)ne * sizeof(double2), st));
    TRY(upd<double2>(c64, R, Bj, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, true));
  }
  norm_kernel<<<1, 256, 0, st>>>(reinterpret_cast<double*>(c64.partial), kRedBlocks, c64.st, 0);
  count_launch();
  double err = INFINITY;
  int bad = 0;
  TRY(read_state(c64, &err, &bad));
  int total = 0;
  *iter_fin = 0;
  *err_fin = err;
  int status = BDDA_NOT_CONVERGED;
  for (int outer = 0; outer < max_outer; ++outer) {
    if (bad == 2 || !(err == err)) { status = BDDA_NOT_CONVERGED; break; }
    if (err < tol) { status = BDDA_OK; break; }
    if (total >= itermax) break;
    // inner FP32 solve of M^-1 A D = r to a relative tolerance
    double tol_in = fmax(inner_tol, 0.3 * tol / err);
    tol_in = fmin(tol_in, 0.5);
    convert_in_kernel<float2><<<kRedBlocks, 256, 0, st>>>(R, c32.vec[7], ne);
    count_launch();
    BDDA_CUDA_TRY(cudaMemsetAsync(c32.vec[0], 0, (size_t)ne * sizeof(float2), st));
    BDDA_CUDA_TRY(cudaMemsetAsync(c32.st, 0, sizeof(SolverState), st));
    int it_in = 0;
    double err_in = INFINITY;
    const int s_in = solver == BDDA_COCG_RQ
                         ? cocg_core<float2>(c32, false, tol_in, itermax - total, &it_in, &err_in, hist ? hist + total : nullptr)
                         : bicgstab_core<float2>(c32, false, tol_in, itermax - total, &it_in, &err_in, hist ? hist + total : nullptr);
    if (s_in == BDDA_BREAKDOWN) return BDDA_BREAKDOWN;
    if (s_in != BDDA_OK && s_in != BDDA_NOT_CONVERGED) return s_in;
    const int ran = it_in + 1;
    if (hist)
      for (int i = 0; i < ran; ++i) hist[total + i] *= err;   // relative to ||M^-1 B||
    total += ran;
    *iter_fin = total - 1;
    if (!(err_in == err_in)) { status = BDDA_NOT_CONVERGED; break; }
    // X += D; r = M^-1 B - M^-1 A X in FP64
    accumulate_kernel<<<kRedBlocks, 256, 0, st>>>(X, c32.vec[0], ne);
    count_launch();
    TRY(mvp<double2>(c64, X, Tm));
    TRY(upd<double2>(c64, R, Bj, nullptr, Tm, c64.sp.r, nullptr, nullptr, nullptr, nullptr, true));
    norm_kernel<<<1, 256, 0, st>>>(reinterpret_cast<double*>(c64.partial), kRedBlocks, c64.st, 0);
    count_launch();
    const double prev = err;
    TRY(read_state(c64, &err, &bad));
    if (!(err < prev)) {   // the correction made things worse (FP32 solve past its accuracy): undo it
      const double2 m1 = make_double2(-1.0, 0.0);
      (void)m1;
      negate_accumulate_kernel<<<kRedBlocks, 256, 0, st>>>(X, c32.vec[0], ne);
      count_launch();
      TRY(mvp<double2>(c64, X, Tm));
      TRY(upd<double2>(c64, R, Bj, nullptr, Tm, c64.sp.r, nullptr, nullptr, nullptr, nullptr, true));
      norm_kernel<<<1, 256, 0, st>>>(reinterpret_cast<double*>(c64.partial), kRedBlocks, c64.st, 0);
      count_launch();
      TRY(read_state(c64, &err, &bad));
      *err_fin = err;
      status = BDDA_NOT_CONVERGED;
      break;
    }
    *err_fin = err;
    if (err < tol) { status = BDDA_OK; break; }
    if (!(err < 0.9 * prev)) { status = BDDA_NOT_CONVERGED; break; }   // refinement stalled
  }
  BDDA_CUDA_TRY(cudaMemcpyAsync(Xout, X, (size_t)ne * sizeof(double2), cudaMemcpyDeviceToDevice, st));
  return status;
}

// ---- complex128 Krylov with complex64 products ------------------------------------
// The block solver keeps X, the residual and every Krylov vector, Gram
// product and L x L step in complex128 and computes the products inside the
// iteration in complex64 (the product dominates the cost).  BiCGSTAB replaces
// its recursive residual by the true one (complex128 product) whenever it
// has dropped 10-fold (bdda_tune_mixed) and before it stops.  Under 1e-7
// perturbations of B, a 100-fold interval let the drift of the recursion
// swing the iteration count of the x=20 particle between 20 and 62
// (complex128: 19) and of a strongly scattering x=9.2 one between 111 and
// 138 (complex128: 86-90); a 10-fold one keeps them at 19-22 and 106-120.
// COCG-rq runs its recursion to
// kInnerFrac * tol.  Then the true residual M^-1 (B - A X) decides; if it is
// not below tol the solver restarts from the current X (warm start).  A
// BiCGSTAB recursion that diverges under the complex64 products is abandoned
// and the problem solved on with complex128 products, warm-started from the X
// of the smallest residual (kept in xbest: at each new minimum until the first
// residual replacement, then at replacements) when that is below the zero
// start's.
constexpr double kInnerFrac = 0.5;

struct MLayout {
  Layout base;
  size_t diag32, jpre32, xbest, total;
};

static MLayout mlayout(const bdda_plan* p, int L, int n_occ) {
  MLayout o;
  o.base = layout(p, BDDA_C128, L, n_occ);
  size_t off = o.base.total;
  o.diag32 = off; off = al(off + (size_t)3 * n_occ * 8);
  o.jpre32 = off; off = al(off + (size_t)3 * n_occ * 8);
  o.xbest = off; off = al(off + (size_t)3 * n_occ * L * 16);
  o.total = off;
  return o;
}

static int run_mixed(int solver, const bdda_plan* p, int L, int n_occ, const void* ghat64, const void* ghat32,
                     const int32_t* cell_map, const double2* diag, const double2* B, const double2* X0, double tol,
                     int itermax, int max_outer, double2* Xout, int* iter_fin, double* err_fin, double* hist,
                     void* work, size_t work_bytes, cudaStream_t st, const DdaPhys* phys = nullptr) {
  const MLayout o = mlayout(p, L, n_occ);
  if (work_bytes < o.total) return BDDA_NO_WORKSPACE;
  unsigned char* w = static_cast<unsigned char*>(work);
  Ctx<double2> c;
  fill_ctx(c, p, L, n_occ, ghat64, cell_map, w, o.base.field, o.base.diag, o.base.jpre, o.base.vec, kVecs,
           o.base.partial, o.base.small, o.base.state, st);
  TRY(allow_smem(bicg_alpha_kernel, c.sm2));
  TRY(allow_smem(bicg_zeta_beta_kernel, c.sm2));
  TRY(allow_smem(cholqr_step_kernel, c.sm2));
  TRY(allow_smem(cocg_alpha_kernel, c.sm3));
  TRY(allow_smem(cocg_xi_kernel, c.sm3));
  TRY(allow_smem(cocg_beta_kernel, c.sm3));
  float2* diag32 = reinterpret_cast<float2*>(w + o.diag32);
  float2* jpre32 = reinterpret_cast<float2*>(w + o.jpre32);
  const int64_t ne = c.n * L;
  // vec: 0 X, 1 R, 4 V, 7 Bj (the solver cores' roles)
  double2 *X = c.vec[0], *R = c.vec[1], *V = c.vec[4], *Bj = c.vec[7];
  if (solver == BDDA_BICGSTAB) c.xbest = reinterpret_cast<double2*>(w + o.xbest);
  BDDA_CUDA_TRY(cudaMemsetAsync(c.st, 0, sizeof(SolverState), st));
  constants_kernel<<<1, 32, 0, st>>>(c.sp);
  if (phys) {
    dda_prologue_kernel<double2, true><<<kRedBlocks, 256, 0, st>>>(*phys, c.diag, c.jpre, Bj, diag32, jpre32);
    count_launch(2);
  } else {
    prepare_kernel<double2><<<kRedBlocks, 256, 0, st>>>(diag, B, c.n, L, c.diag, c.jpre, Bj);
    prepare_kernel<float2><<<kRedBlocks, 256, 0, st>>>(diag, B, c.n, L, diag32, jpre32, nullptr);
    count_launch(3);
  }
  BDDA_CUDA_TRY(cudaGetLastError());
  if (X0) BDDA_CUDA_TRY(cudaMemcpyAsync(X, X0, (size_t)ne * sizeof(double2), cudaMemcpyDeviceToDevice, st));
  else BDDA_CUDA_TRY(cudaMemsetAsync(X, 0, (size_t)ne * sizeof(double2), st));
  int total = 0;
  *iter_fin = 0;
  *err_fin = INFINITY;
  int status = BDDA_NOT_CONVERGED;
  double prev = INFINITY;
  for (int round = 0; round < max_outer && total < itermax; ++round) {
    c.ghat32 = static_cast<const float2*>(ghat32);
    c.diag32 = diag32;
    c.jpre32 = jpre32;
    int it_in = 0;
    double err_in = INFINITY;
    const bool warm = round > 0 || X0 != nullptr;
    // BiCGSTAB judges convergence on a replaced (true) residual; COCG-rq's
    // residual is implicit, so its recursion runs to kInnerFrac * tol
    const int s_in = solver == BDDA_COCG_RQ
                         ? cocg_core<double2>(c, warm, kInnerFrac * tol, itermax - total, &it_in, &err_in,
                                              hist ? hist + total : nullptr)
                         : bicgstab_core<double2>(c, warm, tol, itermax - total, &it_in, &err_in,
                                                  hist ? hist + total : nullptr);
    if (s_in != BDDA_OK && s_in != BDDA_NOT_CONVERGED) return s_in;
    total += it_in + 1;
    *iter_fin = total - 1;
    if (c.diverged) {   // give up the complex64 products
      c.diverged = false;
      c.ghat32 = nullptr;
      // complex128 from the best X so far when the recursion got below the
      // zero start's residual, watched by the same divergence test: block
      // BiCGSTAB restarted from a residual whose columns sit at very
      // different levels can stagnate (a 24 x 28 x 35 GRE did for 480
      // iterations where a zero start converges in 10); then once more
      // from the start, unwatched
      bool warm = c.best < 1.0;
      while (total < itermax) {
        if (warm) {
          BDDA_CUDA_TRY(cudaMemcpyAsync(X, c.xbest, (size_t)ne * sizeof(double2), cudaMemcpyDeviceToDevice, st));
        } else if (X0) {
          BDDA_CUDA_TRY(cudaMemcpyAsync(X, X0, (size_t)ne * sizeof(double2), cudaMemcpyDeviceToDevice, st));
        } else {
          BDDA_CUDA_TRY(cudaMemsetAsync(X, 0, (size_t)ne * sizeof(double2), st));
        }
        c.watch = warm;
        const int s64 = bicgstab_core<double2>(c, warm || X0 != nullptr, tol, itermax - total, &it_in, &err_in,
                                               hist ? hist + total : nullptr);
        c.watch = false;
        if (s64 != BDDA_OK && s64 != BDDA_NOT_CONVERGED) return s64;
        total += it_in + 1;
        *iter_fin = total - 1;
        if (!(warm && c.diverged)) break;
        c.diverged = false;
        warm = false;
      }
      max_outer = round + 1;   // this is the last round
    } else if (solver == BDDA_BICGSTAB && s_in == BDDA_OK) {
      // BiCGSTAB stopped on a replaced residual: it is the true residual already
      *err_fin = err_in;
      status = BDDA_OK;
      break;
    }
    // true residual with the complex128 product
    c.ghat32 = nullptr;
    TRY(mvp_exact<double2>(c, X, V));
    TRY(upd<double2>(c, R, Bj, nullptr, V, c.sp.r, nullptr, nullptr, nullptr, nullptr, true));
    norm_kernel<<<1, 256, 0, st>>>(reinterpret_cast<double*>(c.partial), kRedBlocks, c.st, 0);
    count_launch();
    double err = INFINITY;
    int bad = 0;
    TRY(read_state(c, &err, &bad));
    *err_fin = err;
    if (bad == 2 || !(err == err)) break;
    if (err < tol) { status = BDDA_OK; break; }
    if (!(err < 0.9 * prev)) break;   // restarts no longer gain
    prev = err;
  }
  if (phys) {
    TRY(dda_epilogue<double2>(*phys, X, Xout, status == BDDA_OK, st));
  } else {
    BDDA_CUDA_TRY(cudaMemcpyAsync(Xout, X, (size_t)ne * sizeof(double2), cudaMemcpyDeviceToDevice, st));
  }
  return status;
}

}  // namespace bdda

using namespace bdda;

extern "C" {

size_t bdda_solver_workspace_bytes(const bdda_plan* p, int solver, int prec, int L, int n_occ) {
  if (!p || L < 1 || L > kMaxL || n_occ < 1 || (solver != BDDA_BICGSTAB && solver != BDDA_COCG_RQ) ||
      (prec != BDDA_C128 && prec != BDDA_C64))
    return 0;
  return layout(p, prec, L, n_occ).total;
}

// A solve whose pass kernels gave up waiting for a tile copy left pencils
// unwritten: its result is not trusted (BDDA_TIMEOUT), whatever it converged to.
static int wait_status(const bdda_plan* p, int status, cudaStream_t st) {
  if (status == BDDA_BAD_ARG || status == BDDA_NO_WORKSPACE || status == BDDA_CUDA_ERROR) return status;
  unsigned int n = 0;
  if (cudaMemcpyAsync(&n, plan_err(p), sizeof(n), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return BDDA_CUDA_ERROR;
  return n ? BDDA_TIMEOUT : status;
}

int bdda_solve(const bdda_plan* p, int solver, int prec, int L, int n_occ, const void* ghat,
               const int32_t* cell_map, const void* diag, const void* B, const void* X0, double tol,
               int itermax, void* X, int* iter_fin, double* err_fin, double* history, void* work,
               size_t work_bytes, void* stream) {
  if (!p || L < 1 || L > kMaxL || n_occ < 1 || !ghat || !cell_map || !diag || !B || !X || !iter_fin ||
      !err_fin || itermax < 0 || !(tol == tol))
    return BDDA_BAD_ARG;
  if (solver != BDDA_BICGSTAB && solver != BDDA_COCG_RQ) return BDDA_BAD_ARG;
  if (!work || !p->dev_tables) return BDDA_NO_WORKSPACE;
  *iter_fin = 0;
  *err_fin = INFINITY;
  if (itermax == 0) {   // the reference returns X = 0 without iterating
    BDDA_CUDA_TRY(cudaMemsetAsync(X, 0, (size_t)3 * n_occ * L * sizeof(double2), (cudaStream_t)stream));
    return BDDA_NOT_CONVERGED;
  }
  const cudaStream_t st = (cudaStream_t)stream;
  if (prec == BDDA_C128)
    return wait_status(p,
                       run_solver<double2>(solver, p, L, n_occ, ghat, cell_map, static_cast<const double2*>(diag),
                                           static_cast<const double2*>(B), static_cast<const double2*>(X0), tol,
                                           itermax, static_cast<double2*>(X), iter_fin, err_fin, history, work,
                                           work_bytes, st),
                       st);
  if (prec == BDDA_C64)
    return wait_status(p,
                       run_solver<float2>(solver, p, L, n_occ, ghat, cell_map, static_cast<const double2*>(diag),
                                          static_cast<const double2*>(B), static_cast<const double2*>(X0), tol,
                                          itermax, static_cast<double2*>(X), iter_fin, err_fin, history, work,
                                          work_bytes, st),
                       st);
  return BDDA_BAD_ARG;
}

int bdda_bicgstab(const bdda_plan* p, int prec, int L, int n_occ, const void* ghat,
                  const int32_t* cell_map, const void* diag, const void* B, const void* X0, double tol,
                  int itermax, void* X, int* iter_fin, double* err_fin, double* history, void* work,
                  size_t work_bytes, void* stream) {
  return bdda_solve(p, BDDA_BICGSTAB, prec, L, n_occ, ghat, cell_map, diag, B, X0, tol, itermax, X,
                    iter_fin, err_fin, history, work, work_bytes, stream);
}

int bdda_cocg_rq(const bdda_plan* p, int prec, int L, int n_occ, const void* ghat,
                 const int32_t* cell_map, const void* diag, const void* B, const void* X0, double tol,
                 int itermax, void* X, int* iter_fin, double* err_fin, double* history, void* work,
                 size_t work_bytes, void* stream) {
  return bdda_solve(p, BDDA_COCG_RQ, prec, L, n_occ, ghat, cell_map, diag, B, X0, tol, itermax, X,
                    iter_fin, err_fin, history, work, work_bytes, stream);
}

size_t bdda_refine_workspace_bytes(const bdda_plan* p, int L, int n_occ) {
  if (!p || L < 1 || L > kMaxL || n_occ < 1) return 0;
  return rlayout(p, L, n_occ).total;
}

int bdda_refine_solve(const bdda_plan* p, int solver, int L, int n_occ, const void* ghat_c128,
                      const void* ghat_c64, const int32_t* cell_map, const void* diag, const void* B,
                      const void* X0, double tol, int itermax, double inner_tol, int max_outer, void* X,
                      int* iter_fin, double* err_fin, double* history, void* work, size_t work_bytes,
                      void* stream) {
  if (!p || L < 1 || L > kMaxL || n_occ < 1 || !ghat_c128 || !ghat_c64 || !cell_map || !diag || !B || !X ||
      !iter_fin || !err_fin || itermax < 0 || max_outer == 0 || !(tol == tol) || !(inner_tol > 0.0))
    return BDDA_BAD_ARG;
  if (solver != BDDA_BICGSTAB && solver != BDDA_COCG_RQ) return BDDA_BAD_ARG;
  if (!work || !p->dev_tables) return BDDA_NO_WORKSPACE;
  *iter_fin = 0;
  *err_fin = INFINITY;
  if (itermax == 0) {
    BDDA_CUDA_TRY(cudaMemsetAsync(X, 0, (size_t)3 * n_occ * L * sizeof(double2), (cudaStream_t)stream));
    return BDDA_NOT_CONVERGED;
  }
  // max_outer > 0: restarted refinement; max_outer < 0 with BiCGSTAB: one FP32
  // recursion with FP64 reliable updates (replacement factor inner_tol)
  const bool restart = solver == BDDA_COCG_RQ || max_outer > 0;
  if (max_outer < 0) max_outer = -max_outer;
  return wait_status(p,
                     run_refine(solver, restart, p, L, n_occ, ghat_c128, ghat_c64, cell_map,
                                static_cast<const double2*>(diag), static_cast<const double2*>(B),
                                static_cast<const double2*>(X0), tol, itermax, inner_tol, max_outer,
                                static_cast<double2*>(X), iter_fin, err_fin, history, work, work_bytes,
                                (cudaStream_t)stream),
                     (cudaStream_t)stream);
}

int bdda_tune_solver_graphs(int on) {
  if (on != 0 && on != 1) return BDDA_BAD_ARG;
  g_solver_graphs = on;
  return BDDA_OK;
}

int bdda_tune_mixed(double replace_drop, double switch_ratio, double diverge_factor) {
  if (!(replace_drop > 0.0 && replace_drop < 1.0) || !(switch_ratio >= 0.0) || !(diverge_factor > 1.0))
    return BDDA_BAD_ARG;
  g_replace_drop = replace_drop;
  g_mixed_switch = switch_ratio;
  g_diverge_factor = diverge_factor;
  return BDDA_OK;
}

int bdda_tune_mixed_get(double* replace_drop, double* switch_ratio, double* diverge_factor) {
  if (!replace_drop || !switch_ratio || !diverge_factor) return BDDA_BAD_ARG;
  *replace_drop = g_replace_drop;
  *switch_ratio = g_mixed_switch;
  *diverge_factor = g_diverge_factor;
  return BDDA_OK;
}

size_t bdda_mixed_workspace_bytes(const bdda_plan* p, int L, int n_occ) {
  if (!p || L < 1 || L > kMaxL || n_occ < 1) return 0;
  return mlayout(p, L, n_occ).total;
}

int bdda_mixed_solve(const bdda_plan* p, int solver, int L, int n_occ, const void* ghat_c128, const void* ghat_c64,
                     const int32_t* cell_map, const void* diag, const void* B, const void* X0, double tol,
                     int itermax, int max_outer, void* X, int* iter_fin, double* err_fin, double* history,
                     void* work, size_t work_bytes, void* stream) {
  if (!p || L < 1 || L > kMaxL || n_occ < 1 || !ghat_c128 || !ghat_c64 || !cell_map || !diag || !B || !X ||
      !iter_fin || !err_fin || itermax < 0 || !(tol > 0.0) || max_outer < 1 ||
      (solver != BDDA_BICGSTAB && solver != BDDA_COCG_RQ))
    return BDDA_BAD_ARG;
  if (!p->dev_tables || !work) return BDDA_NO_WORKSPACE;
  return wait_status(p,
                     run_mixed(solver, p, L, n_occ, ghat_c128, ghat_c64, cell_map, static_cast<const double2*>(diag),
                               static_cast<const double2*>(B), static_cast<const double2*>(X0), tol, itermax,
                               max_outer, static_cast<double2*>(X), iter_fin, err_fin, history, work, work_bytes,
                               static_cast<cudaStream_t>(stream)),
                     static_cast<cudaStream_t>(stream));
}

size_t bdda_dda_workspace_bytes(const bdda_plan* p, int mode, int L, int n_occ) {
  if (!p || L < 1 || L > kMaxL || n_occ < 1) return 0;
  size_t base;
  if (mode == BDDA_BATCH_MIXED) base = mlayout(p, L, n_occ).total;
  else if (mode == BDDA_BATCH_C128 || mode == BDDA_BATCH_C64) base = layout(p, mode, L, n_occ).total;
  else return 0;
  return al(base) + al((size_t)kDdaObsBlocks * L * 10 * sizeof(double));
}

int bdda_dda_solve(const bdda_plan* p, const bdda_dda_problem* prob, int solver, int mode, const void* ghat_c128,
                   const void* ghat_c64, const int32_t* cell_map, const void* X0, double tol, int itermax,
                   int max_outer, void* X, void* diag_out, void* eper_out, double* obs, int* iter_fin,
                   double* err_fin, double* history, void* work, size_t work_bytes, void* stream) {
  if (!p || !prob || prob->L < 1 || prob->L > kMaxL || prob->n_occ < 1 || !prob->pos || !prob->vec || !prob->e0 ||
      !(prob->lf > 0.0) || !(prob->m_m > 0.0) || !cell_map || !X || !obs || !iter_fin || !err_fin ||
      itermax < 0 || !(tol == tol) || (solver != BDDA_BICGSTAB && solver != BDDA_COCG_RQ))
    return BDDA_BAD_ARG;
  if (mode != BDDA_BATCH_C128 && mode != BDDA_BATCH_C64 && mode != BDDA_BATCH_MIXED) return BDDA_BAD_ARG;
  if ((mode != BDDA_BATCH_C64 && !ghat_c128) || (mode != BDDA_BATCH_C128 && !ghat_c64)) return BDDA_BAD_ARG;
  if (mode == BDDA_BATCH_MIXED && (max_outer < 1 || !(tol > 0.0))) return BDDA_BAD_ARG;
  const int L = prob->L, n_occ = prob->n_occ;
  const size_t need = bdda_dda_workspace_bytes(p, mode, L, n_occ);
  if (!work || !p->dev_tables || work_bytes < need) return BDDA_NO_WORKSPACE;
  const size_t base = need - al((size_t)kDdaObsBlocks * L * 10 * sizeof(double));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  DdaPhys ph;
  memset(&ph, 0, sizeof(ph));
  ph.n_occ = n_occ; ph.L = L;
  for (int c = 0; c < 3; ++c) ph.mp[c] = make_double2(prob->m_p_xyz[2 * c], prob->m_p_xyz[2 * c + 1]);
  ph.m_m = prob->m_m; ph.lf = prob->lf; ph.k = prob->k; ph.absorbing = prob->absorbing;
  ph.pos = prob->pos; ph.vec = prob->vec; ph.e0 = static_cast<const double2*>(prob->e0);
  ph.diag_out = static_cast<double2*>(diag_out);
  ph.eper_out = static_cast<double2*>(eper_out);
  ph.obs = obs;
  ph.partial = reinterpret_cast<double*>(static_cast<unsigned char*>(work) + base);
  *iter_fin = 0;
  *err_fin = INFINITY;
  double2* Xd = static_cast<double2*>(X);
  const double2* X0d = static_cast<const double2*>(X0);
  if (itermax == 0) {   // the reference returns X = 0 without iterating; the set-up outputs are still made
    unsigned char* w = static_cast<unsigned char*>(work);
    if (mode == BDDA_BATCH_C64) {
      const Layout o = layout(p, BDDA_C64, L, n_occ);
      dda_prologue_kernel<float2, false><<<kRedBlocks, 256, 0, st>>>(
          ph, reinterpret_cast<float2*>(w + o.diag), reinterpret_cast<float2*>(w + o.jpre),
          reinterpret_cast<float2*>(w + o.vec[7]), nullptr, nullptr);
    } else {   // the complex128 layout (also the base of the mixed one)
      const Layout o = layout(p, BDDA_C128, L, n_occ);
      dda_prologue_kernel<double2, false><<<kRedBlocks, 256, 0, st>>>(
          ph, reinterpret_cast<double2*>(w + o.diag), reinterpret_cast<double2*>(w + o.jpre),
          reinterpret_cast<double2*>(w + o.vec[7]), nullptr, nullptr);
    }
    count_launch();
    BDDA_CUDA_TRY(cudaGetLastError());
    BDDA_CUDA_TRY(cudaMemsetAsync(X, 0, (size_t)3 * n_occ * L * sizeof(double2), st));
    BDDA_CUDA_TRY(cudaMemsetAsync(obs, 0, (size_t)L * 12 * sizeof(double), st));
    return BDDA_NOT_CONVERGED;
  }
  int status;
  if (mode == BDDA_BATCH_MIXED)
    status = run_mixed(solver, p, L, n_occ, ghat_c128, ghat_c64, cell_map, nullptr, nullptr, X0d, tol, itermax,
                       max_outer, Xd, iter_fin, err_fin, history, work, base, st, &ph);
  else if (mode == BDDA_BATCH_C128)
    status = run_solver<double2>(solver, p, L, n_occ, ghat_c128, cell_map, nullptr, nullptr, X0d, tol, itermax, Xd,
                                 iter_fin, err_fin, history, work, base, st, &ph);
  else
    status = run_solver<float2>(solver, p, L, n_occ, ghat_c64, cell_map, nullptr, nullptr, X0d, tol, itermax, Xd,
                                iter_fin, err_fin, history, work, base, st, &ph);
  return wait_status(p, status, st);
}

}  // extern "C"
