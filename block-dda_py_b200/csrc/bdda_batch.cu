// Batched block-BiCGSTAB: many independent problems -- particles,
// wavelengths, orientation blocks, each with its own grid, Green's spectrum,
// occupancy map and right-hand sides -- advanced together, one iteration at
// a time (the reference solves them one after another, bl_krylov.py:121-187
// called once per problem from scatterer.py:169-171 / run_dda.py:56-65).
//
// Each step of an iteration is ONE launch for the whole batch.  A one-CTA
// kernel rebuilds, at the start of every iteration, a work list of the
// problems still iterating (device flags) with the prefix sums of their work
// items per step kind; persistent CTAs (SMs x resident CTAs) then walk
// (problem, item) pairs from that list.  Converged problems drop out of the
// list, so they cost nothing, and no host decision is needed per iteration:
// each problem's convergence test runs on the device.  The iteration is
// captured once as a CUDA graph and replayed; the host reads one counter
// (problems still iterating) every kCheckEvery replays.
//
// Modes: complex128; complex64; and the mixed form of bdda_mixed_solve
// (complex128 vectors, Gram products and L x L steps, complex64 products
// inside the iteration, the residual replaced by the complex128 true residual
// M^-1 (B - A X) after every 10-fold drop (bdda_tune_mixed) and before stopping, warm
// restarts while the true residual is above tol).
//
// The pencil passes use the generic run-time-radix kernel body (problems
// have different radix sequences); the Gram, update and dot kernels use the
// L-specialised bodies, so L is one of 8, 16, 32, 64.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "bdda_blas_dev.cuh"
#include "bdda_internal.h"
#include "bdda_pencil.cuh"
#include "bdda_steps.cuh"

namespace bdda {
namespace {

constexpr int kMaxBatch = 1024;   // problems per call (one CTA builds the work list)
constexpr int kNCls = 6;          // work-item classes: the 5 pencil passes, then block kernels
constexpr int kClsBlas = 5;
constexpr int kCheckEvery = 4;    // iterations between host reads of the active count
constexpr int kRowsPerBlasItem = 512;
constexpr size_t kPencilBudget = 80 * 1024;

// ---- device work list -------------------------------------------------------
struct ListDev {
  int nprob;
  int* act;              // [nprob] ids of the listed problems, ascending
  int64_t* start;        // [kNCls][nprob + 1] item prefix over act
  const int64_t* cnt;    // [kNCls][nprob] items per problem and class
  int64_t* total;        // [kNCls]
  int* ctl;              // [0] listed  [1] k of this iteration  [2] next k  [3] still iterating
};

// Inclusive block scan (Hillis-Steele) of one int64 per thread.
__device__ int64_t block_scan(int64_t v, int64_t* sh) {
  const int t = threadIdx.x;
  sh[t] = v;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {
    const int64_t x = t >= o ? sh[t - o] : 0;
    __syncthreads();
    sh[t] += x;
    __syncthreads();
  }
  const int64_t r = sh[t];
  __syncthreads();
  return r;
}

// Lists the problems whose flag is set.  advance: this starts an iteration
// (k = next k, next k + 1); set_left: the "still iterating" count restarts
// at the number listed.
__global__ void __launch_bounds__(kMaxBatch) list_kernel(ListDev l, const int* flags, int advance, int set_left) {
  __shared__ int64_t sh[kMaxBatch];
  __shared__ int64_t last;
  const int t = threadIdx.x;
  const int on = (t < l.nprob && flags[t]) ? 1 : 0;
  const int64_t incl = block_scan(on, sh);
  const int pos = (int)(incl - on);
  if (t == (int)blockDim.x - 1) last = incl;
  __syncthreads();
  const int nact = (int)last;
  if (on) l.act[pos] = t;
  for (int c = 0; c < kNCls; ++c) {
    const int64_t v = on ? l.cnt[(int64_t)c * l.nprob + t] : 0;
    const int64_t inc = block_scan(v, sh);
    int64_t* st = l.start + (int64_t)c * (l.nprob + 1);
    if (on) st[pos] = inc - v;
    if (t == (int)blockDim.x - 1) {
      st[nact] = inc;
      l.total[c] = inc;
    }
  }
  if (t == 0) {
    l.ctl[0] = nact;
    if (advance) {
      l.ctl[1] = l.ctl[2];
      l.ctl[2] = l.ctl[2] + 1;
    }
    if (set_left) l.ctl[3] = nact;
  }
}

// Largest k in [lo, n) with st[k] <= item (st ascending, st[lo] <= item).
__device__ __forceinline__ int list_search(const int64_t* st, int lo, int n, int64_t item) {
  int hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (st[mid] <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Copies one problem's argument struct into shared memory (all threads).
template <typename A>
__device__ __forceinline__ void load_args(A* dst, const A* src) {
  static_assert(sizeof(A) % 4 == 0, "argument structs are word-sized");
  const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
  uint32_t* d = reinterpret_cast<uint32_t*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(A) / 4); i += blockDim.x) d[i] = s[i];
}

// Walks this CTA's items of class cls (grid-stride, so every CTA sees every
// problem and uneven problems balance).  Items arrive in increasing order, so
// the CTA keeps a cursor into the list: it searches only when an item leaves
// the current problem, and reloads the problem's arguments (into sargs) only
// then.  body(p, bid) runs with all threads.
template <typename ArgT, typename F>
__device__ __forceinline__ void for_items(const ListDev& l, int cls, const ArgT* args, ArgT* sargs, F&& body) {
  __shared__ int s_k, s_p, s_changed;
  __shared__ int64_t s_base, s_end;
  const int64_t total = l.total[cls];
  const int n = l.ctl[0];
  const int64_t* st = l.start + (int64_t)cls * (l.nprob + 1);
  if (threadIdx.x == 0) {
    s_k = 0;
    s_p = -1;
    s_end = -1;   // forces the first search
  }
  __syncthreads();
  for (int64_t item = blockIdx.x; item < total; item += gridDim.x) {
    if (threadIdx.x == 0) {
      s_changed = 0;
      if (item >= s_end) {
        const int k = list_search(st, s_end < 0 ? 0 : s_k, n, item);
        s_k = k;
        s_base = st[k];
        s_end = st[k + 1];
        const int p = l.act[k];
        s_changed = p != s_p;
        s_p = p;
      }
    }
    __syncthreads();
    if (s_changed && args) load_args(sargs, args + s_p);
    __syncthreads();
    body(s_p, item - s_base);
    __syncthreads();
  }
}

// ---- per-problem device descriptor -----------------------------------------------
struct ProbDev {
  SmallPtrs sp;          // working-precision solve
  SolverState* st;
  double* dotp;          // [nblk][3]
  double* nrmp;          // [nblk]
  SolverState* st64;     // mixed form: the complex128 true residual
  double* nrmp64;
  int nblk;              // block-kernel items (split of the rows)
  int pad;
};

// ---- persistent batched kernels --------------------------------------------------
template <typename T, int KIND, int LT>
__global__ void __launch_bounds__(256) batch_pencil_kernel(const PassArgs* args, ListDev l, int cls) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ __align__(16) PassArgs sa;
  for_items(l, cls, args, &sa, [&](int, int64_t bid) { generic_pencil<T, KIND, LT>(sa, bid, smraw); });
}

template <typename T, bool CONJ, int L, int NB>
__global__ void __launch_bounds__(256) batch_gram_kernel(const GramArgs* args, const ProbDev* pd, ListDev l) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ __align__(16) GramArgs sg;
  for_items(l, kClsBlas, args, &sg,
            [&](int p, int64_t bid) { gram_fixed_body<T, CONJ, L, NB>(sg, bid, pd[p].nblk, smraw); });
}

// out = sum of the problem's partials, into its sp.g2 (grid: width tiles x nprob)
__global__ void batch_gram_reduce_kernel(const GramArgs* args, const ProbDev* pd, const int* flags, int width) {
  const int p = blockIdx.y;
  if (!flags[p]) return;
  gram_reduce_body(args[p].partial, pd[p].nblk, width, pd[p].sp.g2, blockIdx.x * blockDim.x + threadIdx.x);
}

template <typename T, typename A, int L>
__global__ void __launch_bounds__(256) batch_update_kernel(const UpdateArgs* args, const ProbDev* pd, ListDev l,
                                                            int skip_first) {
  if (skip_first && l.ctl[1] == 0) return;   // first iteration: P = R already
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ __align__(16) UpdateArgs su;
  for_items(l, kClsBlas, args, &su,
            [&](int p, int64_t bid) { update_fixed_body<T, A, L>(su, bid, pd[p].nblk, smraw); });
}

template <typename T>
__global__ void __launch_bounds__(256) batch_dots_kernel(const DotArgs* args, const ProbDev* pd, ListDev l) {
  __shared__ __align__(16) DotArgs sd;
  for_items(l, kClsBlas, args, &sd, [&](int p, int64_t bid) { dots_body<T>(sd, bid, pd[p].nblk); });
}

// Elementwise steps over one problem's n values.
enum ElemOp { E_CONVERT_IN = 0, E_ZERO = 3, E_CONVERT_OUT = 4, E_PREPARE = 5 };
struct ElemArgs {
  int64_t n;        // values (rows x L; E_PREPARE: rows)
  int L;
  int pad;
  void* a;          // E_CONVERT_IN / E_ZERO: T out; E_CONVERT_OUT: double2 out
  const void* b;    // E_CONVERT_IN: double2 in (null: zero); E_CONVERT_OUT: T in
  // E_PREPARE: a = Bj (T), b = B (double2), c = diag (double2), d = diagT, e = jpreT
  const void* c;
  void* d;
  void* e;
};

template <typename T>
__device__ __forceinline__ void elem_body(const ElemArgs& e, int op, int64_t bid, int64_t nblk) {
  const int64_t stride = nblk * blockDim.x;
  const int64_t i0 = bid * blockDim.x + threadIdx.x;
  if (op == E_PREPARE) {   // jpre = 1/diag, Bj = B jpre (bl_krylov.py:146-149)
    const int64_t nv = e.n * e.L;
    for (int64_t i = i0; i < nv; i += stride) {
      const int64_t r = i / e.L;
      const double2 dg = static_cast<const double2*>(e.c)[r];
      const double2 j = zdiv(make_double2(1.0, 0.0), dg);
      static_cast<T*>(e.a)[i] = from_d2<T>(zmul(static_cast<const double2*>(e.b)[i], j));
      if (i % e.L == 0) {
        static_cast<T*>(e.d)[r] = from_d2<T>(dg);
        static_cast<T*>(e.e)[r] = from_d2<T>(j);
      }
    }
    return;
  }
  for (int64_t i = i0; i < e.n; i += stride) {
    switch (op) {
      case E_CONVERT_IN:   // a null source is the zero block (no warm start)
        static_cast<T*>(e.a)[i] = e.b ? from_d2<T>(static_cast<const double2*>(e.b)[i]) : from_d2<T>(make_double2(0.0, 0.0));
        break;
      case E_ZERO: static_cast<T*>(e.a)[i] = from_d2<T>(make_double2(0.0, 0.0)); break;
      case E_CONVERT_OUT: static_cast<double2*>(e.a)[i] = to_d2(static_cast<const T*>(e.b)[i]); break;
      default: break;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) batch_elem_kernel(const ElemArgs* args, const ProbDev* pd, ListDev l, int op) {
  __shared__ __align__(16) ElemArgs se;
  for_items(l, kClsBlas, args, &se, [&](int p, int64_t bid) { elem_body<T>(se, op, bid, pd[p].nblk); });
}

// ---- one CTA per problem ------------------------------------------------------------
__global__ void batch_alpha_kernel(const ProbDev* pd, const int* flags, int L) {
  const int p = blockIdx.x;
  if (!flags[p]) return;
  extern __shared__ double2 sm[];
  bicg_alpha_body(pd[p].sp, L, pd[p].st, sm);
}

__global__ void batch_zeta_beta_kernel(const ProbDev* pd, const int* flags, int L) {
  const int p = blockIdx.x;
  if (!flags[p]) return;
  extern __shared__ double2 sm[];
  bicg_zeta_beta_body(pd[p].sp, L, pd[p].dotp, pd[p].nblk, pd[p].st, sm);
}

// Solver state reset (working precision, and for the FP64 side) and the
// constant -1 used as a block coefficient.
__global__ void batch_reset_kernel(const ProbDev* pd, const int* flags, int reset64) {
  const int p = blockIdx.x;
  if (!flags[p] || threadIdx.x != 0) return;
  memset(pd[p].st, 0, sizeof(SolverState));
  pd[p].sp.r[0] = make_double2(-1.0, 0.0);
  if (reset64 && pd[p].st64) memset(pd[p].st64, 0, sizeof(SolverState));
}

// Per-problem outputs and the mixed form's bookkeeping (device).
struct Outs {
  int* status;       // [nprob] BDDA_* of each problem
  int* iter_fin;     // [nprob]
  double* err_fin;   // [nprob]
  double* hist;      // [nprob][itermax] or null
  int itermax;
  double tol;
  // mixed form
  double replace_drop;     // replace the residual after this drop (the one-problem solver's setting)
  double diverge_factor;   // abandon when the residual exceeds its minimum so far by this (same)
  double* prev;      // [nprob] true residual of the previous round
  int* total;        // [nprob] iterations of all rounds so far
  int* ran;          // [nprob] iterations of the last round; -1 breakdown
  double* rmax;      // [nprob] largest recursive residual since the last replacement
  double* rmin;      // [nprob] smallest recursive residual of the round
  int* repl;         // [nprob] flags: replace the residual this iteration
  int* outer;        // [nprob] flags: problem still running
  int* inner;        // [nprob] flags: recursion iterating
  int* acc;          // [nprob] flags: true residual to evaluate
  int* outflag;      // [nprob] flags: write X out
  int* counters;     // [0] still running  [1] rounds started
};

// ||R|| from the update partials and the convergence test of one iteration
// (bl_krylov.py:177-182).  mode 0: plain solve, final outputs; 1: a round
// of the mixed form; 2: the norm only (set_bnorm: it is ||M^-1 B||).
__global__ void batch_check_kernel(const ProbDev* pd, int* flags, int* left, const int* ctl, Outs o, int mode,
                                   int set_bnorm) {
  const int p = blockIdx.x;
  if (!flags[p]) return;
  norm_body(pd[p].nrmp, pd[p].nblk, pd[p].st, set_bnorm);
  if (mode == 2 || threadIdx.x != 0) return;
  const int k = ctl[1];
  const double err = pd[p].st->err;
  const int bad = pd[p].st->bad;
  bool stop = false;
  if (mode == 0) {
    if (bad == 1) {
      o.status[p] = BDDA_BREAKDOWN;
      stop = true;
    } else {
      if (o.hist) o.hist[(int64_t)p * o.itermax + k] = err;
      o.iter_fin[p] = k;
      o.err_fin[p] = err;
      if (bad == 2) { o.status[p] = BDDA_NOT_CONVERGED; stop = true; }
      else if (err < o.tol) { o.status[p] = BDDA_OK; stop = true; }
      else if (k + 1 >= o.itermax) stop = true;
    }
  } else {   // mixed form: stop only on a replaced (true) residual or the iteration budget
    const int tot = o.total[p];
    if (bad == 1) {
      o.status[p] = BDDA_BREAKDOWN;
      o.ran[p] = -1;
      stop = true;
    } else {
      o.ran[p] = k + 1;
      const double rm = k == 0 ? 0.0 : o.rmax[p];
      if (bad != 2 && err == err && (err < o.tol || err < o.replace_drop * rm)) {
        o.repl[p] = 1;   // the replacement step decides
      } else {
        if (o.hist && tot + k < o.itermax) o.hist[(int64_t)p * o.itermax + tot + k] = err;
        o.rmax[p] = err > rm ? err : rm;
        const double rn = k == 0 ? err : fmin(o.rmin[p], err);
        o.rmin[p] = rn;
        if (bad == 2 || !(err < INFINITY) || tot + k + 1 >= o.itermax) stop = true;
        if (err > o.diverge_factor * rn) {   // diverged: the problem stops unconverged
          o.ran[p] = -2;
          stop = true;
        }
      }
    }
  }
  if (stop) {
    flags[p] = 0;
    atomicSub(left, 1);
  }
}

// Residual replacement of the mixed form: R was recomputed as M^-1 (B - A X)
// with the complex128 product; its norm continues the recursion and is the
// convergence test.
__global__ void batch_replace_kernel(const ProbDev* pd, int* flags, int* left, const int* ctl, Outs o) {
  const int p = blockIdx.x;
  if (!o.repl[p]) return;
  norm_body(pd[p].nrmp, pd[p].nblk, pd[p].st, 0);
  if (threadIdx.x != 0) return;
  o.repl[p] = 0;
  const int k = ctl[1];
  const int tot = o.total[p];
  const double err = pd[p].st->err;
  o.rmax[p] = err;
  if (o.hist && tot + k < o.itermax) o.hist[(int64_t)p * o.itermax + tot + k] = err;
  if (pd[p].st->bad == 2 || !(err < INFINITY) || err < o.tol || tot + k + 1 >= o.itermax) {
    flags[p] = 0;
    atomicSub(left, 1);
  }
}

// ||M^-1 (B - A X)|| / ||M^-1 B|| of the mixed form's true residual (||M^-1 B||
// from the Krylov state, set when the round started).
__global__ void batch_true_residual_kernel(const ProbDev* pd, const int* flags) {
  const int p = blockIdx.x;
  if (!flags[p]) return;
  if (threadIdx.x == 0) {
    pd[p].st64->bnorm = pd[p].st->bnorm;
    pd[p].st64->bad = 0;
  }
  norm_body(pd[p].nrmp64, pd[p].nblk, pd[p].st64, 0);
}

// After a round of the mixed form: count its iterations; flag the true
// residual for evaluation unless the recursion broke down.
__global__ void batch_round_end_kernel(Outs o, const int* started, int nprob) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nprob) return;
  o.acc[p] = 0;
  o.inner[p] = 0;
  if (!started[p]) return;
  const int r = o.ran[p];
  if (r < 0) {   // breakdown (status set) or divergence (stays not converged)
    o.outer[p] = 0;
    atomicSub(&o.counters[0], 1);
    return;
  }
  o.total[p] += r;
  o.iter_fin[p] = o.total[p] - 1;
  o.acc[p] = 1;
}

// The mixed form's decision on the true residual: done, stop, or another round.
__global__ void batch_round_decide_kernel(const ProbDev* pd, Outs o, int nprob, int allow_more) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nprob || !o.acc[p]) return;
  const double err = pd[p].st64->err;
  o.err_fin[p] = err;
  bool stop = true;
  if (pd[p].st64->bad == 2 || !(err == err)) o.status[p] = BDDA_NOT_CONVERGED;
  else if (err < o.tol) o.status[p] = BDDA_OK;
  else if (o.total[p] >= o.itermax || !allow_more || !(err < 0.9 * o.prev[p])) o.status[p] = BDDA_NOT_CONVERGED;
  else {
    stop = false;
    o.prev[p] = err;
    o.inner[p] = 1;
    atomicAdd(&o.counters[1], 1);
  }
  if (stop) {
    o.outer[p] = 0;
    atomicSub(&o.counters[0], 1);
  }
}

__global__ void batch_outflag_kernel(Outs o, int n) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) o.outflag[p] = o.status[p] != BDDA_BREAKDOWN;
}

// ---- host side ------------------------------------------------------------------------
size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

int blas_items(int64_t rows) {
  const int64_t b = (rows + kRowsPerBlasItem - 1) / kRowsPerBlasItem;
  return (int)std::max<int64_t>(1, std::min<int64_t>(kRedBlocks, b));
}

// Column tile width of the batched pencil passes: the widest that fits the
// budget at the largest axis length in the batch.
template <typename T>
int batch_lt(int M, int L, int kind) {
  for (int lt : {8, 4, 2}) {
    if (lt > 2 && lt / 2 >= L) continue;
    if ((size_t)pencil_smem_bytes<T>(M, lt, kind) <= kPencilBudget) return lt;
  }
  return 2;
}

constexpr int kGramSites = 2, kUpdSites = 10, kMvpSites = 4, kElemSites = 9;
enum { U_P = 0, U_T, U_X, U_R, U_RB, U_RX0, U_P0, U_R00, U_TRUE, U_REPL };   // update sites
enum { EL_PREP = 0, EL_X0, EL_OUT, EL_PREP32, EL_P2S, EL_T2S, EL_O2V, EL_O2Z };   // elementwise sites

// Workspace carve-up.
struct ProbLayout {
  size_t field, vec[8], diag, jpre, gpart, dotp, nrmp, small, st;
  size_t in32, out32, diag32, jpre32, nrmp64, st64;   // mixed form
};

struct BatchLayout {
  std::vector<ProbLayout> p;
  size_t act, start, cnt, total, ctl, probdev;
  size_t status, iter, err, hist, prev, rmax, rmin, totalit, ran, flags, counters;
  size_t gram, upd, dots, mvp, elem;
  size_t bytes;
};

int make_layout(const bdda_batch_problem* pr, int nprob, int mode, int L, int itermax, BatchLayout* out) {
  BatchLayout& o = *out;
  o.p.assign(nprob, ProbLayout());
  const bool mixed = mode == BDDA_BATCH_MIXED;
  const size_t cb = mode == BDDA_BATCH_C64 ? 8 : 16;
  const int fprec = mode == BDDA_BATCH_C64 ? BDDA_C64 : BDDA_C128;   // one field buffer serves both products
  size_t off = 0;
  for (int i = 0; i < nprob; ++i) {
    ProbLayout& q = o.p[i];
    memset(&q, 0, sizeof(q));
    const int64_t rows = 3 * (int64_t)pr[i].n_occ;
    const size_t vb = (size_t)rows * L * cb;
    const int nb = blas_items(rows);
    const size_t fb = bdda_mvp_workspace_bytes(pr[i].plan, fprec, L);
    if (fb == 0) return BDDA_BAD_ARG;
    q.field = off; off = al256(off + fb);
    for (int v = 0; v < 8; ++v) { q.vec[v] = off; off = al256(off + vb); }
    q.diag = off; off = al256(off + (size_t)rows * cb);
    q.jpre = off; off = al256(off + (size_t)rows * cb);
    q.gpart = off; off = al256(off + (size_t)nb * 2 * L * L * sizeof(double2));
    q.dotp = off; off = al256(off + (size_t)nb * 3 * sizeof(double));
    q.nrmp = off; off = al256(off + (size_t)nb * sizeof(double));
    q.small = off; off = al256(off + (size_t)kSmallMats * kMaxL * kMaxL * sizeof(double2) + 64 * sizeof(int));
    q.st = off; off = al256(off + sizeof(SolverState));
    if (mixed) {
      const size_t v32 = (size_t)rows * L * 8;
      q.in32 = off; off = al256(off + v32);
      q.out32 = off; off = al256(off + v32);
      q.diag32 = off; off = al256(off + (size_t)rows * 8);
      q.jpre32 = off; off = al256(off + (size_t)rows * 8);
      q.nrmp64 = off; off = al256(off + (size_t)nb * sizeof(double));
      q.st64 = off; off = al256(off + sizeof(SolverState));
    }
  }
  const size_t np = (size_t)nprob;
  o.act = off; off = al256(off + np * sizeof(int));
  o.start = off; off = al256(off + (size_t)kNCls * (np + 1) * sizeof(int64_t));
  o.cnt = off; off = al256(off + (size_t)2 * kNCls * np * sizeof(int64_t));
  o.total = off; off = al256(off + (size_t)kNCls * sizeof(int64_t));
  o.ctl = off; off = al256(off + 16 * sizeof(int));
  o.probdev = off; off = al256(off + np * sizeof(ProbDev));
  o.status = off; off = al256(off + np * sizeof(int));
  o.iter = off; off = al256(off + np * sizeof(int));
  o.err = off; off = al256(off + np * sizeof(double));
  o.hist = off; off = al256(off + np * std::max(itermax, 1) * sizeof(double));
  o.prev = off; off = al256(off + np * sizeof(double));
  o.rmax = off; off = al256(off + np * sizeof(double));
  o.rmin = off; off = al256(off + np * sizeof(double));
  o.totalit = off; off = al256(off + np * sizeof(int));
  o.ran = off; off = al256(off + np * sizeof(int));
  o.flags = off; off = al256(off + 7 * np * sizeof(int));
  o.counters = off; off = al256(off + 16 * sizeof(int));
  o.gram = off; off = al256(off + kGramSites * np * sizeof(GramArgs));
  o.upd = off; off = al256(off + kUpdSites * np * sizeof(UpdateArgs));
  o.dots = off; off = al256(off + np * sizeof(DotArgs));
  o.mvp = off; off = al256(off + kMvpSites * 5 * np * sizeof(PassArgs));
  o.elem = off; off = al256(off + kElemSites * np * sizeof(ElemArgs));
  o.bytes = off;
  return BDDA_OK;
}

int check_problems(const bdda_batch_problem* pr, int nprob, int mode, int L) {
  if (!pr || nprob < 1 || nprob > kMaxBatch) return BDDA_BAD_ARG;
  if (L != 8 && L != 16 && L != 32 && L != 64) return BDDA_BAD_ARG;
  if (mode < BDDA_BATCH_C128 || mode > BDDA_BATCH_MIXED) return BDDA_BAD_ARG;
  for (int i = 0; i < nprob; ++i) {
    const bdda_batch_problem& q = pr[i];
    if (!q.plan || q.n_occ < 1 || !q.cell_map || !q.diag || !q.B || !q.X) return BDDA_BAD_ARG;
    if ((mode != BDDA_BATCH_C64 && !q.ghat) || (mode != BDDA_BATCH_C128 && !q.ghat_c64)) return BDDA_BAD_ARG;
  }
  for (int i = 0; i < nprob; ++i)
    if (!pr[i].plan->dev_tables) return BDDA_NO_WORKSPACE;
  return BDDA_OK;
}

template <typename K>
int persistent_grid(K kern, size_t smem, int nsm, int* grid) {
  int nb = 0;
  BDDA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  BDDA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 256, smem));
  *grid = std::max(1, nb) * nsm;
  return BDDA_OK;
}

#define BTRY(expr)                 \
  do {                             \
    int s_ = (expr);               \
    if (s_ != BDDA_OK) return s_;  \
  } while (0)

// The batched launches in one precision.
template <typename T>
struct Engine {
  typedef typename std::conditional<std::is_same<T, float2>::value, float2, double2>::type A;
  int nprob = 0, L = 0, nsm = 0;
  cudaStream_t st = nullptr;
  ListDev list;
  const ProbDev* pd = nullptr;
  int lt[5] = {2, 2, 2, 2, 2};
  size_t psmem[5] = {0, 0, 0, 0, 0};
  int pgrid[5] = {1, 1, 1, 1, 1};
  int64_t upper[kNCls] = {1, 1, 1, 1, 1, 1};   // items over all problems: bound of the grid
  int gram_grid[2] = {1, 1}, upd_grid = 1, dots_grid = 1, elem_grid = 1;
  size_t gram_smem[2] = {0, 0}, upd_smem = 0;
  unsigned long long launches = 0;

  void count(int n = 1) {
    launches += (unsigned long long)n;
    count_launch(n);
  }
  static int cap(int g, int64_t items) { return (int)std::max<int64_t>(1, std::min<int64_t>(g, items)); }

  template <int KIND, int LTT>
  int setup_pass(int q) {
    // passes of one kind and tile width share a kernel: its shared-memory
    // limit is the largest any of them launches with
    size_t smem = 0;
    for (int r = 0; r < 5; ++r)
      if (kPassKind[r] == KIND && lt[r] == LTT) smem = std::max(smem, psmem[r]);
    return persistent_grid(batch_pencil_kernel<T, KIND, LTT>, smem, nsm, &pgrid[q]);
  }
  template <int KIND>
  int setup_pass_lt(int q) {
    if (lt[q] == 8) return setup_pass<KIND, 8>(q);
    if (lt[q] == 4) return setup_pass<KIND, 4>(q);
    return setup_pass<KIND, 2>(q);
  }
  template <int LL>
  int setup_blas() {
    gram_smem[0] = (size_t)2 * 2 * 16 * LL * sizeof(T);
    gram_smem[1] = (size_t)2 * 3 * 16 * LL * sizeof(T);
    BTRY(persistent_grid(batch_gram_kernel<T, true, LL, 1>, gram_smem[0], nsm, &gram_grid[0]));
    BTRY(persistent_grid(batch_gram_kernel<T, true, LL, 2>, gram_smem[1], nsm, &gram_grid[1]));
    constexpr int TC = LL >= 64 ? 4 : (LL >= 32 ? 2 : 1);
    constexpr int RB = (256 / (LL / TC)) * 2;
    upd_smem = ((size_t)LL * LL + (size_t)RB * LL) * sizeof(A);
    return persistent_grid(batch_update_kernel<T, A, LL>, upd_smem, nsm, &upd_grid);
  }

  int setup(const bdda_batch_problem* pr) {
    int dev = 0;
    BDDA_CUDA_TRY(cudaGetDevice(&dev));
    BDDA_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int axis[5] = {2, 1, 0, 1, 2};
    for (int q = 0; q < 5; ++q) {
      int maxM = 1;
      for (int i = 0; i < nprob; ++i) maxM = std::max(maxM, pr[i].plan->ax[axis[q]].M);
      lt[q] = batch_lt<T>(maxM, L, kPassKind[q]);
      psmem[q] = (size_t)pencil_smem_bytes<T>(maxM, lt[q], kPassKind[q]);
      if (psmem[q] > 226 * 1024) return BDDA_BAD_ARG;
    }
    BTRY(setup_pass_lt<K_FWD>(0));
    BTRY(setup_pass_lt<K_FWD>(1));
    BTRY(setup_pass_lt<K_CONV>(2));
    BTRY(setup_pass_lt<K_INV>(3));
    BTRY(setup_pass_lt<K_INV>(4));
    if (L == 8) BTRY(setup_blas<8>());
    else if (L == 16) BTRY(setup_blas<16>());
    else if (L == 32) BTRY(setup_blas<32>());
    else BTRY(setup_blas<64>());
    BTRY(persistent_grid(batch_dots_kernel<T>, 0, nsm, &dots_grid));
    BTRY(persistent_grid(batch_elem_kernel<T>, 0, nsm, &elem_grid));
    return BDDA_OK;
  }

  int list_build(const int* flags, int advance, int set_left) {
    list_kernel<<<1, kMaxBatch, 0, st>>>(list, flags, advance, set_left);
    count();
    BDDA_CUDA_TRY(cudaGetLastError());
    return BDDA_OK;
  }

  template <int KIND, int LTT>
  int pass_lt(const PassArgs* args, int q) {
    batch_pencil_kernel<T, KIND, LTT><<<cap(pgrid[q], upper[q]), 256, psmem[q], st>>>(args, list, q);
    count();
    BDDA_CUDA_TRY(cudaGetLastError());
    return BDDA_OK;
  }
  template <int KIND>
  int pass(const PassArgs* args, int q) {
    if (lt[q] == 8) return pass_lt<KIND, 8>(args, q);
    if (lt[q] == 4) return pass_lt<KIND, 4>(args, q);
    return pass_lt<KIND, 2>(args, q);
  }
  // site: 5 x nprob PassArgs, pass-major
  int mvp(const PassArgs* site) {
    const size_t n = (size_t)nprob;
    BTRY(pass<K_FWD>(site, 0));
    BTRY(pass<K_FWD>(site + n, 1));
    BTRY(pass<K_CONV>(site + 2 * n, 2));
    BTRY(pass<K_INV>(site + 3 * n, 3));
    BTRY(pass<K_INV>(site + 4 * n, 4));
    return BDDA_OK;
  }

  template <int LL>
  int gram_l(const GramArgs* g, int nb, const int* flags) {
    if (nb == 1)
      batch_gram_kernel<T, true, LL, 1><<<cap(gram_grid[0], upper[kClsBlas]), 256, gram_smem[0], st>>>(g, pd, list);
    else
      batch_gram_kernel<T, true, LL, 2><<<cap(gram_grid[1], upper[kClsBlas]), 256, gram_smem[1], st>>>(g, pd, list);
    BDDA_CUDA_TRY(cudaGetLastError());
    const int width = nb * LL * LL;
    batch_gram_reduce_kernel<<<dim3((width + 255) / 256, nprob), 256, 0, st>>>(g, pd, flags, width);
    BDDA_CUDA_TRY(cudaGetLastError());
    count(2);
    return BDDA_OK;
  }
  int gram(const GramArgs* g, int nb, const int* flags) {
    if (L == 8) return gram_l<8>(g, nb, flags);
    if (L == 16) return gram_l<16>(g, nb, flags);
    if (L == 32) return gram_l<32>(g, nb, flags);
    return gram_l<64>(g, nb, flags);
  }

  template <int LL>
  int upd_l(const UpdateArgs* u, int skip_first) {
    batch_update_kernel<T, A, LL><<<cap(upd_grid, upper[kClsBlas]), 256, upd_smem, st>>>(u, pd, list, skip_first);
    BDDA_CUDA_TRY(cudaGetLastError());
    count();
    return BDDA_OK;
  }
  int upd(const UpdateArgs* u, int skip_first = 0) {
    if (L == 8) return upd_l<8>(u, skip_first);
    if (L == 16) return upd_l<16>(u, skip_first);
    if (L == 32) return upd_l<32>(u, skip_first);
    return upd_l<64>(u, skip_first);
  }

  int dots(const DotArgs* d) {
    batch_dots_kernel<T><<<cap(dots_grid, upper[kClsBlas]), 256, 0, st>>>(d, pd, list);
    BDDA_CUDA_TRY(cudaGetLastError());
    count();
    return BDDA_OK;
  }

  int elem(const ElemArgs* e, int op) {
    batch_elem_kernel<T><<<cap(elem_grid, upper[kClsBlas]), 256, 0, st>>>(e, pd, list, op);
    BDDA_CUDA_TRY(cudaGetLastError());
    count();
    return BDDA_OK;
  }
};

__global__ void batch_init_kernel(Outs o, int nprob, int mixed, int* f_all, int* f_started, int* ctl) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < nprob) {
    o.status[p] = BDDA_NOT_CONVERGED;
    o.iter_fin[p] = 0;
    o.err_fin[p] = INFINITY;
    o.prev[p] = INFINITY;
    o.total[p] = 0;
    o.ran[p] = 0;
    o.rmax[p] = 0.0;
    o.rmin[p] = INFINITY;
    o.repl[p] = 0;
    o.inner[p] = 1;
    o.outer[p] = mixed ? 1 : 0;
    o.acc[p] = 0;
    o.outflag[p] = 0;
    f_all[p] = 1;
    f_started[p] = 0;
  }
  if (p == 0) {
    for (int i = 0; i < 16; ++i) ctl[i] = 0;
    o.counters[0] = mixed ? nprob : 0;
    o.counters[1] = 0;
  }
}

__global__ void zero_int_kernel(int* a, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = 0;
}

__global__ void copy_int_kernel(int* dst, const int* src, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i];
}

// One batched solve; T is the precision of the Krylov vectors (complex128 in
// the mixed form, whose products run in complex64).
template <typename T>
int batch_run(const bdda_batch_problem* pr, int nprob, int mode, int L, double tol, int itermax, int max_outer,
              int use_graph, int* status, int* iter_fin, double* err_fin, double* history, unsigned char* w,
              const BatchLayout& lay, cudaStream_t st) {
  const bool mixed = mode == BDDA_BATCH_MIXED;
  const size_t np = (size_t)nprob;
  Engine<T> e;          // vectors, block kernels, products in the vectors' precision
  Engine<float2> e32;   // mixed form: the products inside the iteration
  e.nprob = e32.nprob = nprob;
  e.L = e32.L = L;
  e.st = e32.st = st;
  BTRY(e.setup(pr));
  if (mixed) BTRY(e32.setup(pr));

  ProbDev* dpd = reinterpret_cast<ProbDev*>(w + lay.probdev);
  GramArgs* dgram = reinterpret_cast<GramArgs*>(w + lay.gram);
  UpdateArgs* dupd = reinterpret_cast<UpdateArgs*>(w + lay.upd);
  DotArgs* ddot = reinterpret_cast<DotArgs*>(w + lay.dots);
  PassArgs* dmvp = reinterpret_cast<PassArgs*>(w + lay.mvp);
  ElemArgs* del = reinterpret_cast<ElemArgs*>(w + lay.elem);
  int* flags = reinterpret_cast<int*>(w + lay.flags);
  int* f_active = flags;                 // recursion iterating
  int* f_outer = flags + np;             // mixed form: problem still running
  int* f_acc = flags + 2 * np;           // mixed form: true residual to evaluate
  int* f_out = flags + 3 * np;
  int* f_all = flags + 4 * np;
  int* f_started = flags + 5 * np;
  int* f_repl = flags + 6 * np;          // mixed form: residual replacement this iteration
  int* ctl = reinterpret_cast<int*>(w + lay.ctl);
  Outs o;
  o.status = reinterpret_cast<int*>(w + lay.status);
  o.iter_fin = reinterpret_cast<int*>(w + lay.iter);
  o.err_fin = reinterpret_cast<double*>(w + lay.err);
  o.hist = history ? reinterpret_cast<double*>(w + lay.hist) : nullptr;
  o.itermax = std::max(itermax, 1);
  o.tol = tol;
  o.replace_drop = mixed_replace_drop();
  o.diverge_factor = mixed_diverge_factor();
  o.prev = reinterpret_cast<double*>(w + lay.prev);
  o.total = reinterpret_cast<int*>(w + lay.totalit);
  o.ran = reinterpret_cast<int*>(w + lay.ran);
  o.rmax = reinterpret_cast<double*>(w + lay.rmax);
  o.rmin = reinterpret_cast<double*>(w + lay.rmin);
  o.repl = f_repl;
  o.outer = f_outer;
  o.inner = f_active;
  o.acc = f_acc;
  o.outflag = f_out;
  o.counters = reinterpret_cast<int*>(w + lay.counters);

  // ---- host images of the descriptors and argument sites ----
  std::vector<ProbDev> hpd(np);
  std::vector<int64_t> hcnt((size_t)2 * kNCls * np, 0);
  std::vector<GramArgs> hgram(kGramSites * np);
  std::vector<UpdateArgs> hupd(kUpdSites * np);
  std::vector<DotArgs> hdot(np);
  std::vector<PassArgs> hmvp(kMvpSites * 5 * np);
  std::vector<ElemArgs> hel(kElemSites * np);
  memset(hpd.data(), 0, hpd.size() * sizeof(ProbDev));
  memset(hgram.data(), 0, hgram.size() * sizeof(GramArgs));
  memset(hupd.data(), 0, hupd.size() * sizeof(UpdateArgs));
  memset(hdot.data(), 0, hdot.size() * sizeof(DotArgs));
  memset(hmvp.data(), 0, hmvp.size() * sizeof(PassArgs));
  memset(hel.data(), 0, hel.size() * sizeof(ElemArgs));
  bool any_x0 = false;
  for (int i = 0; i < nprob; ++i) {
    const ProbLayout& q = lay.p[i];
    const bdda_batch_problem& P = pr[i];
    any_x0 = any_x0 || P.X0 != nullptr;
    const int64_t rows = 3 * (int64_t)P.n_occ;
    ProbDev& d = hpd[i];
    d.sp = small_ptrs(w + q.small);
    d.st = reinterpret_cast<SolverState*>(w + q.st);
    d.dotp = reinterpret_cast<double*>(w + q.dotp);
    d.nrmp = reinterpret_cast<double*>(w + q.nrmp);
    d.nblk = blas_items(rows);
    if (mixed) {
      d.st64 = reinterpret_cast<SolverState*>(w + q.st64);
      d.nrmp64 = reinterpret_cast<double*>(w + q.nrmp64);
    }
    void *X = w + q.vec[0], *R = w + q.vec[1], *Pp = w + q.vec[2], *R0 = w + q.vec[3], *V = w + q.vec[4],
         *Tt = w + q.vec[5], *Z = w + q.vec[6], *Bj = w + q.vec[7];
    void* diagT = w + q.diag;
    void* jpreT = w + q.jpre;
    double2* gpart = reinterpret_cast<double2*>(w + q.gpart);
    GramArgs& g0 = hgram[0 * np + i];
    g0.n = rows; g0.L = L; g0.nB = 2; g0.A = R0; g0.B[0] = V; g0.B[1] = R; g0.partial = gpart;
    GramArgs& g1 = hgram[1 * np + i];
    g1.n = rows; g1.L = L; g1.nB = 1; g1.A = R0; g1.B[0] = Z; g1.B[1] = nullptr; g1.partial = gpart;
    // block updates out = a0 Y0 + a1 Y1 + (X1 + c2 X2) M   (bl_krylov.py:168-185)
    auto U = [&](int site) -> UpdateArgs& {
      UpdateArgs& u = hupd[(size_t)site * np + i];
      u.n = rows;
      u.L = L;
      return u;
    };
    { UpdateArgs& u = U(U_P); u.out = Pp; u.Y0 = R; u.X1 = Pp; u.X2 = V; u.c2 = &d.st->negzeta; u.M = d.sp.beta; }
    { UpdateArgs& u = U(U_T); u.out = Tt; u.Y0 = R; u.X1 = V; u.M = d.sp.negalpha; }
    { UpdateArgs& u = U(U_X); u.out = X; u.Y0 = X; u.Y1 = Tt; u.a1 = &d.st->zeta; u.X1 = Pp; u.M = d.sp.alpha; }
    { UpdateArgs& u = U(U_R); u.out = R; u.Y0 = Tt; u.Y1 = Z; u.a1 = &d.st->negzeta; u.norm_partial = d.nrmp; }
    { UpdateArgs& u = U(U_RB); u.out = R; u.Y0 = Bj; u.norm_partial = d.nrmp; }
    { UpdateArgs& u = U(U_RX0); u.out = R; u.Y0 = Bj; u.Y1 = V; u.a1 = d.sp.r; }
    { UpdateArgs& u = U(U_P0); u.out = Pp; u.Y0 = R; }
    { UpdateArgs& u = U(U_R00); u.out = R0; u.Y0 = R; }
    if (mixed) {
      { UpdateArgs& u = U(U_TRUE); u.out = R; u.Y0 = Bj; u.Y1 = V; u.a1 = d.sp.r; u.norm_partial = d.nrmp64; }
      { UpdateArgs& u = U(U_REPL); u.out = R; u.Y0 = Bj; u.Y1 = Z; u.a1 = d.sp.r; u.norm_partial = d.nrmp; }
    }
    DotArgs& dd = hdot[i];
    dd.n = rows * L; dd.A = Z; dd.B = Tt; dd.partial = d.dotp;
    // products.  Plain modes: site 0 P -> V, site 1 T -> Z, site 2 X -> V (warm
    // start), all in T.  Mixed form: site 0 the complex64 product in32 -> out32
    // (both products of the iteration), site 2 the complex128 X -> V.
    auto put = [&](int site, const void* src, void* dst, bool f32) {
      PassArgs pa[5];
      int64_t P0[5];
      const int* ltv = f32 && mixed ? e32.lt : e.lt;
      if (f32)
        mvp_pass_args<float2>(P.plan, L, static_cast<const float2*>(P.ghat_c64), P.cell_map,
                              static_cast<const float2*>(src),
                              static_cast<const float2*>(mixed ? (const void*)(w + q.diag32) : diagT),
                              static_cast<const float2*>(mixed ? (const void*)(w + q.jpre32) : jpreT),
                              static_cast<float2*>(dst), reinterpret_cast<float2*>(w + q.field), pa, P0);
      else
        mvp_pass_args<double2>(P.plan, L, static_cast<const double2*>(P.ghat), P.cell_map,
                               static_cast<const double2*>(src), static_cast<const double2*>(diagT),
                               static_cast<const double2*>(jpreT), static_cast<double2*>(dst),
                               reinterpret_cast<double2*>(w + q.field), pa, P0);
      const int list = f32 && mixed ? 1 : 0;
      for (int ps = 0; ps < 5; ++ps) {
        pa[ps].ntile = (L + ltv[ps] - 1) / ltv[ps];
        hmvp[((size_t)site * 5 + ps) * np + i] = pa[ps];
        hcnt[((size_t)list * kNCls + ps) * np + i] = P0[ps] * pa[ps].P1 * pa[ps].ntile;
      }
    };
    const bool t32 = std::is_same<T, float2>::value;
    if (mixed) {
      put(0, w + q.in32, w + q.out32, true);
      put(2, X, V, false);
      put(3, X, Z, false);   // residual replacement
    } else {
      put(0, Pp, V, t32);
      put(1, Tt, Z, t32);
      put(2, X, V, t32);
    }
    hcnt[((size_t)0 * kNCls + kClsBlas) * np + i] = d.nblk;
    hcnt[((size_t)1 * kNCls + kClsBlas) * np + i] = d.nblk;
    auto E = [&](int site) -> ElemArgs& { return hel[(size_t)site * np + i]; };
    { ElemArgs& x = E(EL_PREP); x.n = rows; x.L = L; x.a = Bj; x.b = P.B; x.c = P.diag; x.d = diagT; x.e = jpreT; }
    { ElemArgs& x = E(EL_X0); x.n = rows * L; x.a = X; x.b = P.X0; }
    { ElemArgs& x = E(EL_OUT); x.n = rows * L; x.a = P.X; x.b = X; }
    if (mixed) {
      { ElemArgs& x = E(EL_PREP32); x.n = rows; x.L = L; x.a = w + q.in32; x.b = P.B; x.c = P.diag; x.d = w + q.diag32; x.e = w + q.jpre32; }
      { ElemArgs& x = E(EL_P2S); x.n = rows * L; x.a = w + q.in32; x.b = Pp; }
      { ElemArgs& x = E(EL_T2S); x.n = rows * L; x.a = w + q.in32; x.b = Tt; }
      { ElemArgs& x = E(EL_O2V); x.n = rows * L; x.a = V; x.b = w + q.out32; }
      { ElemArgs& x = E(EL_O2Z); x.n = rows * L; x.a = Z; x.b = w + q.out32; }
    }
  }
  for (int list = 0; list < 2; ++list)
    for (int c = 0; c < kNCls; ++c) {
      int64_t sum = 0;
      for (int i = 0; i < nprob; ++i) sum += hcnt[((size_t)list * kNCls + c) * np + i];
      (list == 0 ? e.upper : e32.upper)[c] = std::max<int64_t>(1, sum);
    }
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st) == cudaSuccess ? BDDA_OK : BDDA_CUDA_ERROR;
  };
  BTRY(up(dpd, hpd.data(), np * sizeof(ProbDev)));
  BTRY(up(w + lay.cnt, hcnt.data(), hcnt.size() * sizeof(int64_t)));
  BTRY(up(dgram, hgram.data(), hgram.size() * sizeof(GramArgs)));
  BTRY(up(dupd, hupd.data(), hupd.size() * sizeof(UpdateArgs)));
  BTRY(up(ddot, hdot.data(), hdot.size() * sizeof(DotArgs)));
  BTRY(up(dmvp, hmvp.data(), hmvp.size() * sizeof(PassArgs)));
  BTRY(up(del, hel.data(), hel.size() * sizeof(ElemArgs)));
  ListDev l0;
  l0.nprob = nprob;
  l0.act = reinterpret_cast<int*>(w + lay.act);
  l0.start = reinterpret_cast<int64_t*>(w + lay.start);
  l0.cnt = reinterpret_cast<const int64_t*>(w + lay.cnt);
  l0.total = reinterpret_cast<int64_t*>(w + lay.total);
  l0.ctl = ctl;
  e.list = l0;
  e.pd = dpd;
  e32.list = l0;
  e32.list.cnt = l0.cnt + (size_t)kNCls * np;   // the lists share their buffers: the last build counts
  e32.pd = dpd;
  const int gp = (nprob + 255) / 256;
  const size_t sm2 = (size_t)2 * L * L * sizeof(double2);
  BDDA_CUDA_TRY(cudaFuncSetAttribute(batch_alpha_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
  BDDA_CUDA_TRY(cudaFuncSetAttribute(batch_zeta_beta_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));

  batch_init_kernel<<<gp, 256, 0, st>>>(o, nprob, mixed ? 1 : 0, f_all, f_started, ctl);
  batch_reset_kernel<<<nprob, 32, 0, st>>>(dpd, f_all, mixed ? 1 : 0);
  count_launch(2);
  BDDA_CUDA_TRY(cudaGetLastError());
  auto usite = [&](int s) { return dupd + (size_t)s * np; };
  auto esite = [&](int s) { return del + (size_t)s * np; };
  auto msite = [&](int s) { return dmvp + (size_t)s * 5 * np; };

  // the product inside the iteration: src -> dst in T, or through complex64 in the mixed form
  auto iter_mvp = [&](int site, int to32, int from32) -> int {
    if (!mixed) return e.mvp(msite(site));
    BTRY(e32.elem(esite(to32), E_CONVERT_IN));
    BTRY(e32.mvp(msite(0)));
    return e32.elem(esite(from32), E_CONVERT_OUT);
  };
  // one iteration of block-BiCGSTAB for every listed problem (bl_krylov.py:161-185);
  // the P update of the previous iteration opens it
  const int check_mode = mixed ? 1 : 0;
  auto iteration = [&]() -> int {
    BTRY(e.list_build(f_active, 1, 1));
    if (mixed) BTRY(e32.list_build(f_active, 0, 0));   // complex64 pencil counts; block counts agree
    BTRY(e.upd(usite(U_P), 1));                              // P = R + (P - zeta V) beta
    BTRY(iter_mvp(0, EL_P2S, EL_O2V));                       // V = M^-1 A P
    BTRY(e.gram(dgram, 2, f_active));                        // R0^H V, R0^H R
    batch_alpha_kernel<<<nprob, 256, sm2, st>>>(dpd, f_active, L);
    BTRY(e.upd(usite(U_T)));                                 // T = R - V alpha
    BTRY(iter_mvp(1, EL_T2S, EL_O2Z));                       // Z = M^-1 A T
    BTRY(e.gram(dgram + np, 1, f_active));                   // R0^H Z
    BTRY(e.dots(ddot));                                      // tr(Z^H T), tr(Z^H Z)
    batch_zeta_beta_kernel<<<nprob, 256, sm2, st>>>(dpd, f_active, L);
    BTRY(e.upd(usite(U_X)));                                 // X += P alpha + zeta T
    BTRY(e.upd(usite(U_R)));                                 // R = T - zeta Z, ||R||^2 partials
    batch_check_kernel<<<nprob, 256, 0, st>>>(dpd, f_active, ctl + 3, ctl, o, check_mode, 0);
    e.count(3);
    BDDA_CUDA_TRY(cudaGetLastError());
    if (mixed) {   // residual replacement of the flagged problems, complex128 product
      BTRY(e.list_build(f_repl, 0, 0));
      BTRY(e.mvp(msite(3)));
      BTRY(e.upd(usite(U_REPL)));
      batch_replace_kernel<<<nprob, 256, 0, st>>>(dpd, f_active, ctl + 3, ctl, o);
      e.count();
      BDDA_CUDA_TRY(cudaGetLastError());
    }
    return BDDA_OK;
  };
  // start of a solve for the problems flagged in f_active: R = Bj (- A X), P = R, R0 = R
  auto start_solve = [&](bool warm) -> int {
    BTRY(e.list_build(f_active, 0, 0));
    batch_reset_kernel<<<nprob, 32, 0, st>>>(dpd, f_active, 0);
    count_launch();
    BTRY(e.upd(usite(U_RB)));
    batch_check_kernel<<<nprob, 256, 0, st>>>(dpd, f_active, ctl + 3, ctl, o, 2, 1);   // ||M^-1 B||
    e.count();
    BDDA_CUDA_TRY(cudaGetLastError());
    if (warm) {   // with the exact product
      BTRY(e.mvp(msite(2)));
      BTRY(e.upd(usite(U_RX0)));
    }
    BTRY(e.upd(usite(U_P0)));
    BTRY(e.upd(usite(U_R00)));
    zero_int_kernel<<<1, 32, 0, st>>>(ctl + 1, 2);   // k = 0
    e.count();
    BDDA_CUDA_TRY(cudaGetLastError());
    return BDDA_OK;
  };

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  unsigned long long per_iter = 0;
  auto capture = [&]() -> int {
    if (!use_graph || gexec) return BDDA_OK;
    const unsigned long long before = e.launches + e32.launches;
    BDDA_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int s = iteration();
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (s != BDDA_OK) return s;
    if (ce != cudaSuccess) return BDDA_CUDA_ERROR;
    BDDA_CUDA_TRY(cudaGraphInstantiate(&gexec, graph, 0));
    per_iter = e.launches + e32.launches - before;
    count_launch(-(int)per_iter);   // captured, not run
    return BDDA_OK;
  };
  // iterate until every listed problem stopped (or maxit iterations)
  auto run_iterations = [&](int maxit) -> int {
    BTRY(capture());
    int done = 0;
    while (done < maxit) {
      const int n = std::min(kCheckEvery, maxit - done);
      for (int j = 0; j < n; ++j) {
        if (gexec) {
          BDDA_CUDA_TRY(cudaGraphLaunch(gexec, st));
          count_launch((int)per_iter);
        } else {
          BTRY(iteration());
        }
      }
      done += n;
      int left = 0;
      BDDA_CUDA_TRY(cudaMemcpyAsync(&left, ctl + 3, sizeof(int), cudaMemcpyDeviceToHost, st));
      BDDA_CUDA_TRY(cudaStreamSynchronize(st));
      if (left == 0) break;
    }
    return BDDA_OK;
  };

  const int rc = [&]() -> int {
    BTRY(e.list_build(f_all, 0, 0));
    BTRY(e.elem(esite(EL_PREP), E_PREPARE));
    BTRY(e.elem(esite(EL_X0), E_CONVERT_IN));
    if (!mixed) {
      BTRY(start_solve(any_x0));
      BTRY(run_iterations(itermax));
    } else {
      BTRY(e32.elem(esite(EL_PREP32), E_PREPARE));   // complex64 diagonal and Jacobi factors
      for (int round = 0; round < max_outer; ++round) {
        copy_int_kernel<<<gp, 256, 0, st>>>(f_started, f_active, nprob);
        count_launch();
        BTRY(start_solve(round > 0 || any_x0));
        BTRY(run_iterations(itermax));
        batch_round_end_kernel<<<gp, 256, 0, st>>>(o, f_started, nprob);
        count_launch();
        // the true residual M^-1 (B - A X) with the complex128 product
        BTRY(e.list_build(f_acc, 0, 0));
        BTRY(e.mvp(msite(2)));
        BTRY(e.upd(usite(U_TRUE)));
        batch_true_residual_kernel<<<nprob, 256, 0, st>>>(dpd, f_acc);
        BDDA_CUDA_TRY(cudaMemsetAsync(o.counters + 1, 0, sizeof(int), st));
        batch_round_decide_kernel<<<gp, 256, 0, st>>>(dpd, o, nprob, round + 1 < max_outer ? 1 : 0);
        count_launch(2);
        BDDA_CUDA_TRY(cudaGetLastError());
        int more = 0;
        BDDA_CUDA_TRY(cudaMemcpyAsync(&more, o.counters + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        BDDA_CUDA_TRY(cudaStreamSynchronize(st));
        if (more == 0) break;
      }
    }
    batch_outflag_kernel<<<gp, 256, 0, st>>>(o, nprob);
    count_launch();
    BTRY(e.list_build(f_out, 0, 0));
    return e.elem(esite(EL_OUT), E_CONVERT_OUT);
  }();
  if (gexec) cudaGraphExecDestroy(gexec);
  if (graph) cudaGraphDestroy(graph);
  if (rc != BDDA_OK) return rc;
  BDDA_CUDA_TRY(cudaMemcpyAsync(status, o.status, np * sizeof(int), cudaMemcpyDeviceToHost, st));
  BDDA_CUDA_TRY(cudaMemcpyAsync(iter_fin, o.iter_fin, np * sizeof(int), cudaMemcpyDeviceToHost, st));
  BDDA_CUDA_TRY(cudaMemcpyAsync(err_fin, o.err_fin, np * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (history && itermax > 0)
    BDDA_CUDA_TRY(cudaMemcpyAsync(history, o.hist, np * itermax * sizeof(double), cudaMemcpyDeviceToHost, st));
  BDDA_CUDA_TRY(cudaStreamSynchronize(st));
  int worst = BDDA_OK;
  for (int i = 0; i < nprob; ++i) {
    if (status[i] == BDDA_BREAKDOWN) worst = BDDA_BREAKDOWN;
    else if (status[i] != BDDA_OK && worst == BDDA_OK) worst = BDDA_NOT_CONVERGED;
  }
  return worst;
}

}  // namespace
}  // namespace bdda

using namespace bdda;

extern "C" {

size_t bdda_batch_workspace_bytes(const bdda_batch_problem* problems, int nprob, int mode, int L, int itermax) {
  if (check_problems(problems, nprob, mode, L) == BDDA_BAD_ARG || itermax < 0) return 0;
  BatchLayout lay;
  if (make_layout(problems, nprob, mode, L, itermax, &lay) != BDDA_OK) return 0;
  return lay.bytes;
}

int bdda_batch_bicgstab(const bdda_batch_problem* problems, int nprob, int mode, int L, double tol, int itermax,
                        int max_outer, int use_graph, int* status, int* iter_fin, double* err_fin, double* history,
                        void* work, size_t work_bytes, void* stream) {
  const int c = check_problems(problems, nprob, mode, L);
  if (c != BDDA_OK) return c;
  if (itermax < 0 || !(tol > 0.0) || !status || !iter_fin || !err_fin) return BDDA_BAD_ARG;
  if (mode == BDDA_BATCH_MIXED && max_outer < 1) return BDDA_BAD_ARG;
  BatchLayout lay;
  if (make_layout(problems, nprob, mode, L, itermax, &lay) != BDDA_OK) return BDDA_BAD_ARG;
  if (!work || work_bytes < lay.bytes) return BDDA_NO_WORKSPACE;
  unsigned char* w = static_cast<unsigned char*>(work);
  cudaStream_t user = static_cast<cudaStream_t>(stream);
  // an own stream, ordered after the caller's: a graph cannot capture the legacy stream
  cudaStream_t st = nullptr;
  cudaEvent_t ev = nullptr;
  BDDA_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaStreamDestroy(st);
    return BDDA_CUDA_ERROR;
  }
  int rc = BDDA_CUDA_ERROR;
  if (cudaEventRecord(ev, user) == cudaSuccess && cudaStreamWaitEvent(st, ev, 0) == cudaSuccess) {
    rc = mode == BDDA_BATCH_C64
             ? batch_run<float2>(problems, nprob, mode, L, tol, itermax, max_outer, use_graph, status, iter_fin,
                                 err_fin, history, w, lay, st)
             : batch_run<double2>(problems, nprob, mode, L, tol, itermax, max_outer, use_graph, status, iter_fin,
                                  err_fin, history, w, lay, st);
  }
  cudaEventRecord(ev, st);
  cudaStreamWaitEvent(user, ev, 0);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  cudaEventDestroy(ev);
  return rc;
}

}  // extern "C"
