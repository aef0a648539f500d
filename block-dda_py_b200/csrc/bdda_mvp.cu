// Doubled-grid FFT matrix-vector product of block-DDA on sm_100a.
//
// One block MVP is five pencil passes over a field buffer F of shape
// (Nx, My, Mz, 3L) (x natural; y, z spectra in digit-reversed order):
//   Z   : gather S through the occupancy map, forward z-FFT   (Nx*Ny pencils)
//   Y   : forward y-FFT, Ny rows in, My out                    (Nx*Mz pencils)
//   X   : forward x-FFT, 3x3 symmetric Green multiply, inverse (My*Mz pencils)
//   Y^-1: inverse y-FFT, My rows in, Ny out                    (Nx*Mz pencils)
//   Z^-1: inverse z-FFT, crop, diagonal + Jacobi epilogue, scatter back
// which is the reference's pad -> fftn -> Au_til @ P~ -> ifftn -> crop ->
// gather (mvp_fft/mvp_fft.py:151-169, bl_krylov/bl_krylov.py:47-55) with
// the zero rows never read and the rows that are cropped never written.
#include <climits>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <algorithm>
#include <mutex>
#include <vector>

#include "bdda_internal.h"

#include "bdda_blas.cuh"
#include "bdda_fixed.cuh"
#include "bdda_pencil.cuh"

namespace bdda {

// Generic pencil kernel, one item per CTA.
template <typename T, int KIND, int LT>
__global__ void __launch_bounds__(256) pencil_kernel(const PassArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  generic_pencil<T, KIND, LT>(a, blockIdx.x, smraw);
}

// The same with the tile's source rows brought in by a bulk tensor copy
// (make_tile_map), issued by one thread before the constants are staged.
template <typename T, int KIND, int LT>
__global__ void __launch_bounds__(256) pencil_tma_kernel(const PassArgs a, const __grid_constant__ CUtensorMap tm,
                                                         const TmaTile tt) {
  extern __shared__ __align__(128) unsigned char smraw[];
  // the copy's destination must be 128-byte aligned; dynamic shared memory of
  // a kernel without static shared memory starts on a wider boundary, so a
  // miss is an error (counted like a wait that gave up), not a slower path
  if ((smem_u32(pencil_tile<T, LT>(smraw, a.ax.M)) & 127) != 0) {
    if (threadIdx.x == 0 && a.err) atomicAdd(a.err, 1u);
    return;
  }
  if (threadIdx.x == 0) tma_issue<T, KIND, LT>(a, &tm, tt, smraw, a.ax.M, blockIdx.x);
  generic_pencil<T, KIND, LT, 2>(a, blockIdx.x, smraw);
}

template <typename T>
static size_t pencil_smem(int M, int LT, int kind) {
  return (size_t)pencil_smem_bytes<T>(M, LT, kind);
}

// Launch shape of the pencil passes, per precision (0 c128, 1 c64) and pass
// kind: the shared-memory budget per CTA (the widest column tile that fits is
// used) and the threads per CTA.  Set by bdda_tune_set.
static size_t g_tile_smem_budget[2][3] = {{80 * 1024, 80 * 1024, 80 * 1024},
                                          {80 * 1024, 80 * 1024, 80 * 1024}};
static int g_threads[2][3] = {{256, 256, 256}, {256, 256, 256}};
static_assert(K_FWD == 0 && K_CONV == 1 && K_INV == 2, "tuning tables are indexed by pass kind");

// Per-pass launch choices set by the autotuner (bdda_tune_pass), keyed by
// precision, pass kind, axis length and L: the column tile width lt (0 = the
// shared-memory budget rule) and the kernel variant (0 = the first
// specialised kernel compiled, k > 0 = the one with that id in the tables:
// register bound, CTA size and column pairs as bdda_fixed.cuh numbers them,
// -1 = the generic kernel).
struct PassTune { int prec, kind, M, L, lt, variant; };
static std::vector<PassTune> g_pass_tune;
static std::mutex g_tune_mu;

static PassTune pass_tune(int prec, int kind, int M, int L) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (const auto& e : g_pass_tune)
    if (e.prec == prec && e.kind == kind && e.M == M && e.L == L) return e;
  return PassTune{prec, kind, M, L, 0, 0};
}

static void set_pass_tune(const PassTune& t) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (auto& e : g_pass_tune)
    if (e.prec == t.prec && e.kind == t.kind && e.M == t.M && e.L == t.L) { e = t; return; }
  g_pass_tune.push_back(t);
}

template <typename T>
static int pick_lt(int M, int L, int kind) {
  const PassTune t = pass_tune(prec_of<T>(), kind, M, L);
  if (t.lt > 0 && pencil_smem<T>(M, t.lt, kind) <= 227 * 1024) return t.lt;
  const int cand[3] = {8, 4, 2};
  for (int lt : cand) {
    if (lt > 2 && lt / 2 >= L) continue;
    if (pencil_smem<T>(M, lt, kind) <= g_tile_smem_budget[prec_of<T>()][kind]) return lt;
  }
  return 2;
}

template <typename T, int KIND, int LT>
static int launch_lt(PassArgs a, int64_t P0, cudaStream_t st, bool tma = false) {
  a.ntile = (a.L + LT - 1) / LT;
  const size_t smem = pencil_smem<T>(a.ax.M, LT, KIND);
  if (smem > 227 * 1024) return BDDA_BAD_ARG;
  const int64_t nblk = P0 * a.P1 * a.ntile;
  if (nblk <= 0) return BDDA_OK;
  if (nblk > INT_MAX) return BDDA_BAD_ARG;
  CUtensorMap tm;
  TmaTile tt;
  memset(&tm, 0, sizeof(tm));
  memset(&tt, 0, sizeof(tt));
  if (tma && make_tile_map<T, KIND, LT>(a, P0, a.n_in, &tm, &tt)) {
    auto kern = pencil_tma_kernel<T, KIND, LT>;
    BDDA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<(unsigned)nblk, g_threads[prec_of<T>()][KIND], smem, st>>>(a, tm, tt);
  } else {
    auto kern = pencil_kernel<T, KIND, LT>;
    BDDA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<(unsigned)nblk, g_threads[prec_of<T>()][KIND], smem, st>>>(a);
  }
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BDDA_OK;
}

static int g_use_fixed = 1;   // specialised kernels on (bdda_tune_fixed)

static constexpr int kFixedTables = 10;

static const FixedKernel* fixed_table(int t, int* n) {
  switch (t) {
    case 0: return fixed_table_a(n);
    case 1: return fixed_table_b(n);
    case 2: return fixed_table_c(n);
    case 3: return fixed_table_d(n);
    case 4: return fixed_table_e(n);
    case 5: return fixed_table_f(n);
    case 6: return fixed_table_g(n);
    case 7: return fixed_table_h(n);
    case 8: return fixed_table_i(n);
    default: return fixed_table_j(n);
  }
}

// Column-pair kernels read and write two complex64 values per access: L
// even, every field pointer of the pass 16-byte aligned.
static bool pair_ok(const PassArgs& a) {
  auto al = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  return (a.L % 2) == 0 && al(a.src) && al(a.dst) && al(a.S);
}

// Specialised kernel for (precision, kind, tile width, radix sequence);
// variant as in PassTune; column-pair kernels only if pairs (pair_ok).
static FixedLaunchFn fixed_find(int prec, int kind, int lt, const AxisFFT& ax, int variant, bool pairs) {
  if (!g_use_fixed || variant < 0 || ax.nst > 4) return nullptr;
  int r[4] = {1, 1, 1, 1};
  for (int s = 0; s < ax.nst; ++s) r[s] = ax.rad[s];
  FixedLaunchFn first = nullptr;
  for (int t = 0; t < kFixedTables; ++t) {
    int n = 0;
    const FixedKernel* tab = fixed_table(t, &n);
    for (int i = 0; i < n; ++i) {
      const FixedKernel& f = tab[i];
      if (f.prec == prec && f.kind == kind && f.lt == lt && f.r[0] == r[0] && f.r[1] == r[1] &&
          f.r[2] == r[2] && f.r[3] == r[3] && (pairs || !f.pair)) {
        if (variant == 0 || f.variant == variant) return f.fn;
        if (!first) first = f.fn;
      }
    }
  }
  return first;
}

// Register-bound variants compiled for (precision, kind, tile width, radix sequence).
static std::vector<int> fixed_variants(int prec, int kind, int lt, const AxisFFT& ax, bool pairs) {
  std::vector<int> out;
  if (ax.nst > 4) return out;
  int r[4] = {1, 1, 1, 1};
  for (int s = 0; s < ax.nst; ++s) r[s] = ax.rad[s];
  for (int t = 0; t < kFixedTables; ++t) {
    int n = 0;
    const FixedKernel* tab = fixed_table(t, &n);
    for (int i = 0; i < n; ++i) {
      const FixedKernel& f = tab[i];
      if (f.prec == prec && f.kind == kind && f.lt == lt && f.r[0] == r[0] && f.r[1] == r[1] &&
          f.r[2] == r[2] && f.r[3] == r[3] && (pairs || !f.pair))
        out.push_back(f.variant);
    }
  }
  return out;
}

// Generic kernels: variant -1 with the first stage's global loads, -2 with the
// TMA-filled tile; with no choice made (variant 0) and no specialised kernel
// for the radix sequence, the TMA-filled one where the pass allows it.
template <typename T, int KIND>
static int launch_pass(const PassArgs& a, int64_t P0, int lt, cudaStream_t st) {
  int variant = 0;
  if (!a.green) {
    variant = pass_tune(prec_of<T>(), KIND, a.ax.M, a.L).variant;
    FixedLaunchFn f = fixed_find(prec_of<T>(), KIND, lt, a.ax, variant, pair_ok(a));
    if (f) return f(a, P0, st);
  }
  const bool tma = variant != -1 && g_use_fixed;
  switch (lt) {
    case 16:   // tile width 16 exists as specialised kernels only
    case 8: return launch_lt<T, KIND, 8>(a, P0, st, tma);
    case 4: return launch_lt<T, KIND, 4>(a, P0, st, tma);
    default: return launch_lt<T, KIND, 2>(a, P0, st, tma);
  }
}

template <typename T> struct TwOff;
template <> struct TwOff<double2> { static size_t get(const bdda_plan* p, int ax) { return p->tw64_off[ax]; } };
template <> struct TwOff<float2> { static size_t get(const bdda_plan* p, int ax) { return p->tw32_off[ax]; } };

#define BDDA_TRY(expr)               \
  do {                               \
    int s_ = (expr);                 \
    if (s_ != BDDA_OK) return s_;    \
  } while (0)

// Arguments of the five passes of one product (without launch shape) and
// the pencil-index extent P0 of each: Z, Y, X, Y^-1, Z^-1.
template <typename T>
void mvp_pass_args(const bdda_plan* plan, int L, const T* ghat, const int32_t* cell_map, const T* src,
                   const T* diag, const T* jpre, T* out, T* F, PassArgs a[5], int64_t P0[5]) {
  const int64_t Nx = plan->n[0], Ny = plan->n[1], Nz = plan->n[2];
  const int64_t Mx = plan->ax[0].M, My = plan->ax[1].M, Mz = plan->ax[2].M;
  const int64_t C = 3 * (int64_t)L;
  PassArgs b;
  memset(&b, 0, sizeof(b));
  b.L = L;
  b.C = C;
  b.scale = 1.0;
  b.err = plan_err(plan);
  {  // Z: gather + forward z
    PassArgs& q = a[0];
    q = b;
    q.ax = plan->ax[2]; q.tw = table_ptr<T>(plan, TwOff<T>::get(plan, 2));
    q.n_in = (int)Nz; q.n_out = (int)Mz; q.P1 = (int)Ny;
    q.cell_map = cell_map; q.cell_p0 = Ny * Nz; q.cell_p1 = Nz;
    q.S = src;
    q.src = src; q.src_p0 = Ny * Nz * C; q.src_p1 = Nz * C; q.src_row = C;   // dense cuboid input
    q.dst = F; q.dst_p0 = My * Mz * C; q.dst_p1 = Mz * C; q.dst_row = C;
    P0[0] = Nx;
  }
  PassArgs ay = b;  // Y and Y^-1 share the pencil geometry
  ay.ax = plan->ax[1]; ay.tw = table_ptr<T>(plan, TwOff<T>::get(plan, 1));
  ay.P1 = (int)Mz; ay.src = F; ay.dst = F;
  ay.src_p0 = ay.dst_p0 = My * Mz * C; ay.src_p1 = ay.dst_p1 = C; ay.src_row = ay.dst_row = Mz * C;
  a[1] = ay;
  a[1].n_in = (int)Ny; a[1].n_out = (int)My;
  P0[1] = Nx;
  {  // X: forward, Green multiply, inverse
    PassArgs& q = a[2];
    q = b;
    q.ax = plan->ax[0]; q.tw = table_ptr<T>(plan, TwOff<T>::get(plan, 0));
    q.n_in = (int)Nx; q.n_out = (int)Nx; q.P1 = (int)Mz;
    q.src = F; q.dst = F;
    q.src_p0 = q.dst_p0 = Mz * C; q.src_p1 = q.dst_p1 = C; q.src_row = q.dst_row = My * Mz * C;
    q.ghat = ghat;
    P0[2] = My;
  }
  a[3] = ay;
  a[3].n_in = (int)My; a[3].n_out = (int)Ny;
  P0[3] = Nx;
  {  // Z^-1 + crop + epilogue
    PassArgs& q = a[4];
    q = b;
    q.ax = plan->ax[2]; q.tw = table_ptr<T>(plan, TwOff<T>::get(plan, 2));
    q.n_in = (int)Mz; q.n_out = (int)Nz; q.P1 = (int)Ny;
    q.src = F; q.src_p0 = My * Mz * C; q.src_p1 = Mz * C; q.src_row = C;
    q.cell_map = cell_map; q.cell_p0 = Ny * Nz; q.cell_p1 = Nz;
    q.S = src; q.diag = diag; q.jpre = jpre;
    q.dst = out; q.dst_p0 = Ny * Nz * C; q.dst_p1 = Nz * C; q.dst_row = C;   // dense cuboid output
    q.scale = 1.0 / (double)(Mx * My * Mz);
    P0[4] = Nx;
  }
}
template void mvp_pass_args<double2>(const bdda_plan*, int, const double2*, const int32_t*, const double2*,
                                     const double2*, const double2*, double2*, double2*, PassArgs*, int64_t*);
template void mvp_pass_args<float2>(const bdda_plan*, int, const float2*, const int32_t*, const float2*,
                                    const float2*, const float2*, float2*, float2*, PassArgs*, int64_t*);

// The five passes.  cell_map == nullptr: dense cuboid in and out, no epilogue
// (fft_mvp); otherwise the sparse block MVP with diagonal and Jacobi scaling.
template <typename T>
static int run_mvp(const bdda_plan* plan, int L, const T* ghat, const int32_t* cell_map,
                   const T* src, const T* diag, const T* jpre, T* out, T* F, cudaStream_t st,
                   cudaEvent_t* ev = nullptr, bool wide = false) {
  PassArgs a[5];
  int64_t P0[5];
  mvp_pass_args<T>(plan, L, ghat, cell_map, src, diag, jpre, out, F, a, P0);
  if (wide) a[0].wide = a[4].wide = 1;   // src and out are complex128 (complex64 passes)
  const bool prof = profiling();
  if (prof) profile_mark(0, st, prec_of<T>());
  if (ev) BDDA_CUDA_TRY(cudaEventRecord(ev[0], st));
  for (int q = 0; q < 5; ++q) {
    const int kind = kPassKind[q];
    const int lt = pick_lt<T>(a[q].ax.M, L, kind);
    if (kind == K_FWD) BDDA_TRY((launch_pass<T, K_FWD>(a[q], P0[q], lt, st)));
    else if (kind == K_CONV) BDDA_TRY((launch_pass<T, K_CONV>(a[q], P0[q], lt, st)));
    else BDDA_TRY((launch_pass<T, K_INV>(a[q], P0[q], lt, st)));
    if (prof) profile_mark(q + 1, st);
    if (ev) BDDA_CUDA_TRY(cudaEventRecord(ev[q + 1], st));
  }
  return BDDA_OK;
}

template <typename T>
int block_mvp_impl(const bdda_plan* plan, int L, const T* ghat, const int32_t* cell_map,
                   const T* diag, const T* jpre, const T* S, T* out, T* work, cudaStream_t st) {
  return run_mvp<T>(plan, L, ghat, cell_map, S, diag, jpre, out, work, st);
}
int block_mvp_wide(const bdda_plan* plan, int L, const float2* ghat, const int32_t* cell_map, const float2* diag,
                   const float2* jpre, const double2* S, double2* out, float2* work, cudaStream_t st) {
  if (!cell_map) return BDDA_BAD_ARG;
  return run_mvp<float2>(plan, L, ghat, cell_map, reinterpret_cast<const float2*>(S), diag, jpre,
                         reinterpret_cast<float2*>(out), work, st, nullptr, true);
}

template int block_mvp_impl<double2>(const bdda_plan*, int, const double2*, const int32_t*,
                                     const double2*, const double2*, const double2*, double2*,
                                     double2*, cudaStream_t);
template int block_mvp_impl<float2>(const bdda_plan*, int, const float2*, const int32_t*,
                                    const float2*, const float2*, const float2*, float2*, float2*,
                                    cudaStream_t);

// ---- autotuner -----------------------------------------------------------------
// Times every launch choice of each pass of one block MVP (tile width x
// kernel variant) on the caller's buffers and keeps the fastest per
// (precision, kind, axis length, L).  All passes advance through their
// candidate lists together, one block MVP per round, each pass timed by its
// own pair of events; passes that share a key add their times.
template <typename T>
static int autotune_impl(const bdda_plan* p, int L, const T* ghat, const int32_t* cmap, const T* diag,
                         const T* jpre, const T* S, T* out, T* work, cudaStream_t st, int reps,
                         double* ms_before, double* ms_after) {
  const int prec = prec_of<T>();
  const int pass_kind[5] = {K_FWD, K_FWD, K_CONV, K_INV, K_INV};
  const int pass_axis[5] = {2, 1, 0, 1, 2};
  struct Key {
    int kind, axis;
    std::vector<PassTune> cand;
    std::vector<double> ms;
  };
  std::vector<Key> keys;
  int key_of[5];
  PassArgs pa[5];
  int64_t pp0[5];
  mvp_pass_args<T>(p, L, ghat, cmap, S, diag, jpre, out, work, pa, pp0);
  for (int q = 0; q < 5; ++q) {
    const int M = p->ax[pass_axis[q]].M;
    int k = -1;
    for (size_t i = 0; i < keys.size(); ++i)
      if (keys[i].kind == pass_kind[q] && p->ax[keys[i].axis].M == M) k = (int)i;
    if (k < 0) {
      Key key;
      key.kind = pass_kind[q];
      key.axis = pass_axis[q];
      for (int lt : {16, 8, 4, 2}) {
        if (lt > 2 && lt / 2 >= L) continue;
        if (pencil_smem<T>(M, lt, key.kind) > 227 * 1024) continue;
        for (int v : fixed_variants(prec, key.kind, lt, p->ax[key.axis], pair_ok(pa[q])))
          key.cand.push_back({prec, key.kind, M, L, lt, v});
        if (lt <= 8) {   // generic kernels go up to 8: global loads, TMA-filled tile
          key.cand.push_back({prec, key.kind, M, L, lt, -1});
          key.cand.push_back({prec, key.kind, M, L, lt, -2});
        }
      }
      key.ms.assign(key.cand.size(), 0.0);
      keys.push_back(key);
      k = (int)keys.size() - 1;
    }
    key_of[q] = k;
  }
  size_t rounds = 0;
  for (const auto& k : keys) rounds = std::max(rounds, k.cand.size());
  std::vector<cudaEvent_t> ev(6);
  for (auto& e : ev) BDDA_CUDA_TRY(cudaEventCreate(&e));
  auto timed = [&](double pass_ms[5]) -> int {
    for (int q = 0; q < 5; ++q) pass_ms[q] = 0.0;
    BDDA_TRY(run_mvp<T>(p, L, ghat, cmap, S, diag, jpre, out, work, st));   // warm-up
    for (int r = 0; r < reps; ++r) {
      BDDA_TRY(run_mvp<T>(p, L, ghat, cmap, S, diag, jpre, out, work, st, ev.data()));
      BDDA_CUDA_TRY(cudaEventSynchronize(ev[5]));
      for (int q = 0; q < 5; ++q) {
        float ms = 0.f;
        BDDA_CUDA_TRY(cudaEventElapsedTime(&ms, ev[q], ev[q + 1]));
        pass_ms[q] += ms / reps;
      }
    }
    return BDDA_OK;
  };
  double pm[5];
  int status = timed(pm);
  if (status == BDDA_OK && ms_before) *ms_before = pm[0] + pm[1] + pm[2] + pm[3] + pm[4];
  for (size_t r = 0; r < rounds && status == BDDA_OK; ++r) {
    for (auto& k : keys) set_pass_tune(k.cand[std::min(r, k.cand.size() - 1)]);
    status = timed(pm);
    for (int q = 0; q < 5 && status == BDDA_OK; ++q) {
      Key& k = keys[key_of[q]];
      if (r < k.cand.size()) k.ms[r] += pm[q];
    }
  }
  for (auto& k : keys) {
    if (k.cand.empty()) continue;
    size_t b = 0;
    for (size_t i = 1; i < k.ms.size(); ++i)
      if (k.ms[i] < k.ms[b]) b = i;
    set_pass_tune(k.cand[b]);
  }
  if (status == BDDA_OK) {
    status = timed(pm);
    if (status == BDDA_OK && ms_after) *ms_after = pm[0] + pm[1] + pm[2] + pm[3] + pm[4];
  }
  for (auto& e : ev) cudaEventDestroy(e);
  return status;
}

// ---- small helper kernels ----------------------------------------------------
__global__ void occupancy_kernel(const int64_t* address, int n_occ, int64_t nc, int32_t* cell_map) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n_occ) {
    const int64_t cell = address[m];
    if (cell >= 0 && cell < nc) cell_map[cell] = m;
  }
}

__global__ void convert_kernel(const double2* in, float2* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = make_float2((float)in[i].x, (float)in[i].y);
}

// Real-space A'(r) in natural order, (Mx, My, Mz, 3, 3) (mvp_fft/mvp_fft.py:13-94).
__global__ void green_real_kernel(PassArgs a, double2* out) {
  const int64_t total = (int64_t)a.gM[0] * a.gM[1] * a.gM[2];
  const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int iz = (int)(t % a.gM[2]);
    const int64_t q = t / a.gM[2];
    const int iy = (int)(q % a.gM[1]);
    const int ix = (int)(q / a.gM[1]);
    double2 g[6];
    green_row(a, ix, iy, iz, g);
    for (int c = 0; c < 6; ++c) {
      out[t * 9 + ia[c] * 3 + ib[c]] = g[c];
      out[t * 9 + ib[c] * 3 + ia[c]] = g[c];
    }
  }
}

struct GreenMap {
  int M[3];
  const int32_t* rev[3];
};

// library order [(py*Mz + pz)*Mx + px][6]  <->  natural (kx, ky, kz, 3, 3)
template <bool EXPORT>
__global__ void green_reorder_kernel(GreenMap g, const double2* in, double2* out) {
  const int64_t total = (int64_t)g.M[0] * g.M[1] * g.M[2];
  const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int px = (int)(t % g.M[0]);
    const int64_t q = t / g.M[0];
    const int pz = (int)(q % g.M[2]);
    const int py = (int)(q / g.M[2]);
    const int64_t nat = ((int64_t)g.rev[0][px] * g.M[1] + g.rev[1][py]) * g.M[2] + g.rev[2][pz];
    for (int c = 0; c < 6; ++c) {
      if (EXPORT) {
        const double2 v = in[t * 6 + c];
        out[nat * 9 + ia[c] * 3 + ib[c]] = v;
        out[nat * 9 + ib[c] * 3 + ia[c]] = v;
      } else {
        out[t * 6 + c] = in[nat * 9 + ia[c] * 3 + ib[c]];
      }
    }
  }
}

static bool smooth7(int m) {
  for (int p : {2, 3, 5, 7})
    while (m % p == 0) m /= p;
  return m == 1;
}

// Radices with register kernels, largest first, and the caps the kernels
// are compiled with (RadixCap): any stage <= kStageCap, the X-pass axis'
// last stage (fused with the Green multiply) <= kMidCap.
static const int kRadices[] = {16, 14, 12, 10, 9, 8, 7, 6, 5, 4, 3, 2};
static const int kStageCap = 10;
static const int kMidCap = 4;

static void enum_factorizations(int m, int maxr, std::vector<int>& cur, std::vector<std::vector<int>>& out) {
  if (m == 1) { out.push_back(cur); return; }
  if ((int)cur.size() >= 6) return;
  for (int r : kRadices)
    if (r <= maxr && m % r == 0) {
      cur.push_back(r);
      enum_factorizations(m / r, r, cur, out);
      cur.pop_back();
    }
}

// Fewest stages first, then the most balanced sequence (smallest largest
// radix); radices run largest first.  The X-pass axis (conv) keeps its last
// radix <= kMidCap so the fused middle (3 components x R frequencies on
// registers) stays small.  Returns the stage count (0: no factorization).
static int best_factorization(int M, bool conv, std::vector<int>& best) {
  std::vector<std::vector<int>> all;
  std::vector<int> cur;
  enum_factorizations(M, kStageCap, cur, all);
  int best_key = INT_MAX;
  best.clear();
  for (const auto& f : all) {
    if (conv && f.back() > kMidCap) continue;
    const int key = (int)f.size() * 64 + f.front();
    if (key < best_key) { best_key = key; best = f; }
  }
  return (int)best.size();
}

static int factor_axis(int M, bool conv, AxisFFT& ax) {
  std::vector<int> r;
  if (M == 1) {
    r.clear();
  } else if (best_factorization(M, conv, r) == 0 || (int)r.size() > kMaxStages) {
    return BDDA_BAD_ARG;
  }
  ax.M = M;
  ax.nst = (int)r.size();
  int B = M;
  for (int s = 0; s < ax.nst; ++s) { ax.rad[s] = r[s]; ax.blk[s] = B; B /= r[s]; }
  for (int s = ax.nst; s < kMaxStages; ++s) { ax.rad[s] = 1; ax.blk[s] = 1; }
  return BDDA_OK;
}

// Cyclic length for a cuboid side N: the even 7-smooth M >= 2N minimising
// M x (1 + 1/4 per radix stage beyond the first), searched up to 2N + 2N/4.
static int choose_length(int N, bool conv) {
  int best = -1;
  double best_cost = 1e300;
  for (int M = 2 * N; M <= 2 * N + (2 * N) / 4 + 2; M += 2) {
    if (!smooth7(M)) continue;
    std::vector<int> f;
    const int ns = best_factorization(M, conv, f);
    if (ns == 0) continue;
    const double cost = M * (1.0 + 0.25 * (ns - 1));
    if (cost < best_cost) { best_cost = cost; best = M; }
  }
  if (best < 0) {
    best = 2 * N;
    while (!smooth7(best)) best += 2;
  }
  return best;
}

}  // namespace bdda

using namespace bdda;

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

extern "C" {

const char* bdda_status_string(int s) {
  switch (s) {
    case BDDA_OK: return "ok";
    case BDDA_NOT_CONVERGED: return "not converged";
    case BDDA_BREAKDOWN: return "breakdown: singular or non-finite small system";
    case BDDA_BAD_ARG: return "bad argument";
    case BDDA_NO_WORKSPACE: return "workspace or plan tables missing";
    case BDDA_TIMEOUT: return "device wait timed out";
    case BDDA_CUDA_ERROR: return "CUDA runtime error";
    default: return "unknown status";
  }
}

int bdda_version(void) { return 100; }

int bdda_tune_set(int prec, int kind, size_t smem_budget, int threads) {
  if (prec < 0 || prec > 1 || kind < 0 || kind > 2 || threads < 32 || threads > 512 || (threads & 31) ||
      smem_budget < 1024 || smem_budget > 227 * 1024)
    return BDDA_BAD_ARG;
  g_tile_smem_budget[prec][kind] = smem_budget;
  g_threads[prec][kind] = threads;
  return BDDA_OK;
}

int bdda_tune_pass(int prec, int kind, int M, int L, int lt, int variant) {
  if (prec < 0 || prec > 1 || kind < 0 || kind > 2 || M < 1 || L < 1 || L > kMaxL ||
      (lt != 0 && lt != 2 && lt != 4 && lt != 8 && lt != 16) || variant < -2 || variant >= 4096)
    return BDDA_BAD_ARG;
  set_pass_tune({prec, kind, M, L, lt, variant});
  return BDDA_OK;
}

int bdda_tune_pass_get(int prec, int kind, int M, int L, int* lt, int* variant) {
  if (!lt || !variant) return BDDA_BAD_ARG;
  const PassTune t = pass_tune(prec, kind, M, L);
  *lt = t.lt;
  *variant = t.variant;
  return BDDA_OK;
}

int bdda_tune_pass_variants(const bdda_plan* plan, int prec, int kind, int axis, int lt, int* variants, int cap,
                            int* n) {
  if (!plan || !n || prec < 0 || prec > 1 || kind < 0 || kind > 2 || axis < 0 || axis > 2 || cap < 0 ||
      (cap > 0 && !variants))
    return BDDA_BAD_ARG;
  const std::vector<int> v = fixed_variants(prec, kind, lt, plan->ax[axis], true);
  *n = (int)v.size();
  for (int i = 0; i < (int)v.size() && i < cap; ++i) variants[i] = v[i];
  return BDDA_OK;
}

int bdda_autotune(const bdda_plan* plan, int prec, int L, const void* ghat, const int32_t* cell_map,
                  const void* diag, const void* jpre, const void* S, void* out, void* work, int reps,
                  double* ms_before, double* ms_after, void* stream) {
  if (!plan || L < 1 || L > kMaxL || reps < 1 || !ghat || !cell_map || !diag || !jpre || !S || !out)
    return BDDA_BAD_ARG;
  if (!plan->dev_tables || !work) return BDDA_NO_WORKSPACE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (prec == BDDA_C128)
    return autotune_impl<double2>(plan, L, static_cast<const double2*>(ghat), cell_map,
                                  static_cast<const double2*>(diag), static_cast<const double2*>(jpre),
                                  static_cast<const double2*>(S), static_cast<double2*>(out),
                                  static_cast<double2*>(work), st, reps, ms_before, ms_after);
  if (prec == BDDA_C64)
    return autotune_impl<float2>(plan, L, static_cast<const float2*>(ghat), cell_map,
                                 static_cast<const float2*>(diag), static_cast<const float2*>(jpre),
                                 static_cast<const float2*>(S), static_cast<float2*>(out),
                                 static_cast<float2*>(work), st, reps, ms_before, ms_after);
  return BDDA_BAD_ARG;
}

int bdda_tune_fixed(int on) {
  g_use_fixed = on ? 1 : 0;
  set_fixed_blas(on);
  return BDDA_OK;
}

int bdda_tune_get(int prec, int kind, size_t* smem_budget, int* threads) {
  if (prec < 0 || prec > 1 || kind < 0 || kind > 2 || !smem_budget || !threads) return BDDA_BAD_ARG;
  *smem_budget = g_tile_smem_budget[prec][kind];
  *threads = g_threads[prec][kind];
  return BDDA_OK;
}

int bdda_plan_create(const int n[3], const int m[3], bdda_plan** out) {
  if (!n || !out) return BDDA_BAD_ARG;
  bdda_plan* p = new bdda_plan();
  p->dev_tables = nullptr;
  for (int a = 0; a < 3; ++a) {
    if (n[a] < 1 || n[a] > 16384) { delete p; return BDDA_BAD_ARG; }
    p->n[a] = n[a];
    int M;
    if (m) {
      M = m[a];
      if (M < 2 * n[a] - 1 || M < 1 || !smooth7(M)) { delete p; return BDDA_BAD_ARG; }
    } else {
      M = choose_length(n[a], a == 0);
    }
    if (factor_axis(M, a == 0, p->ax[a]) != BDDA_OK) { delete p; return BDDA_BAD_ARG; }
  }
  // device tables: twiddles (both precisions) and position -> frequency maps
  size_t off = 0;
  for (int a = 0; a < 3; ++a) {
    const int M = p->ax[a].M;
    p->tw64_off[a] = off; off = align256(off + (size_t)M * sizeof(double2));
    p->tw32_off[a] = off; off = align256(off + (size_t)M * sizeof(float2));
    p->rev_off[a] = off;  off = align256(off + (size_t)M * sizeof(int32_t));
  }
  p->err_off = off; off = align256(off + sizeof(uint32_t));
  p->table_bytes = off;
  p->host_tables.assign(off, 0);
  for (int a = 0; a < 3; ++a) {
    const AxisFFT& ax = p->ax[a];
    const int M = ax.M;
    double2* t64 = reinterpret_cast<double2*>(p->host_tables.data() + p->tw64_off[a]);
    float2* t32 = reinterpret_cast<float2*>(p->host_tables.data() + p->tw32_off[a]);
    int32_t* rev = reinterpret_cast<int32_t*>(p->host_tables.data() + p->rev_off[a]);
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int k = 0; k < M; ++k) {
      const long double ang = twopi * (long double)k / (long double)M;
      const double c = (double)cosl(ang), s = -(double)sinl(ang);
      t64[k] = make_double2(c, s);
      t32[k] = make_float2((float)c, (float)s);
      // digit reversal of the DIF stage order: position digits (q0 q1 ...)
      // with position = q0*blk1 + q1*blk2 + ..., frequency = q0 + r0*(q1 + r1*(...))
      int rem = k, mult = 1, f = 0;
      for (int s2 = 0; s2 < ax.nst; ++s2) {
        const int span = ax.blk[s2] / ax.rad[s2];
        const int q = rem / span;
        rem -= q * span;
        f += q * mult;
        mult *= ax.rad[s2];
      }
      rev[k] = f;
    }
  }
  *out = p;
  return BDDA_OK;
}

void bdda_plan_destroy(bdda_plan* p) { delete p; }

int bdda_plan_grid(const bdda_plan* p, int m[3]) {
  if (!p || !m) return BDDA_BAD_ARG;
  for (int a = 0; a < 3; ++a) m[a] = p->ax[a].M;
  return BDDA_OK;
}

int bdda_plan_radices(const bdda_plan* p, int axis, int radices[12], int* nstage) {
  if (!p || axis < 0 || axis > 2 || !radices || !nstage) return BDDA_BAD_ARG;
  *nstage = p->ax[axis].nst;
  for (int s = 0; s < kMaxStages; ++s) radices[s] = s < p->ax[axis].nst ? p->ax[axis].rad[s] : 0;
  return BDDA_OK;
}

size_t bdda_plan_table_bytes(const bdda_plan* p) { return p ? p->table_bytes : 0; }

int bdda_plan_wait_timeouts(const bdda_plan* p, unsigned int* count, void* stream) {
  if (!p || !count) return BDDA_BAD_ARG;
  if (!p->dev_tables) return BDDA_NO_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  BDDA_CUDA_TRY(cudaMemcpyAsync(count, plan_err(p), sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
  BDDA_CUDA_TRY(cudaStreamSynchronize(st));
  return BDDA_OK;
}

int bdda_plan_attach_tables(bdda_plan* p, void* dev, void* stream) {
  if (!p || !dev || (reinterpret_cast<uintptr_t>(dev) & 15)) return BDDA_BAD_ARG;
  BDDA_CUDA_TRY(cudaMemcpyAsync(dev, p->host_tables.data(), p->table_bytes, cudaMemcpyHostToDevice,
                                (cudaStream_t)stream));
  // the host copy must not change before the upload completes
  BDDA_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  p->dev_tables = dev;
  return BDDA_OK;
}

size_t bdda_green_bytes(const bdda_plan* p, int prec) {
  return p ? (size_t)grid_points(p) * 6 * cplx_bytes(prec) : 0;
}

size_t bdda_green_build_workspace_bytes(const bdda_plan* p) {
  return p ? (size_t)grid_points(p) * 6 * sizeof(double2) : 0;
}

int bdda_green_build(const bdda_plan* p, double lf, double k, void* ghat, void* work, void* stream) {
  if (!p || !ghat) return BDDA_BAD_ARG;
  if (!work || !p->dev_tables) return BDDA_NO_WORKSPACE;
  if (!(lf > 0.0) || !std::isfinite(k)) return BDDA_BAD_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t Mx = p->ax[0].M, My = p->ax[1].M, Mz = p->ax[2].M;
  double2* G = static_cast<double2*>(work);
  PassArgs b;
  memset(&b, 0, sizeof(b));
  b.L = 2;   // 6 components = 3 "components" x 2 columns: the tile mapping is the identity
  b.C = 6;
  for (int a = 0; a < 3; ++a) { b.gN[a] = p->n[a]; b.gM[a] = p->ax[a].M; }
  b.lf = lf;
  b.k = k;
  b.scale = 1.0;
  {  // real-space tensor evaluated in the kernel, forward z
    PassArgs a = b;
    a.ax = p->ax[2]; a.tw = table_ptr<double2>(p, p->tw64_off[2]);
    a.n_in = a.n_out = (int)Mz; a.P1 = (int)My;
    a.green = 1;
    a.dst = G; a.dst_p0 = My * Mz * 6; a.dst_p1 = Mz * 6; a.dst_row = 6;
    BDDA_TRY((launch_lt<double2, K_FWD, 2>(a, Mx, st)));
  }
  {  // forward y
    PassArgs a = b;
    a.ax = p->ax[1]; a.tw = table_ptr<double2>(p, p->tw64_off[1]);
    a.n_in = a.n_out = (int)My; a.P1 = (int)Mz;
    a.src = G; a.dst = G;
    a.src_p0 = a.dst_p0 = My * Mz * 6; a.src_p1 = a.dst_p1 = 6; a.src_row = a.dst_row = Mz * 6;
    BDDA_TRY((launch_lt<double2, K_FWD, 2>(a, Mx, st)));
  }
  {  // forward x into the x-pencil-major spectrum
    PassArgs a = b;
    a.ax = p->ax[0]; a.tw = table_ptr<double2>(p, p->tw64_off[0]);
    a.n_in = a.n_out = (int)Mx; a.P1 = (int)Mz;
    a.src = G; a.src_p0 = Mz * 6; a.src_p1 = 6; a.src_row = My * Mz * 6;
    a.dst = ghat; a.dst_p0 = Mz * Mx * 6; a.dst_p1 = Mx * 6; a.dst_row = 6;
    BDDA_TRY((launch_lt<double2, K_FWD, 2>(a, My, st)));
  }
  return BDDA_OK;
}

int bdda_green_real(const bdda_plan* p, double lf, double k, void* full, void* stream) {
  if (!p || !full || !(lf > 0.0) || !std::isfinite(k)) return BDDA_BAD_ARG;
  PassArgs a;
  memset(&a, 0, sizeof(a));
  for (int d = 0; d < 3; ++d) { a.gN[d] = p->n[d]; a.gM[d] = p->ax[d].M; }
  a.lf = lf;
  a.k = k;
  green_real_kernel<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(a, static_cast<double2*>(full));
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BDDA_OK;
}

int bdda_green_convert(const bdda_plan* p, const void* g64, void* g32, void* stream) {
  if (!p || !g64 || !g32) return BDDA_BAD_ARG;
  const int64_t n = grid_points(p) * 6;
  convert_kernel<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(static_cast<const double2*>(g64),
                                                            static_cast<float2*>(g32), n);
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BDDA_OK;
}

static int green_reorder(const bdda_plan* p, const void* in, void* out, void* stream, bool exp) {
  if (!p || !in || !out) return BDDA_BAD_ARG;
  if (!p->dev_tables) return BDDA_NO_WORKSPACE;
  GreenMap g;
  for (int a = 0; a < 3; ++a) {
    g.M[a] = p->ax[a].M;
    g.rev[a] = table_ptr<int32_t>(p, p->rev_off[a]);
  }
  if (exp)
    green_reorder_kernel<true><<<148 * 8, 256, 0, (cudaStream_t)stream>>>(
        g, static_cast<const double2*>(in), static_cast<double2*>(out));
  else
    green_reorder_kernel<false><<<148 * 8, 256, 0, (cudaStream_t)stream>>>(
        g, static_cast<const double2*>(in), static_cast<double2*>(out));
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BDDA_OK;
}

int bdda_green_export(const bdda_plan* p, const void* ghat, void* full, void* stream) {
  return green_reorder(p, ghat, full, stream, true);
}

int bdda_green_import(const bdda_plan* p, const void* full, void* ghat, void* stream) {
  return green_reorder(p, full, ghat, stream, false);
}

size_t bdda_mvp_workspace_bytes(const bdda_plan* p, int prec, int L) {
  if (!p || L < 1) return 0;
  return (size_t)p->n[0] * p->ax[1].M * p->ax[2].M * 3 * (size_t)L * cplx_bytes(prec);
}

int bdda_occupancy_map(const bdda_plan* p, const int64_t* address, int n_occ, int32_t* cell_map,
                       void* stream) {
  if (!p || !cell_map || n_occ < 0 || (n_occ > 0 && !address)) return BDDA_BAD_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t nc = cells(p);
  BDDA_CUDA_TRY(cudaMemsetAsync(cell_map, 0xff, (size_t)nc * sizeof(int32_t), st));
  if (n_occ > 0) {
    occupancy_kernel<<<(n_occ + 255) / 256, 256, 0, st>>>(address, n_occ, nc, cell_map);
    BDDA_CUDA_TRY(cudaGetLastError());
    count_launch();
  }
  return BDDA_OK;
}

int bdda_fft_mvp(const bdda_plan* p, int prec, int L, const void* ghat, const void* P_full,
                 void* Y_full, void* work, void* stream) {
  if (!p || L < 1 || !ghat || !P_full || !Y_full) return BDDA_BAD_ARG;
  if (reinterpret_cast<uintptr_t>(ghat) & 15) return BDDA_BAD_ARG;   // staged with 16-byte async copies
  if (!work || !p->dev_tables) return BDDA_NO_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (prec == BDDA_C128)
    return run_mvp<double2>(p, L, static_cast<const double2*>(ghat), nullptr,
                            static_cast<const double2*>(P_full), nullptr, nullptr,
                            static_cast<double2*>(Y_full), static_cast<double2*>(work), st);
  if (prec == BDDA_C64)
    return run_mvp<float2>(p, L, static_cast<const float2*>(ghat), nullptr,
                           static_cast<const float2*>(P_full), nullptr, nullptr,
                           static_cast<float2*>(Y_full), static_cast<float2*>(work), st);
  return BDDA_BAD_ARG;
}

int bdda_block_mvp(const bdda_plan* p, int prec, int L, const void* ghat, const int32_t* cell_map,
                   const void* diag, const void* jpre, const void* S, void* out, void* work,
                   void* stream) {
  if (!p || L < 1 || !ghat || !cell_map || !diag || !jpre || !S || !out) return BDDA_BAD_ARG;
  if (reinterpret_cast<uintptr_t>(ghat) & 15) return BDDA_BAD_ARG;   // staged with 16-byte async copies
  if (!work || !p->dev_tables) return BDDA_NO_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (prec == BDDA_C128)
    return block_mvp_impl<double2>(p, L, static_cast<const double2*>(ghat), cell_map,
                                   static_cast<const double2*>(diag), static_cast<const double2*>(jpre),
                                   static_cast<const double2*>(S), static_cast<double2*>(out),
                                   static_cast<double2*>(work), st);
  if (prec == BDDA_C64)
    return block_mvp_impl<float2>(p, L, static_cast<const float2*>(ghat), cell_map,
                                  static_cast<const float2*>(diag), static_cast<const float2*>(jpre),
                                  static_cast<const float2*>(S), static_cast<float2*>(out),
                                  static_cast<float2*>(work), st);
  return BDDA_BAD_ARG;
}

}  // extern "C"
