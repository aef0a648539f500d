// Device code shared by the pencil-pass kernels: pass arguments, global row
// access of one pencil x column tile, radix-stage jobs, and the fused X-pass
// middle (last forward stage, Green multiply, first inverse stage).
//
// A CTA owns one pencil (a line of the grid along the transformed axis) and a
// column tile of LT right-hand sides x 3 components, staged in shared memory
// as [row][3 LT].  The first radix stage reads global memory directly and the
// last one writes it, so only the stages between round-trip through shared
// memory.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "bdda_internal.h"

namespace bdda {

enum PassKind { K_FWD = 0, K_CONV = 1, K_INV = 2 };

struct PassArgs {
  AxisFFT ax;
  int n_in, n_out;      // rows read (the rest are zero) / rows written
  int P1;               // pencil index p = p0 * P1 + p1
  int ntile;            // column tiles per pencil
  int L;                // right-hand sides
  int green;            // K_FWD: the rows are A'(r), evaluated in the kernel
  int64_t C;            // complex values per grid row (3L)
  int64_t src_p0, src_p1, src_row;
  int64_t dst_p0, dst_p1, dst_row;
  const void* src;
  void* dst;
  const void* tw;       // this axis' twiddles, M entries
  const int32_t* cell_map;   // K_FWD: gather S through it; K_INV: scatter with the epilogue
  int64_t cell_p0, cell_p1;
  const void* S;
  const void* diag;
  const void* jpre;
  double scale;         // K_INV: factor applied to the output (1/(Mx My Mz) in the last pass)
  const void* ghat;
  int gN[3], gM[3];
  double lf, k;
  unsigned int* err;    // bounded waits that gave up (the plan's counter; null: not counted)
  int wide;             // complex64 passes: S (Z gather, Z^-1 epilogue) and the Z^-1 output are complex128
};

// Element m of a complex128 array as complex64 (round to nearest) and back.
__device__ __forceinline__ float2 narrow_at(const void* p, int64_t i) {
  const double2 d = static_cast<const double2*>(p)[i];
  return make_float2((float)d.x, (float)d.y);
}
__device__ __forceinline__ void widen_to(void* p, int64_t i, float2 v) {
  static_cast<double2*>(p)[i] = make_double2((double)v.x, (double)v.y);
}

struct Pen {
  int64_t p0, p1;
  int tile;
  const void* srcb;      // pencil base of the source: src + p0 src_p0 + p1 src_p1
  void* dstb;            // pencil base of the destination
  const int32_t* cmap;   // this pencil's occupancy-map entries, staged in shared memory (or null)
};

__device__ __forceinline__ bool axis_disp(int I, int N, int M, int& d) {
  if (I <= N - 1) { d = I; return true; }
  if (I >= M - (N - 1)) { d = I - M; return true; }
  d = 0;
  return false;
}

// Six unique components of A'(r) at cyclic index (ix, iy, iz)
// (mvp_fft/mvp_fft.py:49-92 with the displacement map generalised to M >= 2N-1).
static __device__ void green_row(const PassArgs& a, int ix, int iy, int iz, double2* out) {
  int dx, dy, dz;
  const bool ok = axis_disp(ix, a.gN[0], a.gM[0], dx) & axis_disp(iy, a.gN[1], a.gM[1], dy) &
                  axis_disp(iz, a.gN[2], a.gM[2], dz);
  if (!ok || (dx == 0 && dy == 0 && dz == 0)) {
    for (int c = 0; c < 6; ++c) out[c] = make_double2(0.0, 0.0);
    return;
  }
  const double X = dx * a.lf, Y = dy * a.lf, Z = dz * a.lf;
  const double r = sqrt(X * X + Y * Y + Z * Z);
  const double u[3] = {X / r, Y / r, Z / r};
  double sn, cs;
  sincos(a.k * r, &sn, &cs);
  const double pr = cs / r, pim = sn / r;            // e^{ikr} / r
  const double nr = 1.0 / (r * r), ni = -a.k / r;    // (1 - ikr) / r^2
  const double k2 = a.k * a.k;
  const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    const double uu = u[ia[c]] * u[ib[c]];
    const double delta = (ia[c] == ib[c]) ? 1.0 : 0.0;
    const double q = delta - 3.0 * uu;
    const double tr = k2 * (uu - delta) + nr * q, ti = ni * q;
    out[c] = make_double2(pr * tr - pim * ti, pr * ti + pim * tr);
  }
}

// ---- asynchronous global -> shared copies (cp.async, 16-byte granules) ----
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// nbytes is a multiple of 8; both pointers are 16-byte aligned
__device__ __forceinline__ void async_copy(void* dst, const void* src, int nbytes) {
  const int n16 = nbytes >> 4;
  for (int i = threadIdx.x; i < n16; i += blockDim.x)
    cp_async16(static_cast<char*>(dst) + 16 * i, static_cast<const char*>(src) + 16 * i);
  if ((nbytes & 15) && threadIdx.x == 0)
    *reinterpret_cast<uint2*>(static_cast<char*>(dst) + 16 * n16) =
        *reinterpret_cast<const uint2*>(static_cast<const char*>(src) + 16 * n16);
}

__host__ __device__ __forceinline__ int align16(int x) { return (x + 15) & ~15; }
__host__ __device__ __forceinline__ int align128(int x) { return (x + 127) & ~127; }

template <typename T> constexpr int prec_of() { return std::is_same<T, double2>::value ? 0 : 1; }

// Shared memory of one pencil CTA: twiddles, the [row][3 LT] tile (128-byte
// aligned: a bulk tensor copy may fill it), the Green's pencil (X pass), the
// occupancy-map rows and one 8-byte transaction barrier.
template <typename T>
__host__ __device__ __forceinline__ int pencil_smem_bytes(int M, int LT, int kind) {
  return align128(M * (int)sizeof(T)) + align16(M * 3 * LT * (int)sizeof(T)) +
         (kind == K_CONV ? align16(M * 6 * (int)sizeof(T)) : 0) + align16(M * 4) + 16;
}

// Pencil and tile of a CTA (one item per CTA).
template <typename T>
__device__ __forceinline__ Pen pen_of_block(const PassArgs& a, const int32_t* cm, int64_t bid) {
  Pen c;
  c.tile = (int)(bid % a.ntile);
  const int64_t p = bid / a.ntile;
  c.p0 = p / a.P1;
  c.p1 = p - c.p0 * a.P1;
  c.srcb = static_cast<const T*>(a.src) + c.p0 * a.src_p0 + c.p1 * a.src_p1;
  c.dstb = static_cast<T*>(a.dst) + c.p0 * a.dst_p0 + c.p1 * a.dst_p1;
  c.cmap = a.cell_map ? cm : nullptr;
  return c;
}

// Shared-memory carve-up and the asynchronous staging of the twiddles (and,
// for the X pass, the Green's pencil).  Returns after the twiddles landed.
template <typename T, int KIND, int LT>
__device__ __forceinline__ unsigned char* pencil_barrier(unsigned char* smraw, int M) {
  return smraw + align128(M * (int)sizeof(T)) + align16(M * 3 * LT * (int)sizeof(T)) +
         (KIND == K_CONV ? align16(M * 6 * (int)sizeof(T)) : 0) + align16(M * 4);
}
template <typename T, int LT>
__device__ __forceinline__ T* pencil_tile(unsigned char* smraw, int M) {
  return reinterpret_cast<T*>(smraw + align128(M * (int)sizeof(T)));
}

template <typename T, int KIND, int LT>
__device__ __forceinline__ void stage_constants(const PassArgs& a, unsigned char* smraw, int M, T** tw, T** sm,
                                                T** gs, int32_t** cm, int64_t bid) {
  const int o_sm = align128(M * (int)sizeof(T));
  const int o_gs = o_sm + align16(M * 3 * LT * (int)sizeof(T));
  const int o_cm = o_gs + (KIND == K_CONV ? align16(M * 6 * (int)sizeof(T)) : 0);
  *tw = reinterpret_cast<T*>(smraw);
  *sm = reinterpret_cast<T*>(smraw + o_sm);
  *gs = reinterpret_cast<T*>(smraw + o_gs);
  *cm = reinterpret_cast<int32_t*>(smraw + o_cm);
  async_copy(*tw, a.tw, M * (int)sizeof(T));
  cp_async_commit();
  if constexpr (KIND == K_CONV) {
    const int64_t p = bid / a.ntile;
    async_copy(*gs, static_cast<const T*>(a.ghat) + p * (int64_t)M * 6, M * 6 * (int)sizeof(T));
  }
  cp_async_commit();
  if (a.cell_map) {   // the pencil's occupancy-map rows (Z and Z^-1 passes)
    const int64_t p = bid / a.ntile;
    const int64_t p0 = p / a.P1, p1 = p - p0 * a.P1;
    const int32_t* src = a.cell_map + p0 * a.cell_p0 + p1 * a.cell_p1;
    const int rows = KIND == K_INV ? a.n_out : a.n_in;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) (*cm)[i] = src[i];
  }
  cp_async_wait<1>();
  __syncthreads();
}



// ---- the tile's first read by a bulk tensor copy (TMA) ------------------------------------
// With TMA = 1 the pencil's source rows of the CTA's column tile come into the
// shared tile by one or two cp.async.bulk.tensor copies, issued by one thread
// before the constants are staged (all bytes in flight at once); the first
// radix stage then reads shared memory instead of issuing its own global
// loads.  The tensor map views the source field as (l, component, row, p1,
// p0), the last three ordered by stride, so a box lands as rows of the
// [row][3 LT] tile; rows at or past n_in and columns at or past L come back
// as zeros (out-of-bounds fill), as gload returns them.  The boxes cover the
// source rows [0, n_in) only; the first stage reads no row past them (those
// are zero).  Two boxes of box_rows rows start at rows 0 and n_in - box_rows
// (they may overlap by a row or two, written twice with the same bytes) so
// that each starts on a 128-byte boundary of the tile.  The copy completes on a transaction
// barrier; the wait is bounded, and a CTA that gives up counts the event in
// a.err, waits (bounded again) for its copy to land and returns.
struct TmaTile {
  int nbox, box_rows;
  int rows;        // tile rows the boxes cover: [0, rows)
  int dim_of[3];   // dimension 2 + d of the map holds (row, p1, p0)[dim_of[d]]
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, int limit) {
  for (int i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

constexpr int kTmaWaitLimit = 1 << 22;   // try_wait rounds: far beyond any copy's latency, but finite

template <typename T, int KIND, int LT>
__device__ __forceinline__ void tma_issue(const PassArgs& a, const CUtensorMap* tm, const TmaTile& tt,
                                          unsigned char* smraw, int M, int64_t bid) {
  constexpr int E = sizeof(T) / 8;   // 8-byte elements per complex value
  T* sm = pencil_tile<T, LT>(smraw, M);
  const uint32_t bar = smem_u32(pencil_barrier<T, KIND, LT>(smraw, M));
  const int tile = (int)(bid % a.ntile);
  const int64_t p = bid / a.ntile;
  const int64_t p0 = p / a.P1, p1 = p - p0 * a.P1;
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  const uint32_t bytes = (uint32_t)(tt.nbox * tt.box_rows * 3 * LT * (int)sizeof(T));
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
  for (int b = 0; b < tt.nbox; ++b) {
    const int row0 = b == 0 ? 0 : tt.rows - tt.box_rows;
    const int v[3] = {row0, (int)p1, (int)p0};
    int c[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) c[d] = v[tt.dim_of[d]];
    const uint32_t dst = smem_u32(sm + (size_t)row0 * 3 * LT);
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
        "%6}], [%7];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(tile * LT * E), "r"(0), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(bar)
        : "memory");
  }
}

// The same wait as done by every thread of a CTA that issued a tile copy:
// true when it landed; otherwise (the whole CTA decides together) the event
// is counted in a.err and the CTA must return without computing.
template <typename T, int KIND, int LT>
__device__ __forceinline__ bool tile_landed(const PassArgs& a, unsigned char* smraw, int M) {
  const uint32_t bar = smem_u32(pencil_barrier<T, KIND, LT>(smraw, M));
  const bool landed = mbar_wait_bounded(bar, 0, kTmaWaitLimit);
  if (__syncthreads_or(!landed)) {
    if (threadIdx.x == 0) {
      if (a.err) atomicAdd(a.err, 1u);
      mbar_wait_bounded(bar, 0, kTmaWaitLimit);   // the copy lands before the CTA's shared memory is released
    }
    return false;
  }
  return true;
}

// ---- global row access of one pencil x column tile ----
// Column col of the tile is right-hand side tile*LT + col%LT of component
// col/LT, i.e. grid column (col/LT)*L + tile*LT + col%LT.
template <int LT>
__device__ __forceinline__ int tile_gcol(const PassArgs& a, const Pen& c, int col, bool& ok) {
  const int comp = col / LT, l = c.tile * LT + (col - comp * LT);
  ok = l < a.L;
  return comp * a.L + l;
}

template <int KIND, typename T, int LT>
__device__ __forceinline__ T gload(const PassArgs& a, const Pen& c, int row, int col) {
  typedef typename real_of<T>::type F;
  bool ok;
  const int gcol = tile_gcol<LT>(a, c, col, ok);
  if (!ok || row >= a.n_in) return mkc<T>(F(0), F(0));
  if constexpr (KIND == K_FWD) {
    if (c.cmap) {
      const int m = c.cmap[row];
      if (m < 0) return mkc<T>(F(0), F(0));
      if constexpr (std::is_same<T, float2>::value) {
        if (a.wide) return narrow_at(a.S, (int64_t)m * a.C + gcol);
      }
      return static_cast<const T*>(a.S)[(int64_t)m * a.C + gcol];
    }
  }
  return static_cast<const T*>(c.srcb)[(int64_t)row * a.src_row + gcol];
}

template <int KIND, typename T, int LT>
__device__ __forceinline__ void gstore(const PassArgs& a, const Pen& c, int row, int col, T v) {
  typedef typename real_of<T>::type F;
  bool ok;
  const int gcol = tile_gcol<LT>(a, c, col, ok);
  if (!ok || row >= a.n_out) return;
  if constexpr (KIND == K_INV) {
    const F sc = F(a.scale);
    if (c.cmap) {   // crop + gather + diagonal + Jacobi: (diag S + y) jpre (bl_krylov.py:55)
      const int m = c.cmap[row];
      if (m >= 0) {
        const int comp = col / LT;
        const int64_t r3 = 3 * (int64_t)m + comp;
        const int64_t idx = (int64_t)m * a.C + gcol;
        const T d = static_cast<const T*>(a.diag)[r3];
        const T j = static_cast<const T*>(a.jpre)[r3];
        if constexpr (std::is_same<T, float2>::value) {
          if (a.wide) {
            widen_to(a.dst, idx, cmul(cadd(cmul(d, narrow_at(a.S, idx)), cscale(v, sc)), j));
            return;
          }
        }
        const T s = static_cast<const T*>(a.S)[idx];
        static_cast<T*>(a.dst)[idx] = cmul(cadd(cmul(d, s), cscale(v, sc)), j);
      }
      return;
    }
    v = cscale(v, sc);
  }
  static_cast<T*>(c.dstb)[(int64_t)row * a.dst_row + gcol] = v;
}

// ---- one radix-R butterfly of a stage; rows base + q*span of column col ----
// forward (DIF): DFT then twiddles w^(q*tws); inverse (DIT): conj twiddles then IDFT.
// SRC / DST: 1 = global (fused with the load or the store), 0 = shared;
// SRC 2 = shared, rows at or past n_in zero (not read).
template <int R, bool INV, int SRC, int DST, int KIND, typename T, int LT>
__device__ __forceinline__ void stage_job(const PassArgs& a, const Pen& c, T* sm, const T* tw, int col,
                                          int base, int span, int tws) {
  constexpr int W = 3 * LT;
  T v[R];
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const int row = base + q * span;
    if constexpr (SRC == 1) v[q] = gload<KIND, T, LT>(a, c, row, col);
    else if constexpr (SRC == 2) v[q] = row < a.n_in ? sm[row * W + col] : mkc<T>(0, 0);
    else v[q] = sm[row * W + col];
  }
  if constexpr (!INV) {
    dft<R, false>(v);
    if (tws) {
#pragma unroll
      for (int q = 1; q < R; ++q) v[q] = cmul(v[q], tw[q * tws]);
    }
  } else {
    if (tws) {
#pragma unroll
      for (int q = 1; q < R; ++q) v[q] = cmulc(v[q], tw[q * tws]);
    }
    dft<R, true>(v);
  }
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const int row = base + q * span;
    if constexpr (DST) gstore<KIND, T, LT>(a, c, row, col, v[q]);
    else sm[row * W + col] = v[q];
  }
}

// Largest radix compiled into the kernels of one element type (register
// budget: R complex values per job, 3 R in the X-pass middle).
template <typename T> struct RadixCap;
template <> struct RadixCap<double2> { static constexpr int stage = 10, mid = 4; };
template <> struct RadixCap<float2> { static constexpr int stage = 10, mid = 4; };

template <bool INV, int SRC, int DST, int KIND, typename T, int LT>
__device__ void run_stage(const PassArgs& a, const Pen& c, T* sm, const T* tw, int s) {
  constexpr int W = 3 * LT;
  const int M = a.ax.M, r = a.ax.rad[s], B = a.ax.blk[s];
  const int span = B / r, tstep = M / B;
  const int njobs = (M / r) * W;
  for (int job = threadIdx.x; job < njobs; job += blockDim.x) {
    const int col = job % W;
    const int t = job / W;
    const int b = t / span;
    const int j = t - b * span;
    const int base = b * B + j, tws = j * tstep;
    switch (r) {
#define BDDA_RADIX_CASE(RR)                                                          \
  case RR:                                                                           \
    if constexpr (RR <= RadixCap<T>::stage)                                          \
      stage_job<RR, INV, SRC, DST, KIND, T, LT>(a, c, sm, tw, col, base, span, tws); \
    break;
      BDDA_RADIX_CASE(2) BDDA_RADIX_CASE(3) BDDA_RADIX_CASE(4) BDDA_RADIX_CASE(5) BDDA_RADIX_CASE(6)
      BDDA_RADIX_CASE(7) BDDA_RADIX_CASE(8) BDDA_RADIX_CASE(9) BDDA_RADIX_CASE(10) BDDA_RADIX_CASE(12)
      BDDA_RADIX_CASE(14) BDDA_RADIX_CASE(16)
#undef BDDA_RADIX_CASE
      default: break;
    }
  }
}

// X pass middle: the last forward stage (span 1), the per-frequency 3x3
// complex-symmetric Green multiply and the first inverse stage (span 1) on
// registers; one job = R consecutive frequencies x all 3 components of one
// right-hand side, so the 6 unique entries are read once per frequency and
// right-hand side from the pencil staged in shared memory.
template <int R, int SRC, int DST, typename T, int LT>
__device__ __forceinline__ void conv_mid_job(const PassArgs& a, const Pen& c, T* sm, const T* gs, int b,
                                             int li) {
  constexpr int W = 3 * LT;
  T y[3][R];
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int row = b * R + q, col = comp * LT + li;
      if constexpr (SRC == 1) y[comp][q] = gload<K_CONV, T, LT>(a, c, row, col);
      else if constexpr (SRC == 2) y[comp][q] = row < a.n_in ? sm[row * W + col] : mkc<T>(0, 0);
      else y[comp][q] = sm[row * W + col];
    }
    dft<R, false>(y[comp]);
  }
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const T* g = gs + (b * R + q) * 6;
    const T gxx = g[0], gxy = g[1], gxz = g[2], gyy = g[3], gyz = g[4], gzz = g[5];
    const T v0 = y[0][q], v1 = y[1][q], v2 = y[2][q];
    y[0][q] = cadd(cadd(cmul(gxx, v0), cmul(gxy, v1)), cmul(gxz, v2));
    y[1][q] = cadd(cadd(cmul(gxy, v0), cmul(gyy, v1)), cmul(gyz, v2));
    y[2][q] = cadd(cadd(cmul(gxz, v0), cmul(gyz, v1)), cmul(gzz, v2));
  }
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
    dft<R, true>(y[comp]);
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int row = b * R + q, col = comp * LT + li;
      if constexpr (DST) gstore<K_CONV, T, LT>(a, c, row, col, y[comp][q]);
      else sm[row * W + col] = y[comp][q];
    }
  }
}

template <int SRC, int DST, typename T, int LT>
__device__ void run_conv_mid(const PassArgs& a, const Pen& c, T* sm, const T* gs) {
  const int r = a.ax.rad[a.ax.nst - 1];
  const int njobs = (a.ax.M / r) * LT;
  for (int job = threadIdx.x; job < njobs; job += blockDim.x) {
    const int li = job % LT, b = job / LT;
    switch (r) {
#define BDDA_MID_CASE(RR)                                        \
  case RR:                                                         \
    if constexpr (RR <= RadixCap<T>::mid)                          \
      conv_mid_job<RR, SRC, DST, T, LT>(a, c, sm, gs, b, li);      \
    break;
      BDDA_MID_CASE(2) BDDA_MID_CASE(3) BDDA_MID_CASE(4) BDDA_MID_CASE(5) BDDA_MID_CASE(6)
      BDDA_MID_CASE(7) BDDA_MID_CASE(8) BDDA_MID_CASE(9) BDDA_MID_CASE(10) BDDA_MID_CASE(12)
      BDDA_MID_CASE(14) BDDA_MID_CASE(16)
#undef BDDA_MID_CASE
      default: break;
    }
  }
}

// Generic pencil pass of CTA-sized item bid: runtime radix sequence (any
// length factored into radices <= RadixCap).  The specialised kernels
// (bdda_fixed_*.cu) replace it for the radix sequences the workloads use; the
// batched solver runs it from persistent CTAs.
// FIRST: where the first stage reads; 1 = global memory, 2 = the tile, filled
// by a bulk tensor copy the caller issued (rows [0, n_in)).
template <typename T, int KIND, int LT, int FIRST = 1>
__device__ __forceinline__ void generic_pencil(const PassArgs& a, int64_t bid, unsigned char* smraw) {
  const int M = a.ax.M, nst = a.ax.nst;
  T *tw, *sm, *gs;
  int32_t* cm;
  stage_constants<T, KIND, LT>(a, smraw, M, &tw, &sm, &gs, &cm, bid);
  const Pen c = pen_of_block<T>(a, cm, bid);
  if constexpr (FIRST == 2) {
    if (!tile_landed<T, KIND, LT>(a, smraw, M)) return;
  }
  if constexpr (KIND == K_FWD) {
    bool staged = false;
    if constexpr (std::is_same<T, double2>::value) {
      if (a.green) {   // real-space tensor rows evaluated into the tile (3 LT == 6)
        for (int i = threadIdx.x; i < M; i += blockDim.x)
          green_row(a, (int)c.p0, (int)c.p1, i, reinterpret_cast<double2*>(sm) + i * 3 * LT);
        __syncthreads();
        staged = true;
      }
    }
    if (nst == 1) {
      if (staged) run_stage<false, 0, 1, KIND, T, LT>(a, c, sm, tw, 0);
      else run_stage<false, FIRST, 1, KIND, T, LT>(a, c, sm, tw, 0);
      return;
    }
    if (staged) run_stage<false, 0, 0, KIND, T, LT>(a, c, sm, tw, 0);
    else run_stage<false, FIRST, 0, KIND, T, LT>(a, c, sm, tw, 0);
    __syncthreads();
    for (int s = 1; s < nst - 1; ++s) {
      run_stage<false, 0, 0, KIND, T, LT>(a, c, sm, tw, s);
      __syncthreads();
    }
    run_stage<false, 0, 1, KIND, T, LT>(a, c, sm, tw, nst - 1);
  } else if constexpr (KIND == K_INV) {
    if (nst == 1) {
      run_stage<true, FIRST, 1, KIND, T, LT>(a, c, sm, tw, 0);
      return;
    }
    run_stage<true, FIRST, 0, KIND, T, LT>(a, c, sm, tw, nst - 1);
    __syncthreads();
    for (int s = nst - 2; s >= 1; --s) {
      run_stage<true, 0, 0, KIND, T, LT>(a, c, sm, tw, s);
      __syncthreads();
    }
    run_stage<true, 0, 1, KIND, T, LT>(a, c, sm, tw, 0);
  } else {   // K_CONV
    cp_async_wait<0>();
    __syncthreads();
    if (nst == 1) {
      run_conv_mid<FIRST, 1, T, LT>(a, c, sm, gs);
      return;
    }
    run_stage<false, FIRST, 0, KIND, T, LT>(a, c, sm, tw, 0);
    __syncthreads();
    for (int s = 1; s < nst - 1; ++s) {
      run_stage<false, 0, 0, KIND, T, LT>(a, c, sm, tw, s);
      __syncthreads();
    }
    run_conv_mid<0, 0, T, LT>(a, c, sm, gs);
    __syncthreads();
    for (int s = nst - 2; s >= 1; --s) {
      run_stage<true, 0, 0, KIND, T, LT>(a, c, sm, tw, s);
      __syncthreads();
    }
    run_stage<true, 0, 1, KIND, T, LT>(a, c, sm, tw, 0);
  }
}

// Pass kind of the five passes of a product: Z, Y, X, Y^-1, Z^-1.
constexpr int kPassKind[5] = {K_FWD, K_FWD, K_CONV, K_INV, K_INV};

// Arguments of the five passes of one block product (bdda_mvp.cu).
template <typename T>
void mvp_pass_args(const bdda_plan* plan, int L, const T* ghat, const int32_t* cell_map, const T* src,
                   const T* diag, const T* jpre, T* out, T* F, PassArgs a[5], int64_t P0[5]);

// Launch hook of a compile-time-specialised pencil kernel.
typedef int (*FixedLaunchFn)(const PassArgs& a, int64_t P0, cudaStream_t st);
struct FixedKernel {
  int prec, kind, lt;
  int minb;            // register bound: resident CTAs per SM (1 = none)
  int variant;         // id for the autotuner: minb (256 threads) or minb + 16 * threads / 32
  int r[4];            // radix sequence, padded with 1
  FixedLaunchFn fn;
  int pair;            // 1: column-pair jobs (needs even L and 16-byte aligned fields)
};
const FixedKernel* fixed_table_a(int* n);
const FixedKernel* fixed_table_b(int* n);
const FixedKernel* fixed_table_c(int* n);
const FixedKernel* fixed_table_d(int* n);
const FixedKernel* fixed_table_e(int* n);
const FixedKernel* fixed_table_f(int* n);
const FixedKernel* fixed_table_g(int* n);
const FixedKernel* fixed_table_h(int* n);
const FixedKernel* fixed_table_i(int* n);
const FixedKernel* fixed_table_j(int* n);


}  // namespace bdda
