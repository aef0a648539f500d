// Pencil kernels specialised at compile time for one radix sequence.
//
// The generic kernel (bdda_mvp.cu) reads the radix sequence at run time, so
// every butterfly job pays integer divisions and strides it cannot fold.
// Here the sequence (up to four radices, padded with 1), the tile width and
// the CTA size are template parameters: stage spans, twiddle strides, job
// counts and all index divisions are constants; for complex64 a job can take
// two adjacent columns (16-byte accesses).  Each butterfly unrolls; the
// loop over a stage's rounds of jobs does not (unrolling it made the kernels
// large enough to stall on instruction fetch: the complex64 product ran 3 %
// slower).  bdda_fixed_*.cu instantiate the sequences the planner produces
// for the workloads; fixed_find() in bdda_mvp.cu dispatches to them.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "bdda_pencil.cuh"

namespace bdda {

template <int R0, int R1, int R2, int R3>
struct RadixSeq {
  static constexpr int M = R0 * R1 * R2 * R3;
  static constexpr int n = (R1 == 1) ? 1 : (R2 == 1) ? 2 : (R3 == 1) ? 3 : 4;
  static constexpr int r(int s) { return s == 0 ? R0 : s == 1 ? R1 : s == 2 ? R2 : R3; }
  static constexpr int blk(int s) {
    return s == 0 ? M : s == 1 ? M / R0 : s == 2 ? M / (R0 * R1) : M / (R0 * R1 * R2);
  }
};

// ---- column pairs (complex64): one job = two adjacent columns of the tile ----
// Column col (even) and col + 1 are right-hand sides l, l + 1 of the same
// component, contiguous in HBM and in shared memory, so each row is one
// 16-byte access and each twiddle / Green entry serves both columns; the
// arithmetic per column is that of stage_job / conv_mid_job, so results are
// bitwise the same.  Valid when L is even (l < L implies l + 1 < L) and the
// field pointers are 16-byte aligned (pair_ok in bdda_mvp.cu).
__device__ __forceinline__ float4 pack2(float2 p, float2 q) { return make_float4(p.x, p.y, q.x, q.y); }
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

template <int KIND, int LT>
__device__ __forceinline__ float4 gload2(const PassArgs& a, const Pen& c, int row, int col) {
  bool ok;
  const int gcol = tile_gcol<LT>(a, c, col, ok);
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
  if (!ok || row >= a.n_in) return z;
  if constexpr (KIND == K_FWD) {
    if (c.cmap) {
      const int m = c.cmap[row];
      if (m < 0) return z;
      const int64_t i = (int64_t)m * a.C + gcol;
      if (a.wide) return pack2(narrow_at(a.S, i), narrow_at(a.S, i + 1));
      return *reinterpret_cast<const float4*>(static_cast<const float2*>(a.S) + i);
    }
  }
  return *reinterpret_cast<const float4*>(static_cast<const float2*>(c.srcb) + (int64_t)row * a.src_row + gcol);
}

template <int KIND, int LT>
__device__ __forceinline__ void gstore2(const PassArgs& a, const Pen& c, int row, int col, float2 v0, float2 v1) {
  bool ok;
  const int gcol = tile_gcol<LT>(a, c, col, ok);
  if (!ok || row >= a.n_out) return;
  if constexpr (KIND == K_INV) {
    const float sc = float(a.scale);
    if (c.cmap) {   // crop + gather + diagonal + Jacobi, as gstore
      const int m = c.cmap[row];
      if (m >= 0) {
        const int comp = col / LT;
        const int64_t r3 = 3 * (int64_t)m + comp;
        const int64_t idx = (int64_t)m * a.C + gcol;
        const float2 d = static_cast<const float2*>(a.diag)[r3];
        const float2 j = static_cast<const float2*>(a.jpre)[r3];
        if (a.wide) {
          widen_to(a.dst, idx, cmul(cadd(cmul(d, narrow_at(a.S, idx)), cscale(v0, sc)), j));
          widen_to(a.dst, idx + 1, cmul(cadd(cmul(d, narrow_at(a.S, idx + 1)), cscale(v1, sc)), j));
          return;
        }
        const float4 s = *reinterpret_cast<const float4*>(static_cast<const float2*>(a.S) + idx);
        const float2 o0 = cmul(cadd(cmul(d, lo2(s)), cscale(v0, sc)), j);
        const float2 o1 = cmul(cadd(cmul(d, hi2(s)), cscale(v1, sc)), j);
        *reinterpret_cast<float4*>(static_cast<float2*>(a.dst) + idx) = pack2(o0, o1);
      }
      return;
    }
    v0 = cscale(v0, sc);
    v1 = cscale(v1, sc);
  }
  *reinterpret_cast<float4*>(static_cast<float2*>(c.dstb) + (int64_t)row * a.dst_row + gcol) = pack2(v0, v1);
}

template <int R, bool INV, int SRC, int DST, int KIND, int LT>
__device__ __forceinline__ void stage_job2(const PassArgs& a, const Pen& c, float2* sm, const float2* tw, int col,
                                           int base, int span, int tws) {
  constexpr int W = 3 * LT;
  float2 v[R], u[R];
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const int row = base + q * span;
    float4 x;
    if constexpr (SRC == 1) x = gload2<KIND, LT>(a, c, row, col);
    else if constexpr (SRC == 2) x = row < a.n_in ? *reinterpret_cast<const float4*>(sm + row * W + col)
                                                  : make_float4(0.f, 0.f, 0.f, 0.f);
    else x = *reinterpret_cast<const float4*>(sm + row * W + col);
    v[q] = lo2(x);
    u[q] = hi2(x);
  }
  if constexpr (!INV) {
    dft<R, false>(v);
    dft<R, false>(u);
    if (tws) {
#pragma unroll
      for (int q = 1; q < R; ++q) {
        const float2 w = tw[q * tws];
        v[q] = cmul(v[q], w);
        u[q] = cmul(u[q], w);
      }
    }
  } else {
    if (tws) {
#pragma unroll
      for (int q = 1; q < R; ++q) {
        const float2 w = tw[q * tws];
        v[q] = cmulc(v[q], w);
        u[q] = cmulc(u[q], w);
      }
    }
    dft<R, true>(v);
    dft<R, true>(u);
  }
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const int row = base + q * span;
    if constexpr (DST) gstore2<KIND, LT>(a, c, row, col, v[q], u[q]);
    else *reinterpret_cast<float4*>(sm + row * W + col) = pack2(v[q], u[q]);
  }
}

template <int R, int SRC, int DST, int LT>
__device__ __forceinline__ void conv_mid_job2(const PassArgs& a, const Pen& c, float2* sm, const float2* gs, int b,
                                              int li) {
  constexpr int W = 3 * LT;
  float2 y[3][R], z[3][R];
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int row = b * R + q, col = comp * LT + li;
      float4 x;
      if constexpr (SRC == 1) x = gload2<K_CONV, LT>(a, c, row, col);
      else if constexpr (SRC == 2) x = row < a.n_in ? *reinterpret_cast<const float4*>(sm + row * W + col)
                                                    : make_float4(0.f, 0.f, 0.f, 0.f);
      else x = *reinterpret_cast<const float4*>(sm + row * W + col);
      y[comp][q] = lo2(x);
      z[comp][q] = hi2(x);
    }
    dft<R, false>(y[comp]);
    dft<R, false>(z[comp]);
  }
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const float4* g4 = reinterpret_cast<const float4*>(gs + (b * R + q) * 6);
    const float4 g01 = g4[0], g23 = g4[1], g45 = g4[2];
    const float2 gxx = lo2(g01), gxy = hi2(g01), gxz = lo2(g23), gyy = hi2(g23), gyz = lo2(g45), gzz = hi2(g45);
    {
      const float2 v0 = y[0][q], v1 = y[1][q], v2 = y[2][q];
      y[0][q] = cadd(cadd(cmul(gxx, v0), cmul(gxy, v1)), cmul(gxz, v2));
      y[1][q] = cadd(cadd(cmul(gxy, v0), cmul(gyy, v1)), cmul(gyz, v2));
      y[2][q] = cadd(cadd(cmul(gxz, v0), cmul(gyz, v1)), cmul(gzz, v2));
    }
    {
      const float2 v0 = z[0][q], v1 = z[1][q], v2 = z[2][q];
      z[0][q] = cadd(cadd(cmul(gxx, v0), cmul(gxy, v1)), cmul(gxz, v2));
      z[1][q] = cadd(cadd(cmul(gxy, v0), cmul(gyy, v1)), cmul(gyz, v2));
      z[2][q] = cadd(cadd(cmul(gxz, v0), cmul(gyz, v1)), cmul(gzz, v2));
    }
  }
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
    dft<R, true>(y[comp]);
    dft<R, true>(z[comp]);
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int row = b * R + q, col = comp * LT + li;
      if constexpr (DST) gstore2<K_CONV, LT>(a, c, row, col, y[comp][q], z[comp][q]);
      else *reinterpret_cast<float4*>(sm + row * W + col) = pack2(y[comp][q], z[comp][q]);
    }
  }
}

// PAIR: jobs over column pairs (complex64 only); otherwise one column per job.
template <class RS, int S, bool INV, int SRC, int DST, int KIND, typename T, int LT, int NT, int PAIR>
__device__ __forceinline__ void fixed_stage(const PassArgs& a, const Pen& c, T* sm, const T* tw) {
  constexpr int W = 3 * LT;
  constexpr int WJ = PAIR ? W / 2 : W;   // jobs per row
  constexpr int R = RS::r(S), B = RS::blk(S), SPAN = B / R, TSTEP = RS::M / B;
  constexpr int NJOBS = (RS::M / R) * WJ;
  constexpr int ITERS = (NJOBS + NT - 1) / NT;
#pragma unroll 1
  for (int it = 0; it < ITERS; ++it) {
    const int job = threadIdx.x + it * NT;
    if ((NJOBS % NT) == 0 || job < NJOBS) {
      const int cj = job % WJ;
      const int t = job / WJ;
      const int b = t / SPAN;
      const int j = t - b * SPAN;
      if constexpr (PAIR) stage_job2<R, INV, SRC, DST, KIND, LT>(a, c, sm, tw, 2 * cj, b * B + j, SPAN, j * TSTEP);
      else stage_job<R, INV, SRC, DST, KIND, T, LT>(a, c, sm, tw, cj, b * B + j, SPAN, j * TSTEP);
    }
  }
}

template <class RS, int SRC, int DST, typename T, int LT, int NT, int PAIR>
__device__ __forceinline__ void fixed_mid(const PassArgs& a, const Pen& c, T* sm, const T* gs) {
  constexpr int R = RS::r(RS::n - 1);
  constexpr int LJ = PAIR ? LT / 2 : LT;   // jobs per frequency group
  constexpr int NJOBS = (RS::M / R) * LJ;
  constexpr int ITERS = (NJOBS + NT - 1) / NT;
#pragma unroll 1
  for (int it = 0; it < ITERS; ++it) {
    const int job = threadIdx.x + it * NT;
    if ((NJOBS % NT) == 0 || job < NJOBS) {
      if constexpr (PAIR) conv_mid_job2<R, SRC, DST, LT>(a, c, sm, gs, job / LJ, 2 * (job % LJ));
      else conv_mid_job<R, SRC, DST, T, LT>(a, c, sm, gs, job / LJ, job % LJ);
    }
  }
}

// First stage of a pass: reads the TMA-filled tile (from_tile; the copy
// brought rows [0, n_in), the rows past them are zero and not read) or
// global memory.
template <class RS, int S, bool INV, int DST, int KIND, typename T, int LT, int NT, int PAIR, int TMA>
__device__ __forceinline__ void first_stage(const PassArgs& a, const Pen& c, T* sm, const T* tw, bool from_tile) {
  if constexpr (TMA) {
    if (from_tile) {
      fixed_stage<RS, S, INV, 2, DST, KIND, T, LT, NT, PAIR>(a, c, sm, tw);
      return;
    }
  }
  fixed_stage<RS, S, INV, 1, DST, KIND, T, LT, NT, PAIR>(a, c, sm, tw);
}
template <class RS, typename T, int LT, int NT, int PAIR, int TMA>
__device__ __forceinline__ void first_mid(const PassArgs& a, const Pen& c, T* sm, const T* gs, bool from_tile) {
  if constexpr (TMA) {
    if (from_tile) {
      fixed_mid<RS, 2, 1, T, LT, NT, PAIR>(a, c, sm, gs);
      return;
    }
  }
  fixed_mid<RS, 1, 1, T, LT, NT, PAIR>(a, c, sm, gs);
}

// NT: threads per CTA.  MINB: resident CTAs per SM the register allocation
// must allow (the __launch_bounds__ minimum); 1 = no bound.  PAIR: column
// pairs per job (complex64).  TMA: the first read of the tile is a bulk tensor
// copy (dense sources only; make_tile_map).  Kernels are compiled with several
// (NT, MINB, PAIR, TMA) and the autotuner picks per pass.
template <typename T, int KIND, int LT, int NT, int MINB, int R0, int R1, int R2, int R3, int PAIR, int TMA>
__global__ void __launch_bounds__(NT, MINB) fixed_pencil_kernel(const PassArgs a, const __grid_constant__ CUtensorMap tm,
                                                                const TmaTile tt) {
  static_assert(!PAIR || (std::is_same<T, float2>::value && LT % 2 == 0), "column pairs are complex64, even LT");
  using RS = RadixSeq<R0, R1, R2, R3>;
  constexpr int N = RS::n;
  extern __shared__ __align__(128) unsigned char smraw[];
  // the bulk copy needs a 128-byte aligned destination; otherwise (not seen:
  // dynamic shared memory starts on a wide boundary) the plain global reads
  const bool from_tile = TMA && (smem_u32(pencil_tile<T, LT>(smraw, RS::M)) & 127) == 0;
  if constexpr (TMA) {
    if (from_tile && threadIdx.x == 0) tma_issue<T, KIND, LT>(a, &tm, tt, smraw, RS::M, blockIdx.x);
  }
  T *tw, *sm, *gs;
  int32_t* cm;
  stage_constants<T, KIND, LT>(a, smraw, RS::M, &tw, &sm, &gs, &cm, blockIdx.x);
  const Pen c = pen_of_block<T>(a, cm, blockIdx.x);
  if constexpr (TMA) {
    if (from_tile && !tile_landed<T, KIND, LT>(a, smraw, RS::M)) return;
  }
  if constexpr (KIND == K_FWD) {
    if constexpr (N == 1) {
      first_stage<RS, 0, false, 1, KIND, T, LT, NT, PAIR, TMA>(a, c, sm, tw, from_tile);
    } else {
      first_stage<RS, 0, false, 0, KIND, T, LT, NT, PAIR, TMA>(a, c, sm, tw, from_tile);
      __syncthreads();
      if constexpr (N >= 3) { fixed_stage<RS, 1, false, 0, 0, KIND, T, LT, NT, PAIR>(a, c, sm, tw); __syncthreads(); }
      if constexpr (N >= 4) { fixed_stage<RS, 2, false, 0, 0, KIND, T, LT, NT, PAIR>(a, c, sm, tw); __syncthreads(); }
      fixed_stage<RS, N - 1, false, 0, 1, KIND, T, LT, NT, PAIR>(a, c, sm, tw);
    }
  } else if constexpr (KIND == K_INV) {
    if constexpr (N == 1) {
      first_stage<RS, 0, true, 1, KIND, T, LT, NT, PAIR, TMA>(a, c, sm, tw, from_tile);
    } else {
      first_stage<RS, N - 1, true, 0, KIND, T, LT, NT, PAIR, TMA>(a, c, sm, tw, from_tile);
      __syncthreads();
      if constexpr (N >= 4) { fixed_stage<RS, 2, true, 0, 0, KIND, T, LT, NT, PAIR>(a, c, sm, tw); __syncthreads(); }
      if constexpr (N >= 3) { fixed_stage<RS, 1, true, 0, 0, KIND, T, LT, NT, PAIR>(a, c, sm, tw); __syncthreads(); }
      fixed_stage<RS, 0, true, 0, 1, KIND, T, LT, NT, PAIR>(a, c, sm, tw);
    }
  } else {   // K_CONV
    cp_async_wait<0>();
    __syncthreads();
    if constexpr (N == 1) {
      first_mid<RS, T, LT, NT, PAIR, TMA>(a, c, sm, gs, from_tile);
    } else {
      first_stage<RS, 0, false, 0, KIND, T, LT, NT, PAIR, TMA>(a, c, sm, tw, from_tile);
      __syncthreads();
      if constexpr (N >= 3) { fixed_stage<RS, 1, false, 0, 0, KIND, T, LT, NT, PAIR>(a, c, sm, tw); __syncthreads(); }
      if constexpr (N >= 4) { fixed_stage<RS, 2, false, 0, 0, KIND, T, LT, NT, PAIR>(a, c, sm, tw); __syncthreads(); }
      fixed_mid<RS, 0, 0, T, LT, NT, PAIR>(a, c, sm, gs);
      __syncthreads();
      if constexpr (N >= 4) { fixed_stage<RS, 2, true, 0, 0, KIND, T, LT, NT, PAIR>(a, c, sm, tw); __syncthreads(); }
      if constexpr (N >= 3) { fixed_stage<RS, 1, true, 0, 0, KIND, T, LT, NT, PAIR>(a, c, sm, tw); __syncthreads(); }
      fixed_stage<RS, 0, true, 0, 1, KIND, T, LT, NT, PAIR>(a, c, sm, tw);
    }
  }
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (no link against the driver library).
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Rows of the one or two boxes that fill M rows of a tile (box 1 starts at
// M - box_rows, 128-byte aligned in the tile); false if M needs more.
inline bool tile_boxes(int M, int row_bytes, int* nbox, int* box_rows) {
  if (M < 1) return false;
  if (M <= 256) {
    *nbox = 1;
    *box_rows = M;
    return true;
  }
  int g = 1;   // rows per 128-byte granule of the tile
  while ((g * row_bytes) % 128) ++g;
  int br = (M + 1) / 2;
  while ((M - br) % g) ++br;
  if (br > 256 || M > 512) return false;
  *nbox = 2;
  *box_rows = br;
  return true;
}

// Tensor map of the tile copies of a pass, covering tile rows [0, rows)
// (rows = M: the source rows and the zero rows after them; rows = n_in: the
// source rows only, for kernels that never read the others).  False when the
// pass cannot use them: a gathered or evaluated source, a source pointer,
// column offset or stride that is not a 16-byte multiple, or more than two
// boxes.
template <typename T, int KIND, int LT>
bool make_tile_map(const PassArgs& a, int64_t P0, int rows, CUtensorMap* tm, TmaTile* tt) {
  constexpr int E = sizeof(T) / 8;
  const int64_t s = sizeof(T);
  if ((KIND == K_FWD && a.cell_map) || a.green || !a.src) return false;
  // x coordinates are multiples of LT * s bytes: they must be 16-byte multiples
  if ((reinterpret_cast<uintptr_t>(a.src) & 15) || (LT * s) % 16 || (a.L * s) % 16) return false;
  if (a.n_in < 1 || a.P1 < 1 || P0 < 1 || a.L < 1) return false;
  const int64_t strides[3] = {a.src_row * s, a.src_p1 * s, a.src_p0 * s};
  for (int64_t st : strides)
    if (st <= 0 || st % 16 || st >= ((int64_t)1 << 40)) return false;
  int nbox, box_rows;
  if (rows < 1 || !tile_boxes(rows, 3 * LT * (int)s, &nbox, &box_rows)) return false;
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  // dimensions 2..4: (row, p1, p0) ordered by stride
  int order[3] = {0, 1, 2};
  for (int i = 0; i < 3; ++i)
    for (int j = i + 1; j < 3; ++j)
      if (strides[order[j]] < strides[order[i]]) std::swap(order[i], order[j]);
  const int64_t ext[3] = {a.n_in, a.P1, P0};
  const int box3[3] = {box_rows, 1, 1};
  cuuint64_t gdim[5] = {(cuuint64_t)a.L * E, 3, 0, 0, 0};
  cuuint64_t gstride[4] = {(cuuint64_t)(a.L * s), 0, 0, 0};
  cuuint32_t box[5] = {(cuuint32_t)(LT * E), 3, 0, 0, 0};
  cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  for (int d = 0; d < 3; ++d) {
    gdim[2 + d] = (cuuint64_t)ext[order[d]];
    gstride[1 + d] = (cuuint64_t)strides[order[d]];
    box[2 + d] = (cuuint32_t)box3[order[d]];
    tt->dim_of[d] = order[d];
  }
  tt->nbox = nbox;
  tt->box_rows = box_rows;
  tt->rows = rows;
  const CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_UINT64, 5, const_cast<void*>(a.src), gdim, gstride, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <typename T, int KIND, int LT, int MINB, int NT, int PAIR, int R0, int R1, int R2, int R3, int TMA = 0>
int fixed_launch(const PassArgs& a0, int64_t P0, cudaStream_t st) {
  static_assert(NT % 32 == 0 && NT <= 512 && MINB >= 1 && MINB < 16, "variant id encodes whole warps and MINB < 16");
  using RS = RadixSeq<R0, R1, R2, R3>;
  PassArgs a = a0;
  if (a.ax.M != RS::M) return BDDA_BAD_ARG;
  if (PAIR && (a.L % 2) != 0) return BDDA_BAD_ARG;
  a.ntile = (a.L + LT - 1) / LT;
  CUtensorMap tm;
  memset(&tm, 0, sizeof(tm));
  TmaTile tt;
  memset(&tt, 0, sizeof(tt));
  if (TMA && !make_tile_map<T, KIND, LT>(a, P0, a.n_in, &tm, &tt))   // not possible for this pass: the plain kernel
    return fixed_launch<T, KIND, LT, MINB, NT, PAIR, R0, R1, R2, R3, 0>(a0, P0, st);
  auto kern = fixed_pencil_kernel<T, KIND, LT, NT, MINB, R0, R1, R2, R3, PAIR, TMA>;
  const size_t smem = (size_t)pencil_smem_bytes<T>(RS::M, LT, KIND);
  if (smem > 227 * 1024) return BDDA_BAD_ARG;
  const int64_t nblk = P0 * a.P1 * a.ntile;
  if (nblk <= 0) return BDDA_OK;
  if (nblk > 0x7fffffff) return BDDA_BAD_ARG;
  BDDA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)nblk, NT, smem, st>>>(a, tm, tt);
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BDDA_OK;
}

// Table entry of a specialised kernel with 256 threads per CTA (variant id =
// MINB) or NT threads (variant id = MINB + 16 NT/32: the CTA size that makes
// the stages' butterfly jobs fill whole rounds of threads; NT a multiple of
// 32, so that ids stay distinct); column-pair kernels add 512 to the id.
#define BDDA_FIXED(T, PREC, KIND, LT, MINB, R0, R1, R2, R3) \
  { PREC, KIND, LT, MINB, MINB, {R0, R1, R2, R3}, &fixed_launch<T, KIND, LT, MINB, 256, 0, R0, R1, R2, R3>, 0 }
#define BDDA_FIXED_NT(T, PREC, KIND, LT, MINB, NT, R0, R1, R2, R3)                              \
  { PREC, KIND, LT, MINB, MINB + 16 * ((NT) / 32), {R0, R1, R2, R3},                              \
    &fixed_launch<T, KIND, LT, MINB, NT, 0, R0, R1, R2, R3>, 0 }
#define BDDA_FIXED_PAIR(PREC, KIND, LT, MINB, NT, R0, R1, R2, R3)                                 \
  { PREC, KIND, LT, MINB, 512 + MINB + 16 * ((NT) / 32), {R0, R1, R2, R3},                        \
    &fixed_launch<float2, KIND, LT, MINB, NT, 1, R0, R1, R2, R3>, 1 }
// The same with the tile's first read by a bulk tensor copy: ids + 1024.
#define BDDA_FIXED_TMA(T, PREC, KIND, LT, MINB, R0, R1, R2, R3) \
  { PREC, KIND, LT, MINB, 1024 + MINB, {R0, R1, R2, R3}, &fixed_launch<T, KIND, LT, MINB, 256, 0, R0, R1, R2, R3, 1>, 0 }
#define BDDA_FIXED_TMA_NT(T, PREC, KIND, LT, MINB, NT, R0, R1, R2, R3)                          \
  { PREC, KIND, LT, MINB, 1024 + MINB + 16 * ((NT) / 32), {R0, R1, R2, R3},                       \
    &fixed_launch<T, KIND, LT, MINB, NT, 0, R0, R1, R2, R3, 1>, 0 }
#define BDDA_FIXED_TMA_PAIR(PREC, KIND, LT, MINB, NT, R0, R1, R2, R3)                             \
  { PREC, KIND, LT, MINB, 1024 + 512 + MINB + 16 * ((NT) / 32), {R0, R1, R2, R3},                 \
    &fixed_launch<float2, KIND, LT, MINB, NT, 1, R0, R1, R2, R3, 1>, 1 }

}  // namespace bdda
