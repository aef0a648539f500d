// X pass (forward x transform, 3x3 Green multiply, inverse x transform) of an
// axis of length M = A * B in two register stages instead of the plan's
// radix sequence.
//
// The plan-stage X-pass kernels run the plan's stages ([8,8,3] for the x=20
// particle's 192-point axis): four shared-memory round trips of the tile.
// Here the transform of a column is
//   X[k + A k2] = sum_j W_B^(j k2) w^(j k) sum_q x[j + B q] W_A^(q k)
// (j < B, q, k < A, k2 < B, w = exp(-2 pi i / M)):
//   stage 1: per (j, column) a register DFT_A over rows j + B q, the twiddles
//            w^(j k), written to the rows of (j, k) (xrow);
//   middle:  per (k, column) a register DFT_B over the rows of (j, k) of the three
//            components, the Green multiply at frequency k + A k2, the
//            inverse DFT_B, written back;
//   stage 1 inverse: per (j, column) the conjugate twiddles and the inverse
//            DFT_A, stored to the rows below n_out.
// That is two round trips instead of four.  The Green's spectrum stays in
// the plan's storage order in HBM (the position of frequency f under the
// plan's digit reversal, radices P0 P1 P2) and is gathered into natural order
// while it is staged, so the kernel drops into a plan whose x axis is
// factored [P0, P1, P2] and gives the same product to rounding.  Stage 1
// skips the source rows at or past n_in (zero), so a TMA copy needs only
// those rows.
#pragma once
#include "bdda_fixed.cuh"

namespace bdda {

// Position in the plan's digit-reversed storage of frequency f (three DIF
// stages of radices P0, P1, P2).
template <int P0, int P1, int P2>
__device__ __forceinline__ int plan_position(int f) {
  constexpr int M = P0 * P1 * P2;
  const int d0 = f % P0, d1 = (f / P0) % P1, d2 = f / (P0 * P1);
  return d0 * (M / P0) + d1 * (M / (P0 * P1)) + d2;
}

// Twiddles and this pencil's Green's spectrum in natural frequency order
// (gathered from the plan's storage order), both by cp.async; returns after
// they landed.  A middle job reads the entries of frequencies k + A k2 for
// consecutive k across a warp: consecutive 6-entry records, no bank conflict.
template <typename T, int LT, int A, int B, int P0, int P1, int P2>
__device__ __forceinline__ void xconv_stage(const PassArgs& a, unsigned char* smraw, T** tw, T** sm, T** gs,
                                            int64_t bid) {
  constexpr int M = A * B;
  const int o_sm = align128(M * (int)sizeof(T));
  const int o_gs = o_sm + align16(M * 3 * LT * (int)sizeof(T));
  *tw = reinterpret_cast<T*>(smraw);
  *sm = reinterpret_cast<T*>(smraw + o_sm);
  *gs = reinterpret_cast<T*>(smraw + o_gs);
  async_copy(*tw, a.tw, M * (int)sizeof(T));
  const T* g = static_cast<const T*>(a.ghat) + (bid / a.ntile) * (int64_t)M * 6;
  constexpr int CH = 6 * (int)sizeof(T) / 16;   // 16-byte chunks per frequency
  for (int i = threadIdx.x; i < M * CH; i += blockDim.x) {
    const int f = i / CH, part = i - f * CH;
    cp_async16(reinterpret_cast<char*>(*gs + f * 6) + 16 * part,
               reinterpret_cast<const char*>(g + plan_position<P0, P1, P2>(f) * 6) + 16 * part);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
}

// Intermediate layout in the tile (XL): 0 = the value of (j, k) at row
// j + B k, where stage 1 writes the rows it read (in place, any number of jobs
// per thread); 1 = at row j A + k, where a warp's middle jobs (consecutive k)
// read rows one apart instead of B apart, free of bank conflicts for 8-byte
// values, but stage 1 writes rows other jobs read, so each thread holds one
// job (NT = B W) and the writes wait for all reads.
template <int A, int B, int XL>
__device__ __forceinline__ int xrow(int j, int k) {
  return XL ? j * A + k : j + B * k;
}

template <typename T, int LT, int NT, int MINB, int A, int B, int P0, int P1, int P2, int TMA, int XL>
__global__ void __launch_bounds__(NT, MINB) xconv2_kernel(const PassArgs a, const __grid_constant__ CUtensorMap tm,
                                                          const TmaTile tt) {
  constexpr int M = A * B, W = 3 * LT;
  static_assert(M == P0 * P1 * P2, "two-stage split and plan radices describe one axis");
  static_assert(!XL || (NT == B * W), "layout 1 runs one stage-1 job per thread");
  extern __shared__ __align__(128) unsigned char smraw[];
  const bool from_tile = TMA && (smem_u32(pencil_tile<T, LT>(smraw, M)) & 127) == 0;
  if constexpr (TMA) {
    if (from_tile && threadIdx.x == 0) tma_issue<T, K_CONV, LT>(a, &tm, tt, smraw, M, blockIdx.x);
  }
  T *tw, *sm, *gs;
  xconv_stage<T, LT, A, B, P0, P1, P2>(a, smraw, &tw, &sm, &gs, blockIdx.x);
  const Pen c = pen_of_block<T>(a, nullptr, blockIdx.x);
  if constexpr (TMA) {
    if (from_tile && !tile_landed<T, K_CONV, LT>(a, smraw, M)) return;
  }
  const int n_in = a.n_in;
  // stage 1, forward
#pragma unroll 1
  for (int job = threadIdx.x; job < B * W; job += NT) {
    const int col = job % W, j = job / W;
    T v[A];
    if (from_tile) {
#pragma unroll
      for (int q = 0; q < A; ++q) {
        const int row = j + B * q;
        v[q] = row < n_in ? sm[row * W + col] : mkc<T>(0, 0);
      }
    } else {
#pragma unroll
      for (int q = 0; q < A; ++q) v[q] = gload<K_CONV, T, LT>(a, c, j + B * q, col);
    }
    dft<A, false>(v);
#pragma unroll
    for (int k = 1; k < A; ++k) v[k] = cmul(v[k], tw[j * k]);
    if constexpr (XL) __syncthreads();   // every read of the source rows is done
#pragma unroll
    for (int k = 0; k < A; ++k) sm[xrow<A, B, XL>(j, k) * W + col] = v[k];
  }
  __syncthreads();
  // middle: DFT_B of the three components, Green multiply, inverse DFT_B
#pragma unroll 1
  for (int job = threadIdx.x; job < A * LT; job += NT) {
    const int li = job % LT, k = job / LT;
    T y[3][B];
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
#pragma unroll
      for (int jj = 0; jj < B; ++jj) y[comp][jj] = sm[xrow<A, B, XL>(jj, k) * W + comp * LT + li];
      dft<B, false>(y[comp]);
    }
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) {
      const T* g = gs + (k + A * k2) * 6;
      const T gxx = g[0], gxy = g[1], gxz = g[2], gyy = g[3], gyz = g[4], gzz = g[5];
      const T v0 = y[0][k2], v1 = y[1][k2], v2 = y[2][k2];
      y[0][k2] = cadd(cadd(cmul(gxx, v0), cmul(gxy, v1)), cmul(gxz, v2));
      y[1][k2] = cadd(cadd(cmul(gxy, v0), cmul(gyy, v1)), cmul(gyz, v2));
      y[2][k2] = cadd(cadd(cmul(gxz, v0), cmul(gyz, v1)), cmul(gzz, v2));
    }
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      dft<B, true>(y[comp]);
#pragma unroll
      for (int jj = 0; jj < B; ++jj) sm[xrow<A, B, XL>(jj, k) * W + comp * LT + li] = y[comp][jj];
    }
  }
  __syncthreads();
  // stage 1, inverse: rows below n_out to global memory
#pragma unroll 1
  for (int job = threadIdx.x; job < B * W; job += NT) {
    const int col = job % W, j = job / W;
    T v[A];
    v[0] = sm[xrow<A, B, XL>(j, 0) * W + col];
#pragma unroll
    for (int k = 1; k < A; ++k) v[k] = cmulc(sm[xrow<A, B, XL>(j, k) * W + col], tw[j * k]);
    dft<A, true>(v);
#pragma unroll
    for (int q = 0; q < A; ++q) gstore<K_CONV, T, LT>(a, c, j + B * q, col, v[q]);
  }
}

template <typename T, int LT, int NT, int MINB, int A, int B, int P0, int P1, int P2, int TMA, int XL>
int xconv2_launch(const PassArgs& a0, int64_t P0n, cudaStream_t st) {
  static_assert(NT % 32 == 0 && NT <= 448 && MINB >= 1 && MINB < 16, "variant id encodes whole warps and MINB < 16");
  constexpr int M = A * B;
  PassArgs a = a0;
  if (a.ax.M != M || a.ax.nst != 3 || a.ax.rad[0] != P0 || a.ax.rad[1] != P1 || a.ax.rad[2] != P2 || a.green ||
      a.n_in > M)
    return BDDA_BAD_ARG;
  a.ntile = (a.L + LT - 1) / LT;
  CUtensorMap tm;
  memset(&tm, 0, sizeof(tm));
  TmaTile tt;
  memset(&tt, 0, sizeof(tt));
  if (TMA && !make_tile_map<T, K_CONV, LT>(a, P0n, a.n_in, &tm, &tt))   // the plain loads
    return xconv2_launch<T, LT, NT, MINB, A, B, P0, P1, P2, 0, XL>(a0, P0n, st);
  auto kern = xconv2_kernel<T, LT, NT, MINB, A, B, P0, P1, P2, TMA, XL>;
  const size_t smem = (size_t)pencil_smem_bytes<T>(M, LT, K_CONV);
  if (smem > 227 * 1024) return BDDA_BAD_ARG;
  const int64_t nblk = P0n * a.P1 * a.ntile;
  if (nblk <= 0) return BDDA_OK;
  if (nblk > 0x7fffffff) return BDDA_BAD_ARG;
  BDDA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)nblk, NT, smem, st>>>(a, tm, tt);
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BDDA_OK;
}

// Table entry (kind K_CONV, the plan's radix sequence): variant id 2048 +
// MINB + 16 NT/32, + 256 for intermediate layout 1, + 1024 with the
// TMA-filled tile.
#define BDDA_XCONV2(T, PREC, LT, MINB, NT, A, B, P0, P1, P2, TMA, XL)                                  \
  { PREC, K_CONV, LT, MINB, 2048 + 1024 * (TMA) + 256 * (XL) + MINB + 16 * ((NT) / 32), {P0, P1, P2, 1}, \
    &xconv2_launch<T, LT, NT, MINB, A, B, P0, P1, P2, TMA, XL>, 0 }

}  // namespace bdda
