// Pencil kernels specialised at compile time for one radix sequence.
//
// The generic kernel (bdda_mvp.cu) reads the radix sequence at run time, so
// every butterfly job pays integer divisions and strides it cannot fold.
// Here the sequence (up to four radices, padded with 1), the tile width and
// the CTA size are template parameters: stage spans, twiddle strides, job
// counts and all index divisions are constants.  Each butterfly unrolls; the
// loop over a stage's rounds of jobs does not (unrolling it made the kernels
// large enough to stall on instruction fetch: the complex64 product ran 3 %
// slower).  bdda_fixed_*.cu instantiate the sequences the planner produces
// for the workloads; fixed_find() in bdda_mvp.cu dispatches to them.
#pragma once
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

template <class RS, int S, bool INV, int SRC, int DST, int KIND, typename T, int LT, int NT>
__device__ __forceinline__ void fixed_stage(const PassArgs& a, const Pen& c, T* sm, const T* tw) {
  constexpr int W = 3 * LT;
  constexpr int R = RS::r(S), B = RS::blk(S), SPAN = B / R, TSTEP = RS::M / B;
  constexpr int NJOBS = (RS::M / R) * W;
  constexpr int ITERS = (NJOBS + NT - 1) / NT;
#pragma unroll 1
  for (int it = 0; it < ITERS; ++it) {
    const int job = threadIdx.x + it * NT;
    if ((NJOBS % NT) == 0 || job < NJOBS) {
      const int col = job % W;
      const int t = job / W;
      const int b = t / SPAN;
      const int j = t - b * SPAN;
      stage_job<R, INV, SRC, DST, KIND, T, LT>(a, c, sm, tw, col, b * B + j, SPAN, j * TSTEP);
    }
  }
}

template <class RS, int SRC, int DST, typename T, int LT, int NT>
__device__ __forceinline__ void fixed_mid(const PassArgs& a, const Pen& c, T* sm, const T* gs) {
  constexpr int R = RS::r(RS::n - 1);
  constexpr int NJOBS = (RS::M / R) * LT;
  constexpr int ITERS = (NJOBS + NT - 1) / NT;
#pragma unroll 1
  for (int it = 0; it < ITERS; ++it) {
    const int job = threadIdx.x + it * NT;
    if ((NJOBS % NT) == 0 || job < NJOBS) conv_mid_job<R, SRC, DST, T, LT>(a, c, sm, gs, job / LT, job % LT);
  }
}

// NT: threads per CTA.  MINB: resident CTAs per SM the register allocation
// must allow (the __launch_bounds__ minimum); 1 = no bound.  Kernels are
// compiled with several (NT, MINB) and the autotuner picks per pass.
template <typename T, int KIND, int LT, int NT, int MINB, int R0, int R1, int R2, int R3>
__global__ void __launch_bounds__(NT, MINB) fixed_pencil_kernel(const PassArgs a) {
  using RS = RadixSeq<R0, R1, R2, R3>;
  constexpr int N = RS::n;
  extern __shared__ __align__(16) unsigned char smraw[];
  T *tw, *sm, *gs;
  int32_t* cm;
  stage_constants<T, KIND, LT>(a, smraw, RS::M, &tw, &sm, &gs, &cm, blockIdx.x);
  const Pen c = pen_of_block<T>(a, cm, blockIdx.x);
  if constexpr (KIND == K_FWD) {
    if constexpr (N == 1) {
      fixed_stage<RS, 0, false, 1, 1, KIND, T, LT, NT>(a, c, sm, tw);
    } else {
      fixed_stage<RS, 0, false, 1, 0, KIND, T, LT, NT>(a, c, sm, tw);
      __syncthreads();
      if constexpr (N >= 3) { fixed_stage<RS, 1, false, 0, 0, KIND, T, LT, NT>(a, c, sm, tw); __syncthreads(); }
      if constexpr (N >= 4) { fixed_stage<RS, 2, false, 0, 0, KIND, T, LT, NT>(a, c, sm, tw); __syncthreads(); }
      fixed_stage<RS, N - 1, false, 0, 1, KIND, T, LT, NT>(a, c, sm, tw);
    }
  } else if constexpr (KIND == K_INV) {
    if constexpr (N == 1) {
      fixed_stage<RS, 0, true, 1, 1, KIND, T, LT, NT>(a, c, sm, tw);
    } else {
      fixed_stage<RS, N - 1, true, 1, 0, KIND, T, LT, NT>(a, c, sm, tw);
      __syncthreads();
      if constexpr (N >= 4) { fixed_stage<RS, 2, true, 0, 0, KIND, T, LT, NT>(a, c, sm, tw); __syncthreads(); }
      if constexpr (N >= 3) { fixed_stage<RS, 1, true, 0, 0, KIND, T, LT, NT>(a, c, sm, tw); __syncthreads(); }
      fixed_stage<RS, 0, true, 0, 1, KIND, T, LT, NT>(a, c, sm, tw);
    }
  } else {   // K_CONV
    cp_async_wait<0>();
    __syncthreads();
    if constexpr (N == 1) {
      fixed_mid<RS, 1, 1, T, LT, NT>(a, c, sm, gs);
    } else {
      fixed_stage<RS, 0, false, 1, 0, KIND, T, LT, NT>(a, c, sm, tw);
      __syncthreads();
      if constexpr (N >= 3) { fixed_stage<RS, 1, false, 0, 0, KIND, T, LT, NT>(a, c, sm, tw); __syncthreads(); }
      if constexpr (N >= 4) { fixed_stage<RS, 2, false, 0, 0, KIND, T, LT, NT>(a, c, sm, tw); __syncthreads(); }
      fixed_mid<RS, 0, 0, T, LT, NT>(a, c, sm, gs);
      __syncthreads();
      if constexpr (N >= 4) { fixed_stage<RS, 2, true, 0, 0, KIND, T, LT, NT>(a, c, sm, tw); __syncthreads(); }
      if constexpr (N >= 3) { fixed_stage<RS, 1, true, 0, 0, KIND, T, LT, NT>(a, c, sm, tw); __syncthreads(); }
      fixed_stage<RS, 0, true, 0, 1, KIND, T, LT, NT>(a, c, sm, tw);
    }
  }
}

template <typename T, int KIND, int LT, int MINB, int NT, int R0, int R1, int R2, int R3>
int fixed_launch(const PassArgs& a0, int64_t P0, cudaStream_t st) {
  using RS = RadixSeq<R0, R1, R2, R3>;
  PassArgs a = a0;
  if (a.ax.M != RS::M) return BDDA_BAD_ARG;
  a.ntile = (a.L + LT - 1) / LT;
  auto kern = fixed_pencil_kernel<T, KIND, LT, NT, MINB, R0, R1, R2, R3>;
  const size_t smem = (size_t)pencil_smem_bytes<T>(RS::M, LT, KIND);
  if (smem > 227 * 1024) return BDDA_BAD_ARG;
  const int64_t nblk = P0 * a.P1 * a.ntile;
  if (nblk <= 0) return BDDA_OK;
  if (nblk > 0x7fffffff) return BDDA_BAD_ARG;
  BDDA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)nblk, NT, smem, st>>>(a);
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BDDA_OK;
}

// Table entry of a specialised kernel with 256 threads per CTA (variant id =
// MINB) or NT threads (variant id = MINB + 16 NT/32: the CTA size that makes
// the stages' butterfly jobs fill whole rounds of threads).
#define BDDA_FIXED(T, PREC, KIND, LT, MINB, R0, R1, R2, R3) \
  { PREC, KIND, LT, MINB, MINB, {R0, R1, R2, R3}, &fixed_launch<T, KIND, LT, MINB, 256, R0, R1, R2, R3> }
#define BDDA_FIXED_NT(T, PREC, KIND, LT, MINB, NT, R0, R1, R2, R3)                              \
  { PREC, KIND, LT, MINB, MINB + 16 * ((NT) / 32), {R0, R1, R2, R3},                              \
    &fixed_launch<T, KIND, LT, MINB, NT, R0, R1, R2, R3> }

}  // namespace bdda
