// Fourier-neural-operator warm start for the block solvers: hand-written
// forward, backward, optimiser and inference kernels (no counterpart in the
// reference, whose solvers start from X0 = 0, bl_krylov.py:84-85,146).
//
// Network (per sample = one particle lattice x one orientation, B samples of
// one lattice per call), activations FP32, cell-major [B][Nx][Ny][Nz][C]:
//   lift      v0 = P x + p                      (cin -> width, pointwise)
//   layer l   v   = act(W_l v + b_l + K_l v)     (l = 0..layers-1, no act on the last)
//             K_l v = Re IDFT( R_l . DFT(v) ) on the `modes` lowest frequencies
//             per axis (|f| < modes/2), R_l one complex width x width matrix per mode
//   project   y = Q2 gelu(Q1 v + q1) + q2        (width -> proj -> cout)
// The truncated DFT is separable: three axis transforms, each a small complex
// matrix product over the kept modes (no full-length FFT is formed).  act =
// GELU (erf form).  Parameters are one flat FP32 array (layout below).
#include <cmath>
#include <cstring>

#include "bdda_internal.h"
#include "bdda_small.cuh"

namespace bdda {
namespace {

struct FnoCfg {
  int cin, width, cout, proj, layers, modes;
};

// Longest lattice axis the network runs on (its truncated-DFT tables hold
// kMaxAxis x modes entries per axis).
constexpr int kMaxAxis = 512;

// parameter offsets (floats)
struct FnoParams {
  size_t P, p, R[8], W[8], b[8], Q1, q1, Q2, q2, total;
};

FnoParams param_layout(const FnoCfg& c) {
  FnoParams o;
  const size_t K = (size_t)c.modes * c.modes * c.modes;
  size_t off = 0;
  o.P = off; off += (size_t)c.cin * c.width;
  o.p = off; off += c.width;
  for (int l = 0; l < c.layers; ++l) {
    o.R[l] = off; off += K * c.width * c.width * 2;
    o.W[l] = off; off += (size_t)c.width * c.width;
    o.b[l] = off; off += c.width;
  }
  o.Q1 = off; off += (size_t)c.width * c.proj;
  o.q1 = off; off += c.proj;
  o.Q2 = off; off += (size_t)c.proj * c.cout;
  o.q2 = off; off += c.cout;
  o.total = off;
  return o;
}

bool cfg_ok(const bdda_fno_config* c) {
  return c && c->cin >= 1 && c->cin <= 64 && c->width >= 1 && c->width <= 64 && c->cout >= 1 && c->cout <= 64 &&
         c->proj >= 1 && c->proj <= 128 && c->layers >= 1 && c->layers <= 8 && c->modes >= 2 && c->modes <= 32 &&
         (c->modes % 2) == 0;
}

FnoCfg to_cfg(const bdda_fno_config* c) { return FnoCfg{c->cin, c->width, c->cout, c->proj, c->layers, c->modes}; }

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// ---- axis transform: out[o][p][i] = scale * sum_q in[o][q][i] T[q][p] ----------------------
// T complex (Q x P).  IN_C: input complex (else real).  OUT: 0 complex store,
// 1 real part store, 2 real part added to out.
template <bool IN_C, int OUT>
__global__ void __launch_bounds__(256) axis_transform_kernel(const void* in, void* out, const float2* T, int64_t O,
                                                             int Q, int P, int64_t I, float scale) {
  extern __shared__ float2 tsm[];
  for (int e = threadIdx.x; e < Q * P; e += blockDim.x) tsm[e] = T[e];
  __syncthreads();
  constexpr int PC = 8;
  const int64_t icount = I;
  const int64_t nitem = O * icount;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nitem; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = t / icount, i = t - o * icount;
    for (int p0 = 0; p0 < P; p0 += PC) {
      float2 acc[PC];
#pragma unroll
      for (int j = 0; j < PC; ++j) acc[j] = make_float2(0.f, 0.f);
      for (int q = 0; q < Q; ++q) {
        float2 x;
        if constexpr (IN_C) x = static_cast<const float2*>(in)[(o * Q + q) * icount + i];
        else x = make_float2(static_cast<const float*>(in)[(o * Q + q) * icount + i], 0.f);
        const float2* tr = tsm + q * P + p0;
#pragma unroll
        for (int j = 0; j < PC; ++j) {
          if (p0 + j < P) {
            const float2 w = tr[j];
            acc[j].x = fmaf(x.x, w.x, fmaf(-x.y, w.y, acc[j].x));
            acc[j].y = fmaf(x.x, w.y, fmaf(x.y, w.x, acc[j].y));
          }
        }
      }
#pragma unroll
      for (int j = 0; j < PC; ++j) {
        const int p = p0 + j;
        if (p < P) {
          const int64_t idx = (o * P + p) * icount + i;
          if constexpr (OUT == 0) static_cast<float2*>(out)[idx] = make_float2(scale * acc[j].x, scale * acc[j].y);
          else if constexpr (OUT == 1) static_cast<float*>(out)[idx] = scale * acc[j].x;
          else static_cast<float*>(out)[idx] += scale * acc[j].x;
        }
      }
    }
  }
}

// ---- spectral mixing ----------------------------------------------------------------------
// S[b][k][o] = sum_i R[k][i][o] A[b][k][i]
__global__ void spec_mix_kernel(const float2* A, const float2* R, float2* S, int B, int K, int W) {
  const int64_t n = (int64_t)B * K * W;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int o = (int)(t % W);
    const int64_t bk = t / W;
    const int k = (int)(bk % K);
    const float2* a = A + bk * W;
    const float2* r = R + (int64_t)k * W * W + o;
    float2 acc = make_float2(0.f, 0.f);
    for (int i = 0; i < W; ++i) {
      const float2 x = a[i], w = r[(int64_t)i * W];
      acc.x = fmaf(x.x, w.x, fmaf(-x.y, w.y, acc.x));
      acc.y = fmaf(x.x, w.y, fmaf(x.y, w.x, acc.y));
    }
    S[t] = acc;
  }
}

// gA[b][k][i] = sum_o conj(R[k][i][o]) gS[b][k][o]
__global__ void spec_mix_bwd_data_kernel(const float2* gS, const float2* R, float2* gA, int B, int K, int W) {
  const int64_t n = (int64_t)B * K * W;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % W);
    const int64_t bk = t / W;
    const int k = (int)(bk % K);
    const float2* g = gS + bk * W;
    const float2* r = R + ((int64_t)k * W + i) * W;
    float2 acc = make_float2(0.f, 0.f);
    for (int o = 0; o < W; ++o) {
      const float2 x = g[o], w = r[o];   // conj(w) x
      acc.x = fmaf(w.x, x.x, fmaf(w.y, x.y, acc.x));
      acc.y = fmaf(w.x, x.y, fmaf(-w.y, x.x, acc.y));
    }
    gA[t] = acc;
  }
}

// gR[k][i][o] += sum_b conj(A[b][k][i]) gS[b][k][o]
__global__ void spec_mix_bwd_weight_kernel(const float2* A, const float2* gS, float2* gR, int B, int K, int W) {
  const int64_t n = (int64_t)K * W * W;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int o = (int)(t % W);
    const int64_t ki = t / W;
    const int i = (int)(ki % W);
    const int k = (int)(ki / W);
    float2 acc = gR[t];
    for (int b = 0; b < B; ++b) {
      const float2 a = A[((int64_t)b * K + k) * W + i], g = gS[((int64_t)b * K + k) * W + o];
      acc.x = fmaf(a.x, g.x, fmaf(a.y, g.y, acc.x));
      acc.y = fmaf(a.x, g.y, fmaf(-a.y, g.x, acc.y));
    }
    gR[t] = acc;
  }
}

// ---- pointwise layers -----------------------------------------------------------------------
// z[m][o] = sum_i x[m][i] Wt[i][o] + bias[o] (+ add[m][o]); y = act(z) (act 0 none, 1 GELU)
template <int CI, int CO>
__global__ void __launch_bounds__(256) pointwise_fwd_kernel(const float* x, const float* Wt, const float* bias,
                                                            const float* add, float* z, float* y, int64_t M,
                                                            int act) {
  __shared__ float ws[CI * CO];
  __shared__ float bs[CO];
  for (int e = threadIdx.x; e < CI * CO; e += blockDim.x) ws[e] = Wt[e];
  for (int e = threadIdx.x; e < CO; e += blockDim.x) bs[e] = bias[e];
  __syncthreads();
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < M; m += (int64_t)gridDim.x * blockDim.x) {
    float xi[CI];
#pragma unroll
    for (int i = 0; i < CI; ++i) xi[i] = x[m * CI + i];
#pragma unroll 4
    for (int o = 0; o < CO; ++o) {
      float acc = bs[o];
#pragma unroll
      for (int i = 0; i < CI; ++i) acc = fmaf(xi[i], ws[i * CO + o], acc);
      if (add) acc += add[m * CO + o];
      if (z) z[m * CO + o] = acc;
      y[m * CO + o] = act ? gelu(acc) : acc;
    }
  }
}

// gz = gy act'(z) (stored); gx[m][i] = sum_o Wt[i][o] gz[m][o] (set or added)
template <int CI, int CO>
__global__ void __launch_bounds__(256) pointwise_bwd_data_kernel(const float* gy, const float* z, const float* Wt,
                                                                 float* gz, float* gx, int64_t M, int act,
                                                                 int accumulate) {
  __shared__ float ws[CI * CO];
  for (int e = threadIdx.x; e < CI * CO; e += blockDim.x) ws[e] = Wt[e];
  __syncthreads();
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < M; m += (int64_t)gridDim.x * blockDim.x) {
    float g[CO];
#pragma unroll
    for (int o = 0; o < CO; ++o) {
      float v = gy[m * CO + o];
      if (act) v *= gelu_grad(z[m * CO + o]);
      g[o] = v;
      gz[m * CO + o] = v;
    }
    if (!gx) continue;
#pragma unroll 4
    for (int i = 0; i < CI; ++i) {
      float acc = 0.f;
#pragma unroll
      for (int o = 0; o < CO; ++o) acc = fmaf(g[o], ws[i * CO + o], acc);
      if (accumulate) gx[m * CI + i] += acc;
      else gx[m * CI + i] = acc;
    }
  }
}

// gWt[i][o] += sum_m x[m][i] gz[m][o]; gb[o] += sum_m gz[m][o]  (per-CTA partials, atomics)
template <int CI, int CO>
__global__ void __launch_bounds__(256) pointwise_bwd_weight_kernel(const float* x, const float* gz, float* gWt,
                                                                   float* gb, int64_t M) {
  __shared__ float xs[32][CI];
  __shared__ float gs[32][CO];
  constexpr int NE = CI * CO + CO;
  float acc[(NE + 255) / 256];
#pragma unroll
  for (int j = 0; j < (NE + 255) / 256; ++j) acc[j] = 0.f;
  const int64_t rows_per = (M + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = blockIdx.x * rows_per, r1 = min(M, r0 + rows_per);
  for (int64_t rb = r0; rb < r1; rb += 32) {
    const int nr = (int)min((int64_t)32, r1 - rb);
    for (int e = threadIdx.x; e < 32 * CI; e += blockDim.x) {
      const int r = e / CI, i = e - r * CI;
      xs[r][i] = r < nr ? x[(rb + r) * CI + i] : 0.f;
    }
    for (int e = threadIdx.x; e < 32 * CO; e += blockDim.x) {
      const int r = e / CO, o = e - r * CO;
      gs[r][o] = r < nr ? gz[(rb + r) * CO + o] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < (NE + 255) / 256; ++j) {
      const int e = threadIdx.x + 256 * j;
      if (e < CI * CO) {
        const int i = e / CO, o = e - i * CO;
        float s = 0.f;
        for (int r = 0; r < 32; ++r) s = fmaf(xs[r][i], gs[r][o], s);
        acc[j] += s;
      } else if (e < NE) {
        const int o = e - CI * CO;
        float s = 0.f;
        for (int r = 0; r < 32; ++r) s += gs[r][o];
        acc[j] += s;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < (NE + 255) / 256; ++j) {
    const int e = threadIdx.x + 256 * j;
    if (e < CI * CO) atomicAdd(&gWt[e], acc[j]);
    else if (e < NE) atomicAdd(&gb[e - CI * CO], acc[j]);
  }
}

// ---- tensor-core pointwise layers --------------------------------------------------------------
// The CI x CO maps whose sides are multiples of 8 (the width x width layers and
// the first projection) run on the tensor cores: mma.sync m16n8k8 with TF32
// operands and FP32 accumulation, each product split in three,
// a b ~ a_hi b_hi + a_hi b_lo + a_lo b_hi with a_hi = tf32(a), a_lo = tf32(a - a_hi),
// which keeps the accuracy of the FP32 kernels (the dropped a_lo b_lo term is
// below FP32 rounding).  Fragments of m16n8k8 (lane = 4 g + t):
// A (16 x 8) a0 (g, t), a1 (g + 8, t), a2 (g, t + 4), a3 (g + 8, t + 4);
// B (8 x 8) b0 (t, g), b1 (t + 4, g); D (16 x 8) d0 (g, 2t), d1 (g, 2t + 1),
// d2 (g + 8, 2t), d3 (g + 8, 2t + 1).  Each warp owns 16-row tiles of the
// activations, staged in shared memory by 16-byte loads.
__device__ __forceinline__ uint32_t tf32_of(float v) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return r;
}
__device__ __forceinline__ void split_tf32(float v, uint32_t& hi, uint32_t& lo) {
  hi = tf32_of(v);
  lo = tf32_of(v - __uint_as_float(hi));
}
__device__ __forceinline__ void mma_tf32(float* d, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
// d += A B over K = 8 KS columns: A from a 16-row tile at `at` (row stride AS),
// B fragments from split matrices bh / bl (row k, column n, row stride BS)
template <int KS, int NS, int AS, int BS>
__device__ __forceinline__ void tile_mma(float (*acc)[4], const float* at, const uint32_t* bh, const uint32_t* bl,
                                         int g, int t) {
#pragma unroll
  for (int ks = 0; ks < KS; ++ks) {
    uint32_t ah[4], al[4];
    split_tf32(at[g * AS + ks * 8 + t], ah[0], al[0]);
    split_tf32(at[(g + 8) * AS + ks * 8 + t], ah[1], al[1]);
    split_tf32(at[g * AS + ks * 8 + t + 4], ah[2], al[2]);
    split_tf32(at[(g + 8) * AS + ks * 8 + t + 4], ah[3], al[3]);
#pragma unroll
    for (int ns = 0; ns < NS; ++ns) {
      const int wi = (ks * 8 + t) * BS + ns * 8 + g;
      const uint32_t h[2] = {bh[wi], bh[wi + 4 * BS]}, l[2] = {bl[wi], bl[wi + 4 * BS]};
      mma_tf32(acc[ns], al, h);
      mma_tf32(acc[ns], ah, l);
      mma_tf32(acc[ns], ah, h);
    }
  }
}

// stage rows m0 .. m0+R-1 of a row-major (M x C) array into a tile of row stride TS (zero past M)
template <int R, int C, int TS>
__device__ __forceinline__ void stage_rows(const float* src, int64_t m0, int64_t M, float* tile, int lane) {
  for (int e = lane; e < R * C / 4; e += 32) {
    const int r = e / (C / 4), c4 = e - r * (C / 4);
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (m0 + r < M) v = *reinterpret_cast<const float4*>(src + (m0 + r) * C + 4 * c4);
    float* d = tile + r * TS + 4 * c4;
    d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
  }
}

// as pointwise_fwd_kernel: z = x Wt + bias (+ add), y = act(z)
template <int CI, int CO>
__global__ void __launch_bounds__(256) pointwise_fwd_tc_kernel(const float* x, const float* Wt, const float* bias,
                                                               const float* add, float* z, float* y, int64_t M,
                                                               int act) {
  static_assert(CI % 8 == 0 && CO % 8 == 0 && CI <= 64 && CO <= 64, "tensor-core tile shapes");
  constexpr int WS = CO + 8, XS = CI + 4;   // padded strides: conflict-free fragment reads
  __shared__ uint32_t wh[CI * WS], wl[CI * WS];
  __shared__ __align__(16) float xs[8][16 * XS];
  __shared__ float bs[CO];
  for (int e = threadIdx.x; e < CI * CO; e += blockDim.x) {
    const int i = e / CO, o = e - i * CO;
    split_tf32(Wt[e], wh[i * WS + o], wl[i * WS + o]);
  }
  for (int e = threadIdx.x; e < CO; e += blockDim.x) bs[e] = bias[e];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float* xt = xs[warp];
  const int64_t ntile = (M + 15) / 16;
  for (int64_t tile = blockIdx.x * 8LL + warp; tile < ntile; tile += (int64_t)gridDim.x * 8) {
    const int64_t m0 = tile * 16;
    stage_rows<16, CI, XS>(x, m0, M, xt, lane);
    __syncwarp();
    float acc[CO / 8][4];
#pragma unroll
    for (int ns = 0; ns < CO / 8; ++ns) acc[ns][0] = acc[ns][1] = acc[ns][2] = acc[ns][3] = 0.f;
    tile_mma<CI / 8, CO / 8, XS, WS>(acc, xt, wh, wl, g, t);
    __syncwarp();
#pragma unroll
    for (int ns = 0; ns < CO / 8; ++ns) {
#pragma unroll
      for (int hr = 0; hr < 2; ++hr) {
        const int64_t m = m0 + g + 8 * hr;
        if (m >= M) continue;
        const int o = ns * 8 + 2 * t;
        float v0 = acc[ns][2 * hr] + bs[o], v1 = acc[ns][2 * hr + 1] + bs[o + 1];
        if (add) {
          const float2 a2 = *reinterpret_cast<const float2*>(add + m * CO + o);
          v0 += a2.x;
          v1 += a2.y;
        }
        if (z) *reinterpret_cast<float2*>(z + m * CO + o) = make_float2(v0, v1);
        *reinterpret_cast<float2*>(y + m * CO + o) = act ? make_float2(gelu(v0), gelu(v1)) : make_float2(v0, v1);
      }
    }
  }
}

// as pointwise_bwd_data_kernel: gz = gy act'(z) (stored); gx = gz Wt^T (set or added)
template <int CI, int CO>
__global__ void __launch_bounds__(128) pointwise_bwd_data_tc_kernel(const float* gy, const float* z, const float* Wt,
                                                                    float* gz, float* gx, int64_t M, int act,
                                                                    int accumulate) {
  static_assert(CI % 8 == 0 && CO % 8 == 0 && CI <= 64 && CO <= 64, "tensor-core tile shapes");
  constexpr int WS = CI + 8, GS = CO + 4, NW = 4;
  __shared__ uint32_t wh[CO * WS], wl[CO * WS];   // W transposed: row o, column i
  __shared__ __align__(16) float gsm[NW][16 * GS];
  for (int e = threadIdx.x; e < CI * CO; e += blockDim.x) {
    const int i = e / CO, o = e - i * CO;
    split_tf32(Wt[e], wh[o * WS + i], wl[o * WS + i]);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float* gt = gsm[warp];
  const int64_t ntile = (M + 15) / 16;
  for (int64_t tile = blockIdx.x * (int64_t)NW + warp; tile < ntile; tile += (int64_t)gridDim.x * NW) {
    const int64_t m0 = tile * 16;
    for (int e = lane; e < 16 * CO / 4; e += 32) {   // gz tile = gy act'(z), written back
      const int r = e / (CO / 4), c4 = e - r * (CO / 4);
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (m0 + r < M) {
        const int64_t off = (m0 + r) * CO + 4 * c4;
        v = *reinterpret_cast<const float4*>(gy + off);
        if (act) {
          const float4 zz = *reinterpret_cast<const float4*>(z + off);
          v.x *= gelu_grad(zz.x); v.y *= gelu_grad(zz.y); v.z *= gelu_grad(zz.z); v.w *= gelu_grad(zz.w);
        }
        *reinterpret_cast<float4*>(gz + off) = v;
      }
      float* d = gt + r * GS + 4 * c4;
      d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
    }
    __syncwarp();
    if (gx) {
      float acc[CI / 8][4];
#pragma unroll
      for (int ns = 0; ns < CI / 8; ++ns) acc[ns][0] = acc[ns][1] = acc[ns][2] = acc[ns][3] = 0.f;
      tile_mma<CO / 8, CI / 8, GS, WS>(acc, gt, wh, wl, g, t);
#pragma unroll
      for (int ns = 0; ns < CI / 8; ++ns) {
#pragma unroll
        for (int hr = 0; hr < 2; ++hr) {
          const int64_t m = m0 + g + 8 * hr;
          if (m >= M) continue;
          float2* dst = reinterpret_cast<float2*>(gx + m * CI + ns * 8 + 2 * t);
          float2 v = make_float2(acc[ns][2 * hr], acc[ns][2 * hr + 1]);
          if (accumulate) {
            const float2 o = *dst;
            v.x += o.x;
            v.y += o.y;
          }
          *dst = v;
        }
      }
    }
    __syncwarp();
  }
}

// as pointwise_bwd_weight_kernel: gWt += x^T gz, gb += column sums of gz.  K
// runs over the rows: each warp takes 16-row blocks of this CTA's row range,
// A = x^T (CI x 8 per step), B = gz (8 x CO); warps meet in shared memory,
// then one atomic add per element per CTA.
template <int CI, int CO>
__global__ void __launch_bounds__(128) pointwise_bwd_weight_tc_kernel(const float* x, const float* gz, float* gWt,
                                                                      float* gb, int64_t M) {
  static_assert(CI % 16 == 0 && CO % 8 == 0 && CI <= 64 && CO <= 64, "tensor-core tile shapes");
  constexpr int XS = CI + 8, GS = CO + 8, NW = 4, RB = 16;   // row = sample m; RB rows per warp block
  __shared__ __align__(16) float xs[NW][RB * XS];
  __shared__ __align__(16) float gs[NW][RB * GS];
  __shared__ float red[CI * CO + CO];
  for (int e = threadIdx.x; e < CI * CO + CO; e += blockDim.x) red[e] = 0.f;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float* xt = xs[warp];
  float* gt = gs[warp];
  const int64_t rows_per = (M + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = blockIdx.x * rows_per, r1 = min(M, r0 + rows_per);
  float acc[CI / 16][CO / 8][4];
#pragma unroll
  for (int mt = 0; mt < CI / 16; ++mt)
#pragma unroll
    for (int ns = 0; ns < CO / 8; ++ns) acc[mt][ns][0] = acc[mt][ns][1] = acc[mt][ns][2] = acc[mt][ns][3] = 0.f;
  float bsum[(CO + 31) / 32];
#pragma unroll
  for (int q = 0; q < (CO + 31) / 32; ++q) bsum[q] = 0.f;
  for (int64_t rb = r0 + (int64_t)RB * warp; rb < r1; rb += (int64_t)RB * NW) {
    stage_rows<RB, CI, XS>(x, rb, r1, xt, lane);
    stage_rows<RB, CO, GS>(gz, rb, r1, gt, lane);
    __syncwarp();
#pragma unroll
    for (int ks = 0; ks < RB / 8; ++ks) {   // 8 samples per step
      const int k0 = ks * 8;
      uint32_t bh[CO / 8][2], bl[CO / 8][2];
#pragma unroll
      for (int ns = 0; ns < CO / 8; ++ns) {
        split_tf32(gt[(k0 + t) * GS + ns * 8 + g], bh[ns][0], bl[ns][0]);
        split_tf32(gt[(k0 + t + 4) * GS + ns * 8 + g], bh[ns][1], bl[ns][1]);
      }
#pragma unroll
      for (int mt = 0; mt < CI / 16; ++mt) {
        uint32_t ah[4], al[4];   // A[i][m] = x[m][i]
        split_tf32(xt[(k0 + t) * XS + mt * 16 + g], ah[0], al[0]);
        split_tf32(xt[(k0 + t) * XS + mt * 16 + g + 8], ah[1], al[1]);
        split_tf32(xt[(k0 + t + 4) * XS + mt * 16 + g], ah[2], al[2]);
        split_tf32(xt[(k0 + t + 4) * XS + mt * 16 + g + 8], ah[3], al[3]);
#pragma unroll
        for (int ns = 0; ns < CO / 8; ++ns) {
          mma_tf32(acc[mt][ns], al, bh[ns]);
          mma_tf32(acc[mt][ns], ah, bl[ns]);
          mma_tf32(acc[mt][ns], ah, bh[ns]);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < (CO + 31) / 32; ++q) {   // bias gradient: column sums
      const int o = lane + 32 * q;
      if (o < CO)
        for (int r = 0; r < RB; ++r) bsum[q] += gt[r * GS + o];
    }
    __syncwarp();
  }
#pragma unroll
  for (int q = 0; q < (CO + 31) / 32; ++q)
    if (lane + 32 * q < CO) atomicAdd(&red[CI * CO + lane + 32 * q], bsum[q]);
#pragma unroll
  for (int mt = 0; mt < CI / 16; ++mt)
#pragma unroll
    for (int ns = 0; ns < CO / 8; ++ns)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int i = mt * 16 + g + 8 * (q >> 1), o = ns * 8 + 2 * t + (q & 1);
        atomicAdd(&red[i * CO + o], acc[mt][ns][q]);
      }
  __syncthreads();
  for (int e = threadIdx.x; e < CI * CO; e += blockDim.x) atomicAdd(&gWt[e], red[e]);
  for (int e = threadIdx.x; e < CO; e += blockDim.x) atomicAdd(&gb[e], red[CI * CO + e]);
}

// ---- loss: masked relative squared error per sample -------------------------------------------
// L = (1/B) sum_b sum_m mask |y - t|^2 / sum_m mask |t|^2 ; gy = dL/dy
__global__ void loss_kernel(const float* y, const float* t, const float* mask, int64_t ncell, int C, int B,
                            const double* den, float* gy, double* loss) {
  const int64_t n = (int64_t)B * ncell * C;
  double local = 0.0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t bm = e / C;
    const int b = (int)(bm / ncell);
    const int64_t m = bm - (int64_t)b * ncell;
    const float w = mask[m];
    const float d = y[e] - t[e];
    const double s = 1.0 / (den[b] * B);
    gy[e] = (float)(2.0 * s * w * d);
    local += s * w * d * d;
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, local);
}

// den[b] = sum_m mask |t[b]|^2
__global__ void loss_den_kernel(const float* t, const float* mask, int64_t ncell, int C, double* den) {
  const int b = blockIdx.y;
  double local = 0.0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ncell * C; e += (int64_t)gridDim.x * blockDim.x) {
    const float v = t[(int64_t)b * ncell * C + e];
    local += mask[e / C] * (double)v * v;
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(&den[b], local);
}

// ---- Adam -------------------------------------------------------------------------------------
__global__ void adam_kernel(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2,
                            float eps, float c1, float c2, float wd) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i] + wd * p[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// ---- features and warm start ---------------------------------------------------------------------
// x[b][cell][:] = (mask, Re/Im chi_x, chi_y, chi_z, Re/Im J_x, J_y, J_z / scale) with
// J = B / diag the Jacobi guess of orientation b; zero outside the particle
// except the mask channel
__global__ void features_kernel(const int32_t* cell_map, int64_t ncell, int n_occ, int L, const double2* diag,
                                const double2* B, const double* chi, const double* scale, float* x, int cin) {
  const int64_t n = (int64_t)L * ncell;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(t / ncell);
    const int64_t cell = t - (int64_t)b * ncell;
    float* o = x + t * cin;
    const int mi = cell_map[cell];
    for (int c = 0; c < cin; ++c) o[c] = 0.f;
    if (mi < 0 || mi >= n_occ) continue;
    o[0] = 1.f;
    for (int c = 0; c < 6; ++c) o[1 + c] = (float)chi[c];
    const double s = 1.0 / scale[b];
    for (int a = 0; a < 3; ++a) {
      const int64_t r = 3 * (int64_t)mi + a;
      const double2 j = zdiv(B[r * L + b], diag[r]);
      o[7 + 2 * a] = (float)(j.x * s);
      o[8 + 2 * a] = (float)(j.y * s);
    }
  }
}

// scale[b] = sqrt(mean_r |B[r][b] / diag[r]|^2)
__global__ void jacobi_scale_kernel(const double2* diag, const double2* B, int64_t rows, int L, double* scale) {
  const int b = blockIdx.x;
  double local = 0.0;
  for (int64_t r = threadIdx.x; r < rows; r += blockDim.x) {
    const double2 j = zdiv(B[r * L + b], diag[r]);
    local += j.x * j.x + j.y * j.y;
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = local;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    scale[b] = sqrt(s / (double)rows) + 1e-300;
  }
}

// X0[3m + a][b] = J + scale[b] (y_re + i y_im) at the occupied cells
__global__ void warm_start_kernel(const int32_t* cell_map, int64_t ncell, int n_occ, int L, const double2* diag,
                                  const double2* B, const double* scale, const float* y, int cout, double2* X0) {
  const int64_t n = (int64_t)L * ncell;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(t / ncell);
    const int64_t cell = t - (int64_t)b * ncell;
    const int mi = cell_map[cell];
    if (mi < 0 || mi >= n_occ) continue;
    const float* o = y + t * cout;
    for (int a = 0; a < 3; ++a) {
      const int64_t r = 3 * (int64_t)mi + a;
      const double2 j = zdiv(B[r * L + b], diag[r]);
      X0[r * L + b] = make_double2(j.x + scale[b] * o[2 * a], j.y + scale[b] * o[2 * a + 1]);
    }
  }
}

// target t[b][cell][:] = (X - J) / scale at occupied cells, 0 elsewhere
__global__ void target_kernel(const int32_t* cell_map, int64_t ncell, int n_occ, int L, const double2* diag,
                              const double2* B, const double2* X, const double* scale, float* t6) {
  const int64_t n = (int64_t)L * ncell;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(t / ncell);
    const int64_t cell = t - (int64_t)b * ncell;
    const int mi = cell_map[cell];
    float* o = t6 + t * 6;
    for (int c = 0; c < 6; ++c) o[c] = 0.f;
    if (mi < 0 || mi >= n_occ) continue;
    const double s = 1.0 / scale[b];
    for (int a = 0; a < 3; ++a) {
      const int64_t r = 3 * (int64_t)mi + a;
      const double2 j = zdiv(B[r * L + b], diag[r]);
      const double2 x = X[r * L + b];
      o[2 * a] = (float)((x.x - j.x) * s);
      o[2 * a + 1] = (float)((x.y - j.y) * s);
    }
  }
}

__global__ void mask_kernel(const int32_t* cell_map, int64_t ncell, float* mask) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += (int64_t)gridDim.x * blockDim.x)
    mask[t] = cell_map[t] >= 0 ? 1.f : 0.f;
}

// ---- host orchestration -----------------------------------------------------------------------------
#define BDDA_TRY_F(expr)           \
  do {                             \
    int s_ = (expr);               \
    if (s_ != BDDA_OK) return s_;  \
  } while (0)

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

// forward (dir = -1) or inverse (dir = +1) transform table of one axis: T[q][p]
// forward: q = cell n (N), p = mode slot j (M): exp(-2 pi i f_j n / N)
// inverse: q = mode slot j (M), p = cell n (N): exp(+2 pi i f_j n / N)
void axis_table(int N, int M, bool inverse, std::vector<float2>& T) {
  T.resize((size_t)N * M);
  const int h = M / 2;
  for (int j = 0; j < M; ++j) {
    const int f = j < h ? j : N - (M - j);
    for (int n = 0; n < N; ++n) {
      const long double ang = 2.0L * 3.14159265358979323846264338327950288L * (long double)((int64_t)f * n % N) / N;
      const float c = (float)cosl(ang), s = (float)sinl(ang);
      if (!inverse) T[(size_t)n * M + j] = make_float2(c, -s);
      else T[(size_t)j * N + n] = make_float2(c, s);
    }
  }
}

// workspace carve-up for one (B, lattice) shape
struct FnoWork {
  size_t x, v[9], z[9], zq, h, y, A[8], S, t1, t2, gv, gv2, gz, gh, gs, gS, gA, tabs, mask, tgt, gy, den, chi, loss,
      total;
};

struct Shape {
  int B, n[3];
  int64_t ncell, M;    // cells, rows = B * ncell
  int K;               // modes^3
};

FnoWork work_layout(const FnoCfg& c, const Shape& s) {
  FnoWork w;
  size_t off = 0;
  auto take = [&](size_t bytes) { const size_t o = off; off = (off + bytes + 255) & ~(size_t)255; return o; };
  const int64_t M = s.M;
  const int Wd = c.width, md = c.modes;
  w.x = take(M * c.cin * 4);
  for (int l = 0; l <= c.layers; ++l) w.v[l] = take(M * Wd * 4);
  for (int l = 0; l < c.layers; ++l) w.z[l] = take(M * Wd * 4);
  w.zq = take(M * c.proj * 4);
  w.h = take(M * c.proj * 4);
  w.y = take(M * c.cout * 4);
  for (int l = 0; l < c.layers; ++l) w.A[l] = take((size_t)s.B * s.K * Wd * 8);
  w.S = take((size_t)s.B * s.K * Wd * 8);
  // axis intermediates: after z: B Nx Ny md Wd; after y: B Nx md md Wd (complex)
  const size_t t1 = (size_t)s.B * s.n[0] * s.n[1] * md * Wd * 8;
  const size_t t2 = (size_t)s.B * s.n[0] * md * md * Wd * 8;
  w.t1 = take(t1);
  w.t2 = take(t2);
  w.gv = take(M * std::max(Wd, c.proj) * 4);
  w.gv2 = take(M * std::max(Wd, c.proj) * 4);
  w.gz = take(M * std::max(Wd, c.proj) * 4);
  w.gh = take(M * c.proj * 4);
  w.gs = take(M * Wd * 4);
  w.gS = take((size_t)s.B * s.K * Wd * 8);
  w.gA = take((size_t)s.B * s.K * Wd * 8);
  w.tabs = take((size_t)6 * kMaxAxis * 32 * 8);
  w.mask = take(s.ncell * 4);
  w.tgt = take(M * c.cout * 4);
  w.gy = take(M * c.cout * 4);
  w.den = take((size_t)s.B * 8);
  w.chi = take(6 * 8);
  w.loss = take(64);
  w.total = off;
  return w;
}

struct Ctx {
  FnoCfg c;
  FnoParams pl;
  Shape s;
  FnoWork wl;
  unsigned char* w;
  const float* prm;
  float* grad;
  cudaStream_t st;
  float2* tab[6];   // fwd z, y, x; inv x, y, z
};

template <typename Tp>
Tp* at(Ctx& x, size_t off) { return reinterpret_cast<Tp*>(x.w + off); }

int upload_tables(Ctx& x) {
  const int md = x.c.modes;
  float2* base = at<float2>(x, x.wl.tabs);
  const int ax_of[6] = {2, 1, 0, 0, 1, 2};
  std::vector<float2> T;
  for (int t = 0; t < 6; ++t) {
    const int N = x.s.n[ax_of[t]];
    axis_table(N, md, t >= 3, T);
    x.tab[t] = base + (size_t)t * kMaxAxis * 32;
    BDDA_CUDA_TRY(cudaMemcpyAsync(x.tab[t], T.data(), T.size() * sizeof(float2), cudaMemcpyHostToDevice, x.st));
  }
  return BDDA_OK;
}

template <bool IN_C, int OUT>
int transform(Ctx& x, const void* in, void* out, const float2* T, int64_t O, int Q, int P, int64_t I, float scale) {
  const size_t smem = (size_t)Q * P * sizeof(float2);
  auto k = axis_transform_kernel<IN_C, OUT>;
  BDDA_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k<<<grid_for(O * I), 256, smem, x.st>>>(in, out, T, O, Q, P, I, scale);
  count_launch();
  BDDA_CUDA_TRY(cudaGetLastError());
  return BDDA_OK;
}

// truncated forward DFT of a real [B][Nx][Ny][Nz][W] field into A [B][md^3][W] (scale s)
int dft_fwd(Ctx& x, const float* v, float2* A, float scale) {
  const int B = x.s.B, Nx = x.s.n[0], Ny = x.s.n[1], Nz = x.s.n[2], md = x.c.modes, W = x.c.width;
  float2* t1 = at<float2>(x, x.wl.t1);
  float2* t2 = at<float2>(x, x.wl.t2);
  BDDA_TRY_F((transform<false, 0>(x, v, t1, x.tab[0], (int64_t)B * Nx * Ny, Nz, md, W, 1.f)));
  BDDA_TRY_F((transform<true, 0>(x, t1, t2, x.tab[1], (int64_t)B * Nx, Ny, md, (int64_t)md * W, 1.f)));
  return transform<true, 0>(x, t2, A, x.tab[2], (int64_t)B, Nx, md, (int64_t)md * md * W, scale);
}

// real part of the truncated inverse DFT of S [B][md^3][W] into [B][Nx][Ny][Nz][W] (scale s; add)
int dft_inv(Ctx& x, const float2* S, float* out, float scale, bool add) {
  const int B = x.s.B, Nx = x.s.n[0], Ny = x.s.n[1], Nz = x.s.n[2], md = x.c.modes, W = x.c.width;
  float2* t2 = at<float2>(x, x.wl.t2);
  float2* t1 = at<float2>(x, x.wl.t1);
  BDDA_TRY_F((transform<true, 0>(x, S, t2, x.tab[3], (int64_t)B, md, Nx, (int64_t)md * md * W, 1.f)));
  BDDA_TRY_F((transform<true, 0>(x, t2, t1, x.tab[4], (int64_t)B * Nx, md, Ny, (int64_t)md * W, 1.f)));
  if (add) return transform<true, 2>(x, t1, out, x.tab[5], (int64_t)B * Nx * Ny, md, Nz, W, scale);
  return transform<true, 1>(x, t1, out, x.tab[5], (int64_t)B * Nx * Ny, md, Nz, W, scale);
}

// Layers whose sides are multiples of 8 (16 for the input side of the weight
// gradient) run on the tensor cores; the lift (13 inputs) and the last
// projection (6 outputs) keep the FP32 kernels.
template <int CI, int CO>
constexpr bool tc_shape() { return CI % 16 == 0 && CO % 8 == 0 && CI <= 64 && CO <= 64; }

template <int CI, int CO>
int pw_fwd(Ctx& x, const float* in, const float* Wt, const float* b, const float* add, float* z, float* y, int act) {
  if constexpr (tc_shape<CI, CO>()) {
    const int64_t tiles = (x.s.M + 15) / 16;
    pointwise_fwd_tc_kernel<CI, CO><<<(int)std::min<int64_t>(148 * 8, (tiles + 7) / 8), 256, 0, x.st>>>(
        in, Wt, b, add, z, y, x.s.M, act);
  } else {
    pointwise_fwd_kernel<CI, CO><<<grid_for(x.s.M), 256, 0, x.st>>>(in, Wt, b, add, z, y, x.s.M, act);
  }
  count_launch();
  BDDA_CUDA_TRY(cudaGetLastError());
  return BDDA_OK;
}
template <int CI, int CO>
int pw_bwd(Ctx& x, const float* gy, const float* z, const float* in, const float* Wt, float* gz, float* gx,
           float* gWt, float* gb, int act, int accumulate) {
  const int wgrid = (int)std::min<int64_t>(148 * 4, (x.s.M + 255) / 256 + 1);
  if constexpr (tc_shape<CI, CO>()) {
    const int64_t tiles = (x.s.M + 15) / 16;
    pointwise_bwd_data_tc_kernel<CI, CO><<<(int)std::min<int64_t>(148 * 16, (tiles + 3) / 4), 128, 0, x.st>>>(
        gy, z, Wt, gz, gx, x.s.M, act, accumulate);
    pointwise_bwd_weight_tc_kernel<CI, CO><<<wgrid, 128, 0, x.st>>>(in, gz, gWt, gb, x.s.M);
  } else {
    pointwise_bwd_data_kernel<CI, CO><<<grid_for(x.s.M), 256, 0, x.st>>>(gy, z, Wt, gz, gx, x.s.M, act,
                                                                         accumulate);
    pointwise_bwd_weight_kernel<CI, CO><<<wgrid, 256, 0, x.st>>>(in, gz, gWt, gb, x.s.M);
  }
  count_launch(2);
  BDDA_CUDA_TRY(cudaGetLastError());
  return BDDA_OK;
}

// Fixed shapes of the shipped network (cin 13, width 32, cout 6, proj 64).
constexpr int kCin = 13, kW = 32, kCout = 6, kProj = 64;

bool shipped(const FnoCfg& c) { return c.cin == kCin && c.width == kW && c.cout == kCout && c.proj == kProj; }

int forward(Ctx& x, bool train) {
  const FnoCfg& c = x.c;
  const float* P = x.prm;
  float* v0 = at<float>(x, x.wl.v[0]);
  BDDA_TRY_F((pw_fwd<kCin, kW>(x, at<float>(x, x.wl.x), P + x.pl.P, P + x.pl.p, nullptr, nullptr, v0, 0)));
  const float inv = 1.f / (float)x.s.ncell;
  for (int l = 0; l < c.layers; ++l) {
    float* vl = at<float>(x, x.wl.v[l]);
    float* vn = at<float>(x, x.wl.v[l + 1]);
    float2* A = at<float2>(x, x.wl.A[train ? l : 0]);
    float2* S = at<float2>(x, x.wl.S);
    BDDA_TRY_F(dft_fwd(x, vl, A, 1.f));
    spec_mix_kernel<<<grid_for((int64_t)x.s.B * x.s.K * kW), 256, 0, x.st>>>(
        A, reinterpret_cast<const float2*>(P + x.pl.R[l]), S, x.s.B, x.s.K, kW);
    count_launch();
    float* sg = at<float>(x, x.wl.gs);   // spectral branch in grid space
    BDDA_TRY_F(dft_inv(x, S, sg, inv, false));
    const int act = l + 1 < c.layers ? 1 : 0;
    BDDA_TRY_F((pw_fwd<kW, kW>(x, vl, P + x.pl.W[l], P + x.pl.b[l], sg, train ? at<float>(x, x.wl.z[l]) : nullptr,
                               vn, act)));
  }
  float* vL = at<float>(x, x.wl.v[c.layers]);
  BDDA_TRY_F((pw_fwd<kW, kProj>(x, vL, P + x.pl.Q1, P + x.pl.q1, nullptr, at<float>(x, x.wl.zq), at<float>(x, x.wl.h),
                                1)));
  return pw_fwd<kProj, kCout>(x, at<float>(x, x.wl.h), P + x.pl.Q2, P + x.pl.q2, nullptr, nullptr,
                              at<float>(x, x.wl.y), 0);
}

// gradient of the loss w.r.t. every parameter, given gy in wl.gz-sized buffer `gy`
int backward(Ctx& x, const float* gy) {
  const FnoCfg& c = x.c;
  const float* P = x.prm;
  float* G = x.grad;
  float* gz = at<float>(x, x.wl.gz);
  float* gh = at<float>(x, x.wl.gh);
  float* gv = at<float>(x, x.wl.gv);
  float* gv2 = at<float>(x, x.wl.gv2);
  const float inv = 1.f / (float)x.s.ncell;
  // y = Q2 h + q2
  BDDA_TRY_F((pw_bwd<kProj, kCout>(x, gy, nullptr, at<float>(x, x.wl.h), P + x.pl.Q2, gz, gh, G + x.pl.Q2, G + x.pl.q2,
                                   0, 0)));
  // h = gelu(Q1 v + q1)
  BDDA_TRY_F((pw_bwd<kW, kProj>(x, gh, at<float>(x, x.wl.zq), at<float>(x, x.wl.v[c.layers]), P + x.pl.Q1, gz, gv,
                                G + x.pl.Q1, G + x.pl.q1, 1, 0)));
  for (int l = c.layers - 1; l >= 0; --l) {
    const int act = l + 1 < c.layers ? 1 : 0;
    float* vl = at<float>(x, x.wl.v[l]);
    // pointwise branch: gz = gv act'(z); gv2 = W^T gz
    float* gzl = at<float>(x, x.wl.gs);
    BDDA_TRY_F((pw_bwd<kW, kW>(x, gv, at<float>(x, x.wl.z[l]), vl, P + x.pl.W[l], gzl, gv2, G + x.pl.W[l],
                               G + x.pl.b[l], act, 0)));
    // spectral branch: s = inv Re IDFT(S): gS = inv DFT(gz); gA = R^H gS; gR += conj(A) gS; gv2 += Re IDFT(gA)
    float2* gS = at<float2>(x, x.wl.gS);
    float2* gA = at<float2>(x, x.wl.gA);
    BDDA_TRY_F(dft_fwd(x, gzl, gS, inv));
    spec_mix_bwd_data_kernel<<<grid_for((int64_t)x.s.B * x.s.K * kW), 256, 0, x.st>>>(
        gS, reinterpret_cast<const float2*>(P + x.pl.R[l]), gA, x.s.B, x.s.K, kW);
    spec_mix_bwd_weight_kernel<<<grid_for((int64_t)x.s.K * kW * kW), 256, 0, x.st>>>(
        at<float2>(x, x.wl.A[l]), gS, reinterpret_cast<float2*>(G + x.pl.R[l]), x.s.B, x.s.K, kW);
    count_launch(2);
    BDDA_CUDA_TRY(cudaGetLastError());
    BDDA_TRY_F(dft_inv(x, gA, gv2, 1.f, true));
    std::swap(gv, gv2);
  }
  // v0 = P x + p (x has no gradient)
  return pw_bwd<kCin, kW>(x, gv, nullptr, at<float>(x, x.wl.x), P + x.pl.P, gz, nullptr, G + x.pl.P, G + x.pl.p, 0, 0);
}

// tables: write the axis DFT tables into the workspace (bdda_fno_features
// does; the other entry points use the tables it left there)
int make_ctx(Ctx& x, const bdda_fno_config* cfg, int B, const int n[3], void* work, size_t work_bytes,
             const float* params, float* grads, cudaStream_t st, bool tables = false) {
  if (!cfg_ok(cfg) || B < 1 || !n) return BDDA_BAD_ARG;
  x.c = to_cfg(cfg);
  if (!shipped(x.c)) return BDDA_BAD_ARG;
  x.pl = param_layout(x.c);
  x.s.B = B;
  for (int a = 0; a < 3; ++a) {
    if (n[a] < x.c.modes || n[a] > kMaxAxis) return BDDA_BAD_ARG;
    x.s.n[a] = n[a];
  }
  x.s.ncell = (int64_t)n[0] * n[1] * n[2];
  x.s.M = x.s.ncell * B;
  x.s.K = x.c.modes * x.c.modes * x.c.modes;
  x.wl = work_layout(x.c, x.s);
  if (!work || work_bytes < x.wl.total) return BDDA_NO_WORKSPACE;
  x.w = static_cast<unsigned char*>(work);
  x.prm = params;
  x.grad = grads;
  x.st = st;
  float2* base = at<float2>(x, x.wl.tabs);
  for (int t = 0; t < 6; ++t) x.tab[t] = base + (size_t)t * kMaxAxis * 32;
  return tables ? upload_tables(x) : BDDA_OK;
}

}  // namespace
}  // namespace bdda

using namespace bdda;

extern "C" {

size_t bdda_fno_param_count(const bdda_fno_config* cfg) {
  if (!cfg_ok(cfg)) return 0;
  return param_layout(to_cfg(cfg)).total;
}

size_t bdda_fno_workspace_bytes(const bdda_fno_config* cfg, int B, const int n[3]) {
  if (!cfg_ok(cfg) || B < 1 || !n) return 0;
  Shape s;
  s.B = B;
  for (int a = 0; a < 3; ++a) s.n[a] = n[a];
  s.ncell = (int64_t)n[0] * n[1] * n[2];
  s.M = s.ncell * B;
  s.K = cfg->modes * cfg->modes * cfg->modes;
  return work_layout(to_cfg(cfg), s).total;
}

int bdda_fno_features(const bdda_fno_config* cfg, const int n[3], int n_occ, int L, const int32_t* cell_map,
                      const void* diag, const void* B, const double chi[6], double* scale, void* work,
                      size_t work_bytes, void* stream) {
  if (!cfg_ok(cfg) || !n || n_occ < 1 || L < 1 || !cell_map || !diag || !B || !chi || !scale) return BDDA_BAD_ARG;
  Ctx x;
  const int s = make_ctx(x, cfg, L, n, work, work_bytes, nullptr, nullptr, static_cast<cudaStream_t>(stream), true);
  if (s != BDDA_OK) return s;
  double* tmp = at<double>(x, x.wl.chi);
  BDDA_CUDA_TRY(cudaMemcpyAsync(tmp, chi, 6 * sizeof(double), cudaMemcpyHostToDevice, x.st));
  jacobi_scale_kernel<<<L, 256, 0, x.st>>>(static_cast<const double2*>(diag), static_cast<const double2*>(B),
                                           3 * (int64_t)n_occ, L, scale);
  features_kernel<<<grid_for(x.s.M), 256, 0, x.st>>>(cell_map, x.s.ncell, n_occ, L, static_cast<const double2*>(diag),
                                                     static_cast<const double2*>(B), tmp, scale, at<float>(x, x.wl.x),
                                                     x.c.cin);
  mask_kernel<<<grid_for(x.s.ncell), 256, 0, x.st>>>(cell_map, x.s.ncell, at<float>(x, x.wl.mask));
  count_launch(3);
  BDDA_CUDA_TRY(cudaGetLastError());
  return BDDA_OK;
}

int bdda_fno_forward(const bdda_fno_config* cfg, int B, const int n[3], const float* params, int train, void* work,
                     size_t work_bytes, void* stream) {
  Ctx x;
  const int s = make_ctx(x, cfg, B, n, work, work_bytes, params, nullptr, static_cast<cudaStream_t>(stream));
  if (s != BDDA_OK) return s;
  if (!params) return BDDA_BAD_ARG;
  return forward(x, train != 0);
}

int bdda_fno_loss(const bdda_fno_config* cfg, int B, const int n[3], int n_occ, const int32_t* cell_map,
                  const void* diag, const void* Bm, const void* X, const double* scale, double* loss, void* work,
                  size_t work_bytes, void* stream) {
  Ctx x;
  const int s = make_ctx(x, cfg, B, n, work, work_bytes, nullptr, nullptr, static_cast<cudaStream_t>(stream));
  if (s != BDDA_OK) return s;
  if (!cell_map || !diag || !Bm || !X || !scale || !loss) return BDDA_BAD_ARG;
  float* tgt = at<float>(x, x.wl.tgt);
  double* den = at<double>(x, x.wl.den);
  double* dl = at<double>(x, x.wl.loss);
  target_kernel<<<grid_for(x.s.M), 256, 0, x.st>>>(cell_map, x.s.ncell, n_occ, B, static_cast<const double2*>(diag),
                                                   static_cast<const double2*>(Bm), static_cast<const double2*>(X),
                                                   scale, tgt);
  BDDA_CUDA_TRY(cudaMemsetAsync(den, 0, (size_t)B * sizeof(double), x.st));
  BDDA_CUDA_TRY(cudaMemsetAsync(dl, 0, sizeof(double), x.st));
  loss_den_kernel<<<dim3(grid_for(x.s.ncell * kCout) / 4 + 1, B), 256, 0, x.st>>>(tgt, at<float>(x, x.wl.mask),
                                                                                 x.s.ncell, kCout, den);
  loss_kernel<<<grid_for(x.s.M * kCout), 256, 0, x.st>>>(at<float>(x, x.wl.y), tgt, at<float>(x, x.wl.mask),
                                                         x.s.ncell, kCout, B, den, at<float>(x, x.wl.gy), dl);
  count_launch(3);
  BDDA_CUDA_TRY(cudaGetLastError());
  BDDA_CUDA_TRY(cudaMemcpyAsync(loss, dl, sizeof(double), cudaMemcpyDeviceToHost, x.st));
  return BDDA_OK;
}

int bdda_fno_backward(const bdda_fno_config* cfg, int B, const int n[3], const float* params, const float* grad_out,
                      float* grads, void* work, size_t work_bytes, void* stream) {
  Ctx x;
  const int s = make_ctx(x, cfg, B, n, work, work_bytes, params, grads, static_cast<cudaStream_t>(stream));
  if (s != BDDA_OK) return s;
  if (!params || !grads) return BDDA_BAD_ARG;
  const float* gy = grad_out ? grad_out : at<float>(x, x.wl.gy);
  return backward(x, gy);
}

int bdda_fno_adam(float* params, const float* grads, float* m, float* v, size_t n, float lr, float beta1, float beta2,
                  float eps, float weight_decay, int step, void* stream) {
  if (!params || !grads || !m || !v || n == 0 || step < 1) return BDDA_BAD_ARG;
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  adam_kernel<<<grid_for((int64_t)n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      params, grads, m, v, (int64_t)n, lr, beta1, beta2, eps, c1, c2, weight_decay);
  count_launch();
  BDDA_CUDA_TRY(cudaGetLastError());
  return BDDA_OK;
}

int bdda_fno_warm_start(const bdda_fno_config* cfg, const int n[3], int n_occ, int L, const int32_t* cell_map,
                        const void* diag, const void* B, const double* scale, void* X0, void* work,
                        size_t work_bytes, void* stream) {
  Ctx x;
  const int s = make_ctx(x, cfg, L, n, work, work_bytes, nullptr, nullptr, static_cast<cudaStream_t>(stream));
  if (s != BDDA_OK) return s;
  if (!cell_map || !diag || !B || !scale || !X0) return BDDA_BAD_ARG;
  warm_start_kernel<<<grid_for(x.s.M), 256, 0, x.st>>>(cell_map, x.s.ncell, n_occ, L, static_cast<const double2*>(diag),
                                                       static_cast<const double2*>(B), scale, at<float>(x, x.wl.y),
                                                       kCout, static_cast<double2*>(X0));
  count_launch();
  BDDA_CUDA_TRY(cudaGetLastError());
  return BDDA_OK;
}

size_t bdda_fno_buffer_offset(const bdda_fno_config* cfg, int B, const int n[3], int which) {
  if (!cfg_ok(cfg) || B < 1 || !n) return (size_t)-1;
  Shape s;
  s.B = B;
  for (int a = 0; a < 3; ++a) s.n[a] = n[a];
  s.ncell = (int64_t)n[0] * n[1] * n[2];
  s.M = s.ncell * B;
  s.K = cfg->modes * cfg->modes * cfg->modes;
  const FnoWork w = work_layout(to_cfg(cfg), s);
  switch (which) {
    case 0: return w.x;
    case 1: return w.y;
    case 2: return w.mask;
    case 3: return w.gy;
    case 4: return w.tgt;
    default: return (size_t)-1;
  }
}

size_t bdda_fno_offset(const bdda_fno_config* cfg, int what, int layer) {
  if (!cfg_ok(cfg)) return (size_t)-1;
  const FnoParams p = param_layout(to_cfg(cfg));
  if (layer < 0 || layer >= cfg->layers) layer = 0;
  switch (what) {
    case 0: return p.P;
    case 1: return p.p;
    case 2: return p.R[layer];
    case 3: return p.W[layer];
    case 4: return p.b[layer];
    case 5: return p.Q1;
    case 6: return p.q1;
    case 7: return p.Q2;
    case 8: return p.q2;
    default: return (size_t)-1;
  }
}

}  // extern "C"
