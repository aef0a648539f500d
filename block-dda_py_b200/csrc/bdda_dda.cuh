// The physics around one DDA solve, as device code shared by the separate
// entry points (bdda_polarizability, bdda_incident_rhs, bdda_observables)
// and by the fused one (bdda_dda_solve), whose prologue forms the Jacobi-
// scaled right-hand side directly and whose epilogue accumulates the
// observables in the pass that writes X.
//
// References (bl_dda/scatterer.py): polarizability and diag_A :137-148, RHS
// :153-161, E = 4 pi P / ((eps_r - 1) v) :182-184, C_abs :187-193, C_ext
// :196-199, S_fw (PCAS) :202-213, S_bk (OCBS) :216-227.
#pragma once
#include <cmath>
#include <cstring>

#include "bdda_blas.cuh"
#include "bdda_internal.h"
#include "bdda_small.cuh"

namespace bdda {

__device__ __forceinline__ double2 cexpi(double t) {
  double s, c;
  sincos(t, &s, &c);
  return make_double2(c, s);
}

// eps_r = m_p^2 / m_m^2; Clausius-Mossotti polarizability with the CR2009
// radiative correction M = (8 pi / 3) ((1 - i k a) e^{i k a} - 1),
// a = (3 v / 4 pi)^(1/3); returns diag_A = 1 / alpha (scatterer.py:137-148)
__device__ __forceinline__ double2 cr_diag(double2 m, double m_m, double lf, double k, double2* eper_r) {
  const double vol = lf * lf * lf;
  const double a = cbrt(3.0 * vol / (4.0 * M_PI));
  const double2 e = cexpi(k * a);
  const double2 t = zmul(make_double2(1.0, -k * a), e);
  const double2 Mterm = make_double2((8.0 * M_PI / 3.0) * (t.x - 1.0), (8.0 * M_PI / 3.0) * t.y);
  const double2 m2 = zmul(m, m);
  const double2 er = make_double2(m2.x / (m_m * m_m), m2.y / (m_m * m_m));
  const double2 cm0 = zdiv(make_double2(er.x - 1.0, er.y), make_double2(er.x + 2.0, er.y));
  const double2 cm = make_double2((3.0 / (4.0 * M_PI)) * cm0.x * vol, (3.0 / (4.0 * M_PI)) * cm0.y * vol);
  const double2 mc = zmul(Mterm, cm);
  const double2 den = make_double2(1.0 - mc.x / vol, -mc.y / vol);
  const double2 alpha = zdiv(cm, den);
  *eper_r = er;
  return zdiv(make_double2(1.0, 0.0), alpha);
}

// phase of the incident plane wave of orientation l at dipole n: exp(i k u_l . r_n)
__device__ __forceinline__ double2 incident_phase(double k, const double* u, const double* r) {
  const double d = u[0] * r[0] + u[1] * r[1] + u[2] * r[2];
  return cexpi(k * d);
}

// Inputs of one DDA problem for the fused entry point.
struct DdaPhys {
  int n_occ, L;
  double2 mp[3];            // m_p per axis
  double m_m, lf, k;
  const double* pos;        // (N, 3)
  const double* vec;        // (L, 21): u_inc, u_fw, theta_fw, phi_fw, u_bk, theta_bk, phi_bk
  const double2* e0;        // (L, 3)
  int absorbing;            // mean Im eps_r >= 1e-12 (scatterer.py:189)
  double2* diag_out;        // nullable: diag_A (3N), as bdda_polarizability writes it
  double2* eper_out;        // nullable: eps_r (3N)
  double* obs;              // (L, 12) observables
  double* partial;          // kDdaObsBlocks x L x 10 partial sums
};

constexpr int kDdaObsBlocks = 296;

// Prologue: diag, jpre (and the complex64 copies) per row and
// Bj = jpre * e0 exp(i k u . r) for every (row, orientation); B itself is
// never stored.  Same operations, in the same order, as the polarizability,
// RHS and prepare kernels of the unfused path.
template <typename T, bool C64_COPY>
__global__ void dda_prologue_kernel(DdaPhys p, T* diagT, T* jpreT, T* Bj, float2* diag32, float2* jpre32) {
  double2 d[3], j[3], er[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    d[c] = cr_diag(p.mp[c], p.m_m, p.lf, p.k, &er[c]);
    j[c] = zdiv(make_double2(1.0, 0.0), d[c]);
  }
  const int L = p.L;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)p.n_occ * L;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = i / L;
    const int l = (int)(i - n * L);
    const double2 ph = incident_phase(p.k, p.vec + (size_t)l * 21, p.pos + 3 * n);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double2 B = zmul(p.e0[3 * l + c], ph);
      Bj[(3 * n + c) * L + l] = from_d2<T>(zmul(B, j[c]));
    }
    if (l == 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int64_t r = 3 * n + c;
        diagT[r] = from_d2<T>(d[c]);
        jpreT[r] = from_d2<T>(j[c]);
        if constexpr (C64_COPY) {
          diag32[r] = from_d2<float2>(d[c]);
          jpre32[r] = from_d2<float2>(j[c]);
        }
        if (p.diag_out) p.diag_out[r] = d[c];
        if (p.eper_out) p.eper_out[r] = er[c];
      }
    }
  }
}

// Ten per-orientation sums of dipole n (C_abs, C_ext, S_fw theta/phi re/im,
// S_bk theta/phi re/im) for polarizations P[3] of orientation l.
__device__ __forceinline__ void dipole_observables(const DdaPhys& p, int64_t n, int l, const double2* P,
                                                   const double2* eper_r_row, double* acc) {
  const double r2 = 1.4142135623730950488;
  const double* v = p.vec + (size_t)l * 21;
  const double* r = p.pos + 3 * n;
  const double vol = p.lf * p.lf * p.lf;
  if (p.absorbing) {   // C_abs: Im(P conj(E)), E = 4 pi P / ((eps_r - 1) v)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double2 er = eper_r_row[c];
      const double2 E = zdiv(make_double2(4.0 * M_PI * P[c].x, 4.0 * M_PI * P[c].y),
                             make_double2((er.x - 1.0) * vol, er.y * vol));
      acc[0] += P[c].y * E.x - P[c].x * E.y;
    }
  }
  const double2 ph = cexpi(p.k * (v[0] * r[0] + v[1] * r[1] + v[2] * r[2]));   // C_ext: Im(P conj(E_inc))
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double2 Ei = zmul(p.e0[3 * l + c], ph);
    acc[1] += P[c].y * Ei.x - P[c].x * Ei.y;
  }
#pragma unroll
  for (int dd = 0; dd < 2; ++dd) {   // sum (P . e) conj(sqrt2 e_dir) and conj(sqrt2 i e_dir)
    const double* u = v + 3 + 9 * dd;
    const double* th = u + 3;
    const double* phv = u + 6;
    const double2 e = cexpi(p.k * (u[0] * r[0] + u[1] * r[1] + u[2] * r[2]));
    double2 pt = make_double2(0, 0), pp = make_double2(0, 0);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      pt = make_double2(pt.x + P[c].x * th[c], pt.y + P[c].y * th[c]);
      pp = make_double2(pp.x + P[c].x * phv[c], pp.y + P[c].y * phv[c]);
    }
    const double2 ce = make_double2(r2 * e.x, -r2 * e.y);     // conj(sqrt2 e)
    const double2 ci = make_double2(-r2 * e.y, -r2 * e.x);    // conj(sqrt2 i e)
    const double2 st = zmul(pt, ce), sp = zmul(pp, ci);
    acc[2 + 4 * dd] += st.x; acc[3 + 4 * dd] += st.y;
    acc[4 + 4 * dd] += sp.x; acc[5 + 4 * dd] += sp.y;
  }
}

// Epilogue: Xout = X (widened to complex128) and, in the same pass over X,
// the observables' partial sums of this CTA's dipoles.  Thread t handles
// orientation t % L of dipoles n0 + t / L + k R (R = blockDim / L rows of
// threads), then the R row sums of each orientation are added in a fixed
// order, so the result does not depend on scheduling.
template <typename T>
__global__ void dda_epilogue_kernel(DdaPhys p, const T* X, double2* Xout, const double2* eper_r) {
  extern __shared__ double sacc[];   // [R][L][10]
  const int L = p.L;
  const int R = blockDim.x / L;
  const int t = threadIdx.x;
  const int l = t % L, row = t / L;
  const int64_t chunk = ((int64_t)p.n_occ + gridDim.x - 1) / gridDim.x;
  const int64_t n0 = blockIdx.x * chunk, n1 = min((int64_t)p.n_occ, n0 + chunk);
  double acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  double2 er[3];   // eps_r per axis: from the array, or (null) from m_p as the prologue has it
  if (!eper_r) {
#pragma unroll
    for (int c = 0; c < 3; ++c) cr_diag(p.mp[c], p.m_m, p.lf, p.k, &er[c]);
  }
  if (row < R) {
    for (int64_t n = n0 + row; n < n1; n += R) {
      double2 P[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int64_t idx = (3 * n + c) * L + l;
        P[c] = to_d2(X[idx]);
        if (Xout) Xout[idx] = P[c];
        if (eper_r) er[c] = eper_r[3 * n + c];
      }
      dipole_observables(p, n, l, P, er, acc);
    }
#pragma unroll
    for (int q = 0; q < 10; ++q) sacc[((size_t)row * L + l) * 10 + q] = acc[q];
  }
  __syncthreads();
  for (int e = t; e < L * 10; e += blockDim.x) {
    double s = 0.0;
    for (int r = 0; r < R; ++r) s += sacc[(size_t)r * L * 10 + e];
    p.partial[(size_t)blockIdx.x * L * 10 + e] = s;
  }
}

// totals over CTAs -> C_abs, C_ext, S_fw_theta, S_fw_phi, S_bk_theta, S_bk_phi, S_bk
static __global__ void observables_finalize_kernel(const double* partial, int nblk, int L, double k, int absorbing,
                                            double* out) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= L) return;
  double s[10];
  for (int q = 0; q < 10; ++q) {
    double t = 0.0;
    for (int b = 0; b < nblk; ++b) t += partial[((size_t)b * L + l) * 10 + q];
    s[q] = t;
  }
  const double c4 = 4.0 * M_PI * k, k2 = k * k, r2 = 1.4142135623730950488;
  double* o = out + (size_t)l * 12;
  o[0] = absorbing ? c4 * s[0] : 0.0;
  o[1] = c4 * s[1];
  for (int q = 2; q < 10; ++q) o[q] = k2 * s[q];
  o[10] = (-o[6] + o[8]) / r2;
  o[11] = (-o[7] + o[9]) / r2;
}

// threads of the epilogue kernel for L orientations: a whole number of rows of L
inline int dda_epilogue_threads(int L) { return (256 / L) * L; }
inline size_t dda_epilogue_smem(int L) { return (size_t)(256 / L) * L * 10 * sizeof(double); }

}  // namespace bdda
