// DDA physics around the solve: polarizability / diagonal, incident field
// right-hand side, and the per-orientation observables.
//
// References (bl_dda/scatterer.py): polarizability and diag_A :137-148, RHS
// :153-161, E = 4 pi P / ((eps_r - 1) v) :182-184, C_abs :187-193, C_ext
// :196-199, S_fw (PCAS) :202-213, S_bk (OCBS) :216-227.
#include <cmath>

#include "bdda_blas.cuh"
#include "bdda_internal.h"
#include "bdda_small.cuh"

namespace bdda {

__device__ __forceinline__ double2 cexpi(double t) {
  double s, c;
  sincos(t, &s, &c);
  return make_double2(c, s);
}

// eps_r = m_p^2 / m_m^2 per axis; CM polarizability with the CR2009 radiative
// correction; diag_A = 1 / alpha, ordered [x0 y0 z0 x1 ...]
__global__ void polarizability_kernel(int n_occ, double2 mx, double2 my, double2 mz, double m_m, double lf,
                                      double k, double2* diag, double2* eper_r) {
  const double vol = lf * lf * lf;
  const double a = cbrt(3.0 * vol / (4.0 * M_PI));
  // M = (8 pi / 3) ((1 - i k a) e^{i k a} - 1)
  const double2 e = cexpi(k * a);
  const double2 t = zmul(make_double2(1.0, -k * a), e);
  const double2 Mterm = make_double2((8.0 * M_PI / 3.0) * (t.x - 1.0), (8.0 * M_PI / 3.0) * t.y);
  const double2 mp[3] = {mx, my, mz};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * (int64_t)n_occ;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 m = mp[i % 3];
    const double2 m2 = zmul(m, m);
    const double2 er = make_double2(m2.x / (m_m * m_m), m2.y / (m_m * m_m));
    const double2 cm0 = zdiv(make_double2(er.x - 1.0, er.y), make_double2(er.x + 2.0, er.y));
    const double2 cm = make_double2((3.0 / (4.0 * M_PI)) * cm0.x * vol, (3.0 / (4.0 * M_PI)) * cm0.y * vol);
    const double2 mc = zmul(Mterm, cm);
    const double2 den = make_double2(1.0 - mc.x / vol, -mc.y / vol);
    const double2 alpha = zdiv(cm, den);
    diag[i] = zdiv(make_double2(1.0, 0.0), alpha);
    if (eper_r) eper_r[i] = er;
  }
}

// B[3n + c, l] = e0[l, c] exp(i k u_l . r_n)
__global__ void rhs_kernel(int n_occ, int L, double k, const double* pos, const double* u_inc,
                           const double2* e0, double2* B) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)n_occ * L;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = i / L;
    const int l = (int)(i - n * L);
    const double d = u_inc[3 * l] * pos[3 * n] + u_inc[3 * l + 1] * pos[3 * n + 1] + u_inc[3 * l + 2] * pos[3 * n + 2];
    const double2 ph = cexpi(k * d);
    for (int c = 0; c < 3; ++c) B[(3 * n + c) * L + l] = zmul(e0[3 * l + c], ph);
  }
}

struct ObsArgs {
  int n_occ, L;
  double k, vol;
  int absorbing;            // mean Im eps_r >= 1e-12
  const double* pos;        // N x 3
  const double2* eper_r;    // 3N
  const double2* X;         // 3N x L
  const double* vec;        // L x 7 x 3: u_inc, u_fw, theta_fw, phi_fw, u_bk, theta_bk, phi_bk
  const double2* e0;        // L x 3
  double* partial;          // [nblk][L][10]
};

// per-orientation sums over dipoles; one CTA row-chunk x all L orientations
__global__ void observables_kernel(ObsArgs a) {
  const int L = a.L;
  const int64_t chunk = ((int64_t)a.n_occ + gridDim.x - 1) / gridDim.x;
  const int64_t n0 = blockIdx.x * chunk, n1 = min((int64_t)a.n_occ, n0 + chunk);
  const double r2 = 1.4142135623730950488;
  for (int l = 0; l < L; ++l) {
    const double* v = a.vec + (size_t)l * 21;
    double acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t n = n0 + threadIdx.x; n < n1; n += blockDim.x) {
      const double* r = a.pos + 3 * n;
      double2 P[3];
      for (int c = 0; c < 3; ++c) P[c] = a.X[(3 * n + c) * L + l];
      // C_abs: Im(P conj(E)), E = 4 pi P / ((eps_r - 1) v)
      if (a.absorbing) {
        for (int c = 0; c < 3; ++c) {
          const double2 er = a.eper_r[3 * n + c];
          const double2 E = zdiv(make_double2(4.0 * M_PI * P[c].x, 4.0 * M_PI * P[c].y),
                                 make_double2((er.x - 1.0) * a.vol, er.y * a.vol));
          acc[0] += P[c].y * E.x - P[c].x * E.y;
        }
      }
      // C_ext: Im(P conj(E_inc))
      const double2 ph = cexpi(a.k * (v[0] * r[0] + v[1] * r[1] + v[2] * r[2]));
      for (int c = 0; c < 3; ++c) {
        const double2 Ei = zmul(a.e0[3 * l + c], ph);
        acc[1] += P[c].y * Ei.x - P[c].x * Ei.y;
      }
      // scattering amplitudes: sum (P . e) conj(sqrt2 e_dir) and conj(sqrt2 i e_dir)
      for (int d = 0; d < 2; ++d) {
        const double* u = v + 3 + 9 * d;
        const double* th = u + 3;
        const double* ph2 = u + 6;
        const double2 e = cexpi(a.k * (u[0] * r[0] + u[1] * r[1] + u[2] * r[2]));
        double2 pt = make_double2(0, 0), pp = make_double2(0, 0);
        for (int c = 0; c < 3; ++c) {
          pt = make_double2(pt.x + P[c].x * th[c], pt.y + P[c].y * th[c]);
          pp = make_double2(pp.x + P[c].x * ph2[c], pp.y + P[c].y * ph2[c]);
        }
        const double2 ce = make_double2(r2 * e.x, -r2 * e.y);     // conj(sqrt2 e)
        const double2 ci = make_double2(-r2 * e.y, -r2 * e.x);    // conj(sqrt2 i e) = -sqrt2 (s + i c)
        const double2 st = zmul(pt, ce), sp = zmul(pp, ci);
        acc[2 + 4 * d] += st.x; acc[3 + 4 * d] += st.y;
        acc[4 + 4 * d] += sp.x; acc[5 + 4 * d] += sp.y;
      }
    }
    for (int q = 0; q < 10; ++q) {
      const double s = block_sum(acc[q]);
      if (threadIdx.x == 0) a.partial[((size_t)blockIdx.x * L + l) * 10 + q] = s;
    }
  }
}

// totals over CTAs -> C_abs, C_ext, S_fw_theta, S_fw_phi, S_bk_theta, S_bk_phi, S_bk
__global__ void observables_finalize_kernel(const double* partial, int nblk, int L, double k, int absorbing,
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

}  // namespace bdda

using namespace bdda;

constexpr int kObsBlocks = 148;

extern "C" {

int bdda_polarizability(int n_occ, const double m_p_xyz[6], double m_m, double lf, double k, void* diag,
                        void* eper_r, void* stream) {
  if (n_occ < 1 || !m_p_xyz || !diag || !(lf > 0.0) || !(m_m > 0.0)) return BDDA_BAD_ARG;
  polarizability_kernel<<<kRedBlocks, 256, 0, (cudaStream_t)stream>>>(
      n_occ, make_double2(m_p_xyz[0], m_p_xyz[1]), make_double2(m_p_xyz[2], m_p_xyz[3]),
      make_double2(m_p_xyz[4], m_p_xyz[5]), m_m, lf, k, static_cast<double2*>(diag),
      static_cast<double2*>(eper_r));
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BDDA_OK;
}

int bdda_incident_rhs(int n_occ, int L, double k, const double* pos, const double* u_inc, const void* e0,
                      void* B, void* stream) {
  if (n_occ < 1 || L < 1 || !pos || !u_inc || !e0 || !B) return BDDA_BAD_ARG;
  rhs_kernel<<<kRedBlocks, 256, 0, (cudaStream_t)stream>>>(n_occ, L, k, pos, u_inc,
                                                           static_cast<const double2*>(e0),
                                                           static_cast<double2*>(B));
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BDDA_OK;
}

size_t bdda_observables_workspace_bytes(int L) {
  return L < 1 ? 0 : (size_t)kObsBlocks * L * 10 * sizeof(double);
}

int bdda_observables(int n_occ, int L, double k, double lf, int absorbing, const double* pos,
                     const void* eper_r, const void* X, const double* vec, const void* e0, double* out,
                     void* work, void* stream) {
  if (n_occ < 1 || L < 1 || !pos || !eper_r || !X || !vec || !e0 || !out) return BDDA_BAD_ARG;
  if (!work) return BDDA_NO_WORKSPACE;
  ObsArgs a;
  a.n_occ = n_occ; a.L = L; a.k = k; a.vol = lf * lf * lf; a.absorbing = absorbing;
  a.pos = pos; a.eper_r = static_cast<const double2*>(eper_r); a.X = static_cast<const double2*>(X);
  a.vec = vec; a.e0 = static_cast<const double2*>(e0); a.partial = static_cast<double*>(work);
  observables_kernel<<<kObsBlocks, 256, 0, (cudaStream_t)stream>>>(a);
  BDDA_CUDA_TRY(cudaGetLastError());
  observables_finalize_kernel<<<(L + 63) / 64, 64, 0, (cudaStream_t)stream>>>(
      static_cast<double*>(work), kObsBlocks, L, k, absorbing, out);
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch(2);
  return BDDA_OK;
}

}  // extern "C"
