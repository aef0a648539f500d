// DDA physics around the solve: polarizability / diagonal, incident field
// right-hand side, and the per-orientation observables.
//
// References (bl_dda/scatterer.py): polarizability and diag_A :137-148, RHS
// :153-161, E = 4 pi P / ((eps_r - 1) v) :182-184, C_abs :187-193, C_ext
// :196-199, S_fw (PCAS) :202-213, S_bk (OCBS) :216-227.
#include "bdda_dda.cuh"

namespace bdda {

// diag_A = 1 / alpha per row, ordered [x0 y0 z0 x1 ...], and eps_r
__global__ void polarizability_kernel(int n_occ, double2 mx, double2 my, double2 mz, double m_m, double lf,
                                      double k, double2* diag, double2* eper_r) {
  const double2 mp[3] = {mx, my, mz};
  double2 d[3], er[3];
  for (int c = 0; c < 3; ++c) d[c] = cr_diag(mp[c], m_m, lf, k, &er[c]);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * (int64_t)n_occ;
       i += (int64_t)gridDim.x * blockDim.x) {
    diag[i] = d[i % 3];
    if (eper_r) eper_r[i] = er[i % 3];
  }
}

// B[3n + c, l] = e0[l, c] exp(i k u_l . r_n)
__global__ void rhs_kernel(int n_occ, int L, double k, const double* pos, const double* u_inc,
                           const double2* e0, double2* B) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)n_occ * L;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = i / L;
    const int l = (int)(i - n * L);
    const double2 ph = incident_phase(k, u_inc + 3 * l, pos + 3 * n);
    for (int c = 0; c < 3; ++c) B[(3 * n + c) * L + l] = zmul(e0[3 * l + c], ph);
  }
}

}  // namespace bdda

using namespace bdda;

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
  return L < 1 ? 0 : (size_t)kDdaObsBlocks * L * 10 * sizeof(double);
}

int bdda_observables(int n_occ, int L, double k, double lf, int absorbing, const double* pos,
                     const void* eper_r, const void* X, const double* vec, const void* e0, double* out,
                     void* work, void* stream) {
  if (n_occ < 1 || L < 1 || !pos || !eper_r || !X || !vec || !e0 || !out) return BDDA_BAD_ARG;
  if (!work) return BDDA_NO_WORKSPACE;
  DdaPhys a;
  memset(&a, 0, sizeof(a));
  a.n_occ = n_occ; a.L = L; a.k = k; a.lf = lf; a.absorbing = absorbing;
  a.pos = pos; a.vec = vec; a.e0 = static_cast<const double2*>(e0); a.obs = out;
  a.partial = static_cast<double*>(work);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  dda_epilogue_kernel<double2><<<kDdaObsBlocks, dda_epilogue_threads(L), dda_epilogue_smem(L), st>>>(
      a, static_cast<const double2*>(X), nullptr, static_cast<const double2*>(eper_r));
  BDDA_CUDA_TRY(cudaGetLastError());
  observables_finalize_kernel<<<(L + 63) / 64, 64, 0, st>>>(a.partial, kDdaObsBlocks, L, k, absorbing, out);
  BDDA_CUDA_TRY(cudaGetLastError());
  count_launch(2);
  return BDDA_OK;
}

}  // extern "C"
