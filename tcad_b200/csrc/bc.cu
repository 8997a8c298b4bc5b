// Boundary-condition set-up kernels: contact targets and warm-start stamping.
#include "common.cuh"

namespace tcad {

__global__ void k_set_contacts(const int64_t* __restrict__ nodes, int64_t count,
                               const int32_t* __restrict__ cid, const double* __restrict__ vv,
                               const double* __restrict__ L, const double* __restrict__ n0,
                               const double* __restrict__ p0, double* __restrict__ psi0,
                               double* __restrict__ bn0, double* __restrict__ bp0) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const int64_t k = nodes[t];
  psi0[k] = vv[cid[t]] + L[t];
  bn0[k] = n0[t];
  bp0[k] = p0[t];
}

__global__ void k_stamp_contacts(const tcad_pack_t pk, const int64_t* __restrict__ nodes,
                                 int64_t count, double* __restrict__ psi,
                                 double* __restrict__ nn, double* __restrict__ pp) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const int64_t k = nodes[t];
  psi[k] = pk.bc_psi0[k];
  nn[k] = pk.bc_n0[k];
  pp[k] = pk.bc_p0[k];
}

// Secant predictor along a bias sweep.  For instance i with step ratio
// s = ratio[i] (the new bias step over the previous one, when the two are
// parallel): psi <- psi + s (psi - psi_prev); n <- n (n / n_prev)^s and the
// same for p (extrapolation of log n, log p, i.e. of the quasi-Fermi levels,
// which keeps the densities positive; the factor is held to [1/10, 10], the
// Newton update's own per-step density clip).  The state before the
// prediction is saved into *_prev.  s = 0 only saves the state.
__global__ void __launch_bounds__(kFlatThreads)
k_extrapolate(const tcad_pack_t pk, double* __restrict__ psi, double* __restrict__ nn,
              double* __restrict__ pp, double* __restrict__ psi_prev,
              double* __restrict__ n_prev, double* __restrict__ p_prev,
              const double* __restrict__ ratio) {
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  const double s = ratio[fb.inst];
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += kFlatThreads) {
    const double a = psi[k], n1 = nn[k], p1 = pp[k];
    const double a0 = psi_prev[k], n0 = n_prev[k], p0 = p_prev[k];
    psi_prev[k] = a;
    n_prev[k] = n1;
    p_prev[k] = p1;
    if (s != 0.0) {
      psi[k] = a + s * (a - a0);
      if (n0 > 0.0 && n1 > 0.0)
        nn[k] = n1 * fmin(fmax(exp(s * log(n1 / n0)), 0.1), 10.0);
      if (p0 > 0.0 && p1 > 0.0)
        pp[k] = p1 * fmin(fmax(exp(s * log(p1 / p0)), 0.1), 10.0);
    }
  }
}

}  // namespace tcad

using namespace tcad;

extern "C" int tcad_state_extrapolate(const tcad_pack_t* pk, double* psi, double* n, double* p,
                                      double* psi_prev, double* n_prev, double* p_prev,
                                      const double* ratio, void* stream) {
  if (!pack_ok(pk) || !psi || !n || !p || !psi_prev || !n_prev || !p_prev || !ratio)
    return TCAD_ERR_ARG;
  if (pk->n_flat <= 0) return TCAD_OK;
  k_extrapolate<<<(unsigned)pk->n_flat, kFlatThreads, 0, (cudaStream_t)stream>>>(
      *pk, psi, n, p, psi_prev, n_prev, p_prev, ratio);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

extern "C" int tcad_set_contacts(const tcad_pack_t* pk, const int64_t* nodes, int64_t count,
                                 const int32_t* cid, const double* vv, const double* L,
                                 const double* n0, const double* p0, double* bc_psi0,
                                 double* bc_n0, double* bc_p0, void* stream) {
  if (!pack_ok(pk) || count < 0) return TCAD_ERR_ARG;
  if (count == 0) return TCAD_OK;
  k_set_contacts<<<(unsigned)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      nodes, count, cid, vv, L, n0, p0, bc_psi0, bc_n0, bc_p0);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

extern "C" int tcad_stamp_contacts(const tcad_pack_t* pk, const int64_t* nodes, int64_t count,
                                   double* psi, double* n, double* p, void* stream) {
  if (!pack_ok(pk) || count < 0) return TCAD_ERR_ARG;
  if (count == 0) return TCAD_OK;
  k_stamp_contacts<<<(unsigned)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      *pk, nodes, count, psi, n, p);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}
