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

}  // namespace tcad

using namespace tcad;

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
