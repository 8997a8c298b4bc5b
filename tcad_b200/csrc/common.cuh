// Shared device helpers of the tcad_b200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/tcad_b200.h"

#define TCAD_CUDA_CHECK(expr)                        \
  do {                                               \
    cudaError_t e_ = (expr);                         \
    if (e_ != cudaSuccess) return TCAD_ERR_CUDA;     \
  } while (0)

#define TCAD_LAUNCH_CHECK() TCAD_CUDA_CHECK(cudaGetLastError())

namespace tcad {

// Count of kernels this library launched (defined in capi.cu).
void note_launch(uint64_t n = 1);

constexpr int kFlatThreads = 256;
constexpr int kTileThreads = TCAD_TILE_X * TCAD_TILE_Y;           // 256

// Host-side sanity of the pack's launch-shape fields (the tables themselves
// are the caller's responsibility).
inline bool pack_ok(const tcad_pack_t* pk) {
  return pk && (pk->dim == 2 || pk->dim == 3) && pk->n_inst >= 0 && pk->flat_nodes >= 1 &&
         (pk->dim == 2 || (pk->tile_z >= 1 && pk->tile_z <= TCAD_TILE_Z));
}

// Geometry of one instance as seen by a kernel.
struct Inst {
  int nx, ny, nz;
  int64_t off;  // first node
  int64_t n;    // node count
};

__device__ __forceinline__ Inst load_inst(const tcad_pack_t& pk, int inst) {
  Inst g;
  g.nx = pk.shape[3 * inst + 0];
  g.ny = pk.shape[3 * inst + 1];
  g.nz = pk.shape[3 * inst + 2];
  g.off = pk.node_off[inst];
  g.n = (int64_t)g.nx * g.ny * g.nz;  // instances may sit apart (node_off need not be dense)
  return g;
}

// Deterministic block reduction (fixed tree order) of one double per thread.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* smem) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = lane < NT / 32 ? smem[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;  // valid in thread 0
}

template <int NT>
__device__ __forceinline__ double block_max(double v, double* smem) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = lane < NT / 32 ? smem[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, o));
  }
  __syncthreads();
  return r;
}

// Flat-block addressing: block b of the pack covers pk.flat_nodes nodes of
// exactly one instance.  Returns the instance, the first node of the block
// and the instance's end node.
struct FlatBlock {
  int inst;
  int64_t begin, end;  // packed node range [begin, end) handled by this block
  int64_t ioff, iend;  // instance node range
};

__device__ __forceinline__ FlatBlock flat_block(const tcad_pack_t& pk, int64_t b) {
  FlatBlock fb;
  fb.inst = pk.flat_inst[b];
  fb.ioff = pk.node_off[fb.inst];
  fb.iend = fb.ioff + (int64_t)pk.shape[3 * fb.inst] * pk.shape[3 * fb.inst + 1] *
                          pk.shape[3 * fb.inst + 2];
  const int64_t local = b - pk.flat_off[fb.inst];
  fb.begin = fb.ioff + local * pk.flat_nodes;
  fb.end = fb.begin + pk.flat_nodes < fb.iend ? fb.begin + pk.flat_nodes : fb.iend;
  return fb;
}

// Coupled assembly over a list of tiles (nullptr: all n_tiles); the Newton
// driver uses it to assemble only the instances still iterating.
int sg_assemble_tiles(const tcad_pack_t* pk, const double* psi, const double* n,
                      const double* p, double* F, double* J, int mode, const int32_t* tiles,
                      int64_t n_list, cudaStream_t s);

// Theta-scheme storage term of a time step on the assembled rows, over a list
// of flat blocks (nullptr: all n_flat).
int storage_terms(const tcad_pack_t* pk, const double* n, const double* p,
                  const double* n_old, const double* p_old, const double* fn_old,
                  const double* fp_old, double dt, double theta, double* F, double* J,
                  const int32_t* blk, int64_t n_list, cudaStream_t s);

}  // namespace tcad
