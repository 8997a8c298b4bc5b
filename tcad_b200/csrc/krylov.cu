// Node-block linear algebra, Krylov solvers and the Newton drivers.
//
// All kernels are "flat": block b owns pk.flat_nodes consecutive nodes of
// one instance (flat_block()).  Reductions are per instance and
// deterministic: each block writes its partial sums, and the LAST block of
// the instance to finish (atomic ticket) sums the partials in block order and
// updates the instance's scalar state (alpha, omega, ...).  The host only
// looks at the per-instance state every few iterations, so the iteration
// itself runs without host round trips; blocks of finished instances return
// immediately, which is the per-instance convergence mask of a packed batch.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <vector>

#include "common.cuh"

namespace tcad {

constexpr int NT = kFlatThreads;

// Per-instance Krylov state (device memory, mirrored to the host).
struct KState {
  double rho, rho_prev, alpha, omega, beta;
  double rr, bb, tol2, r0n2, rv, ss;
  int32_t it, maxit, status, active, restart, early, pad0, pad1;
};

template <int DIM>
struct Stencil {
  static constexpr int NE = DIM == 2 ? TCAD_NE2 : TCAD_NE3;
  static constexpr int ND = 2 * DIM;
};

__device__ __forceinline__ int64_t clampi(int64_t m, int64_t lo, int64_t hi) {
  return m < lo ? lo : (m >= hi ? hi - 1 : m);
}

__device__ __forceinline__ void nbr_offsets(const Inst& g, int64_t* off) {
  const int64_t sxy = (int64_t)g.nx * g.ny;
  off[0] = -1; off[1] = 1; off[2] = -(int64_t)g.nx; off[3] = g.nx;
  off[4] = -sxy; off[5] = sxy;
}

// --------------------------------------------------------------------------
// partial sums -> per-instance totals.  store(): this block's sums into
// partial[b * 4 + q]; total(): the instance's block partials summed in block
// order (valid in thread 0).  run(): both, the total taken by the LAST block
// of the instance to finish (atomic ticket); true in every thread of that
// block.
template <int NS>
struct Reduce {
  __device__ static void store(int64_t b, double (&v)[NS], double* partial) {
    __shared__ double sm[32];
    __shared__ double st[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      const double r = block_sum<NT>(v[q], sm);
      if (threadIdx.x == 0) st[q] = r;
    }
    if (threadIdx.x == 0) {
#pragma unroll
      for (int q = 0; q < NS; ++q) partial[b * 4 + q] = st[q];
    }
  }
  __device__ static void total(const tcad_pack_t& pk, int inst, const double* partial,
                               double* tot) {
    __shared__ double sm[32];
    const int64_t b0 = pk.flat_off[inst], b1 = pk.flat_off[inst + 1];
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      double s = 0.0;
      for (int64_t bb = b0 + threadIdx.x; bb < b1; bb += NT) s += __ldcg(&partial[bb * 4 + q]);
      const double r = block_sum<NT>(s, sm);
      if (threadIdx.x == 0) tot[q] = r;
    }
  }
  __device__ static bool run(const tcad_pack_t& pk, int64_t b, int inst, double (&v)[NS],
                             double* partial, unsigned* ticket, double* tot) {
    __shared__ int last;
    store(b, v, partial);
    if (threadIdx.x == 0) {
      __threadfence();
      const int64_t nb = pk.flat_off[inst + 1] - pk.flat_off[inst];
      const unsigned prev = atomicAdd(&ticket[inst], 1u);
      last = (prev == (unsigned)(nb - 1));
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    total(pk, inst, partial, tot);
    if (threadIdx.x == 0) ticket[inst] = 0u;
    return true;
  }
};

// --------------------------------------------------------------------------
// BiCGStab scalar updates of one instance from its totals.  Both the
// launch-per-step kernels (last block of the instance) and the fused
// persistent kernel (every CTA, on its shared copy) use these.
__device__ __forceinline__ void fin_init(KState& s, double tot, double rt, int maxit,
                                         int pre) {
  s.bb = tot; s.rr = tot; s.r0n2 = tot;
  s.tol2 = rt * rt * tot;
  s.rho = tot; s.rho_prev = 1.0; s.alpha = 1.0; s.omega = 1.0;
  s.beta = 0.0; s.it = 0; s.maxit = maxit; s.restart = 0; s.early = 0;
  s.status = pre;
  const bool done = s.status != TCAD_OK || !(tot > 0.0) || !isfinite(tot);
  if (s.status == TCAD_OK && !isfinite(tot)) s.status = TCAD_ERR_NONFINITE;
  s.active = done ? 0 : 1;
}

// alpha = rho / (rh, v)
__device__ __forceinline__ void fin_v(KState& s, double rv) {
  s.restart = 0;
  s.rv = rv;
  if (rv == 0.0 || !isfinite(rv)) {
    s.status = TCAD_ERR_BREAKDOWN;
    s.active = 0;
  } else {
    s.alpha = s.rho / rv;
  }
}

// (s, s): early exit when s alone meets the tolerance
__device__ __forceinline__ void fin_s(KState& s, double ss) {
  s.ss = ss;
  s.early = ss <= s.tol2 ? 1 : 0;
}

// omega = (t, s) / (t, t)
__device__ __forceinline__ void fin_t(KState& s, double ts, double tt) {
  s.omega = (s.early || !(tt > 0.0)) ? 0.0 : ts / tt;
}

// rho = (rh, r), convergence on (r, r), restart when the shadow residual is lost
__device__ __forceinline__ void fin_x(KState& s, double rhr, double rr, double hh) {
  s.it += 1;
  s.rr = rr;
  s.rho_prev = s.rho;
  s.rho = rhr;
  if (!isfinite(rr)) {
    s.status = TCAD_ERR_NONFINITE;
    s.active = 0;
  } else if (rr <= s.tol2) {
    s.active = 0;                     // converged (true residual checked next)
  } else if (s.it >= s.maxit) {
    s.status = TCAD_ERR_NOCONV;
    s.active = 0;
  } else if (s.omega == 0.0 || fabs(rhr) <= 1e-14 * sqrt(rr * hh)) {
    s.restart = 1;                    // shadow residual lost: restart from r
    s.rho = rr;
    s.r0n2 = rr;
    s.beta = 0.0;
  } else {
    s.beta = (s.rho / s.rho_prev) * (s.alpha / s.omega);
  }
}

// true residual norm; re-arm a restart when the recursive residual drifted
__device__ __forceinline__ void fin_true(KState& s, double rr, int rearm) {
  s.rr = rr;
  if (rearm && s.status == TCAD_OK && s.bb > 0.0 && rr > 4.0 * s.tol2 && s.it < s.maxit &&
      isfinite(rr)) {
    s.active = 1;
    s.restart = 1;
    s.rho = rr;
    s.r0n2 = rr;
  }
}

}  // namespace tcad
#include "ilu.cuh"
namespace tcad {

// --------------------------------------------------------------------------
// block-Jacobi set-up: invert the 3x3 diagonal blocks, scale the rhs
//
// With densities (nn, pp non-null) the unknowns become relative updates
// (dpsi, dn/s_n, dp/s_p), s = max(density, floor): the operator is
// S^-1 D^-1 A S -- a similarity transform of the block-scaled operator, so
// the same SpMV applies -- with the n/p rows of D^-1 divided by the node's s
// and every neighbour block's n<-n / p<-p entry multiplied by that neighbour's
// s.  Every component of the Krylov vectors is then on the scale of the
// Newton update test, which is what an FP32 inner solve needs.
template <int DIM>
__global__ void __launch_bounds__(NT)
k_bj_setup(const tcad_pack_t pk, double* __restrict__ J, double* __restrict__ F,
           int32_t* __restrict__ status, const double* __restrict__ nn,
           const double* __restrict__ pp, double floor_, const int32_t* __restrict__ blk,
           const double* __restrict__ floor_inst = nullptr) {
  const FlatBlock fb = flat_block(pk, blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x);
  if (floor_inst) floor_ = floor_inst[fb.inst];   // per-instance floor of this step
  const int64_t NN = pk.n_nodes;
  const bool rel = nn != nullptr;
  int64_t off[6];
  if (rel) nbr_offsets(load_inst(pk, fb.inst), off);
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
    double a[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) a[e] = J[(int64_t)e * NN + k];
    const double c00 = a[4] * a[8] - a[5] * a[7];
    const double c01 = a[5] * a[6] - a[3] * a[8];
    const double c02 = a[3] * a[7] - a[4] * a[6];
    const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    bool ok = isfinite(det) && fabs(det) >= 1e-300;
#pragma unroll
    for (int e = 0; e < 9; ++e) ok = ok && isfinite(a[e]);
    double inv[9];
    if (ok) {
      const double id = 1.0 / det;
      inv[0] = c00 * id;
      inv[1] = (a[2] * a[7] - a[1] * a[8]) * id;
      inv[2] = (a[1] * a[5] - a[2] * a[4]) * id;
      inv[3] = c01 * id;
      inv[4] = (a[0] * a[8] - a[2] * a[6]) * id;
      inv[5] = (a[2] * a[3] - a[0] * a[5]) * id;
      inv[6] = c02 * id;
      inv[7] = (a[1] * a[6] - a[0] * a[7]) * id;
      inv[8] = (a[0] * a[4] - a[1] * a[3]) * id;
    } else {
      atomicExch(&status[fb.inst], TCAD_ERR_SINGULAR);
#pragma unroll
      for (int e = 0; e < 9; ++e) inv[e] = (e % 4 == 0) ? 1.0 : 0.0;
    }
    double sn = 1.0, sp = 1.0;
    if (rel) {
      sn = fmax(nn[k], floor_);
      sp = fmax(pp[k], floor_);
      const double isn = 1.0 / sn, isp = 1.0 / sp;
      inv[3] *= isn; inv[4] *= isn; inv[5] *= isn;
      inv[6] *= isp; inv[7] *= isp; inv[8] *= isp;
#pragma unroll
      for (int d = 0; d < 2 * DIM; ++d) {
        const int64_t m = clampi(k + off[d], fb.ioff, fb.iend);
        const int64_t en = (int64_t)(9 + 5 * d + 2) * NN + k;   // n <- n
        const int64_t ep = (int64_t)(9 + 5 * d + 4) * NN + k;   // p <- p
        J[en] = J[en] * fmax(nn[m], floor_);
        J[ep] = J[ep] * fmax(pp[m], floor_);
      }
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) J[(int64_t)e * NN + k] = inv[e];
    const double r0 = -F[k], r1 = -F[NN + k], r2 = -F[2 * NN + k];
    if (!(isfinite(r0) && isfinite(r1) && isfinite(r2)))
      atomicExch(&status[fb.inst], TCAD_ERR_NONFINITE);
    F[k] = inv[0] * r0 + inv[1] * r1 + inv[2] * r2;
    F[NN + k] = inv[3] * r0 + inv[4] * r1 + inv[5] * r2;
    F[2 * NN + k] = inv[6] * r0 + inv[7] * r1 + inv[8] * r2;
  }
}

// y = x + Dinv * (sum_d A_d x_nbr(d))      (SCALED)
// y = D x + sum_d A_d x_nbr(d)             (raw J, !SCALED)
// T is the storage and arithmetic type (double: plain path; float: the
// mixed-precision inner solves).
// The vector is read through X(m, c) = x[c * NN + m] (spmv_node) or any
// other functor giving the same values (the fused solve forms neighbour
// values on the fly); the arithmetic is the same either way.
template <int DIM, bool SCALED, class T, class XF, class TJ>
__device__ __forceinline__ void spmv_node_f(const TJ* __restrict__ J, const XF& X, int64_t k,
                                            int64_t NN, const int64_t* off, int64_t lo,
                                            int64_t hi, T& y0, T& y1, T& y2) {
  T t0 = T(0), t1 = T(0), t2 = T(0);
#pragma unroll
  for (int d = 0; d < 2 * DIM; ++d) {
    const int64_t m = clampi(k + off[d], lo, hi);
    const int e = 9 + 5 * d;
    const T xs = X(m, 0), xn = X(m, 1), xp = X(m, 2);
    t0 += T(J[(int64_t)e * NN + k]) * xs;
    t1 += T(J[(int64_t)(e + 1) * NN + k]) * xs + T(J[(int64_t)(e + 2) * NN + k]) * xn;
    t2 += T(J[(int64_t)(e + 3) * NN + k]) * xs + T(J[(int64_t)(e + 4) * NN + k]) * xp;
  }
  const T x0 = X(k, 0), x1 = X(k, 1), x2 = X(k, 2);
  T d[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) d[e] = T(J[(int64_t)e * NN + k]);
  if (SCALED) {
    y0 = x0 + (d[0] * t0 + d[1] * t1 + d[2] * t2);
    y1 = x1 + (d[3] * t0 + d[4] * t1 + d[5] * t2);
    y2 = x2 + (d[6] * t0 + d[7] * t1 + d[8] * t2);
  } else {
    y0 = d[0] * x0 + d[1] * x1 + d[2] * x2 + t0;
    y1 = d[3] * x0 + d[4] * x1 + d[5] * x2 + t1;
    y2 = d[6] * x0 + d[7] * x1 + d[8] * x2 + t2;
  }
}

template <int DIM, bool SCALED, class T, class TJ = T>
__device__ __forceinline__ void spmv_node(const TJ* __restrict__ J, const T* __restrict__ x,
                                          int64_t k, int64_t NN, const int64_t* off,
                                          int64_t lo, int64_t hi, T& y0, T& y1, T& y2) {
  spmv_node_f<DIM, SCALED, T>(J, [&](int64_t m, int c) { return x[c * NN + m]; }, k, NN, off,
                              lo, hi, y0, y1, y2);
}

template <int DIM, bool SCALED>
__global__ void __launch_bounds__(NT)
k_spmv(const tcad_pack_t pk, const double* __restrict__ J, const double* __restrict__ x,
       double* __restrict__ y) {
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  const Inst g = load_inst(pk, fb.inst);
  int64_t off[6];
  nbr_offsets(g, off);
  const int64_t NN = pk.n_nodes;
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
    double y0, y1, y2;
    spmv_node<DIM, SCALED, double>(J, x, k, NN, off, fb.ioff, fb.iend, y0, y1, y2);
    y[k] = y0; y[NN + k] = y1; y[2 * NN + k] = y2;
  }
}

// --------------------------------------------------------------------------
// BiCGStab on A^ (per instance).  Vectors: r, rh (shadow), p, v, s, t; x.
// Scalars and dot products are always FP64.  Each step's per-block work is a
// body function (returning the thread's partial dot products), shared by the
// launch-per-step kernels and the fused persistent kernel, so both run the
// same arithmetic in the same order.
template <class T>
struct BiVecT {
  T *r, *rh, *p, *v, *s, *t;
  T *ph, *sh;  // M^-1 p and M^-1 s (right preconditioner); = p, s without one
};
using BiVec = BiVecT<double>;

// x = 0, r = rh = b, p = v = 0; (b, b)
template <class T>
__device__ __forceinline__ double bi_init_body(const tcad_pack_t& pk, const FlatBlock& fb,
                                               const T* __restrict__ b, T* __restrict__ x,
                                               const BiVecT<T>& w) {
  const int64_t NN = pk.n_nodes;
  double v = 0.0;
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t q = c * NN + k;
      const T bv = b[q];
      x[q] = T(0); w.r[q] = bv; w.rh[q] = bv; w.p[q] = T(0); w.v[q] = T(0);
      v += (double)bv * (double)bv;
    }
  }
  return v;
}

// p = r + beta (p - omega v)   (restart: rh = r, p = r)
// The vector bodies read through restrict-qualified locals and issue every
// load of two nodes before any store, so each thread keeps a dozen loads in
// flight (the struct members alone would force load-store serialisation).
template <class T>
__device__ __forceinline__ void bi_p_body(const tcad_pack_t& pk, const FlatBlock& fb,
                                          const BiVecT<T>& w, T beta, T omega, int restart) {
  const int64_t NN = pk.n_nodes;
  const T* __restrict__ R = w.r;
  const T* __restrict__ V = w.v;
  T* __restrict__ P = w.p;
  T* __restrict__ RH = w.rh;
  for (int64_t k0 = fb.begin + threadIdx.x; k0 < fb.end; k0 += 2 * NT) {
    const int64_t k1 = k0 + NT;
    const bool two = k1 < fb.end;
    T r[6], pv[6], vv[6];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      r[c] = R[c * NN + k0];
      if (!restart) { pv[c] = P[c * NN + k0]; vv[c] = V[c * NN + k0]; }
      if (two) {
        r[3 + c] = R[c * NN + k1];
        if (!restart) { pv[3 + c] = P[c * NN + k1]; vv[3 + c] = V[c * NN + k1]; }
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (h == 1 && !two) break;
      const int64_t k = h ? k1 : k0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int q = 3 * h + c;
        if (restart) {
          RH[c * NN + k] = r[q];
          P[c * NN + k] = r[q];
        } else {
          P[c * NN + k] = r[q] + beta * (pv[q] - omega * vv[q]);
        }
      }
    }
  }
}

// v = A^ ph; (rh, v)
template <int DIM, class T, class TJ = T>
__device__ __forceinline__ double bi_v_body(const tcad_pack_t& pk, const FlatBlock& fb,
                                            const TJ* __restrict__ J, const BiVecT<T>& w) {
  const Inst g = load_inst(pk, fb.inst);
  int64_t off[6];
  nbr_offsets(g, off);
  const int64_t NN = pk.n_nodes;
  double v = 0.0;
  const T* __restrict__ X = w.ph;
  const T* __restrict__ RH = w.rh;
  T* __restrict__ Vo = w.v;
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
    T y0, y1, y2;
    spmv_node<DIM, true, T>(J, X, k, NN, off, fb.ioff, fb.iend, y0, y1, y2);
    const T h0 = RH[k], h1 = RH[NN + k], h2 = RH[2 * NN + k];
    Vo[k] = y0; Vo[NN + k] = y1; Vo[2 * NN + k] = y2;
    v += (double)h0 * y0 + (double)h1 * y1 + (double)h2 * y2;
  }
  return v;
}

// s = r - alpha v; (s, s)
template <class T>
__device__ __forceinline__ double bi_s_body(const tcad_pack_t& pk, const FlatBlock& fb,
                                            const BiVecT<T>& w, T alpha) {
  const int64_t NN = pk.n_nodes;
  const T* __restrict__ R = w.r;
  const T* __restrict__ V = w.v;
  T* __restrict__ S = w.s;
  double v = 0.0;
  for (int64_t k0 = fb.begin + threadIdx.x; k0 < fb.end; k0 += 2 * NT) {
    const int64_t k1 = k0 + NT;
    const bool two = k1 < fb.end;
    T r[6], vv[6];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      r[c] = R[c * NN + k0];
      vv[c] = V[c * NN + k0];
      if (two) { r[3 + c] = R[c * NN + k1]; vv[3 + c] = V[c * NN + k1]; }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (h == 1 && !two) break;
      const int64_t k = h ? k1 : k0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T sv = r[3 * h + c] - alpha * vv[3 * h + c];
        S[c * NN + k] = sv;
        v += (double)sv * (double)sv;
      }
    }
  }
  return v;
}

// t = A^ sh; (t, s), (t, t)
template <int DIM, class T, class TJ = T>
__device__ __forceinline__ void bi_t_body(const tcad_pack_t& pk, const FlatBlock& fb,
                                          const TJ* __restrict__ J, const BiVecT<T>& w,
                                          double (&v)[2]) {
  const Inst g = load_inst(pk, fb.inst);
  int64_t off[6];
  nbr_offsets(g, off);
  const int64_t NN = pk.n_nodes;
  v[0] = 0.0; v[1] = 0.0;
  const T* __restrict__ X = w.sh;
  const T* __restrict__ S = w.s;
  T* __restrict__ To = w.t;
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
    T y0, y1, y2;
    spmv_node<DIM, true, T>(J, X, k, NN, off, fb.ioff, fb.iend, y0, y1, y2);
    const T s0 = S[k], s1 = S[NN + k], s2 = S[2 * NN + k];
    To[k] = y0; To[NN + k] = y1; To[2 * NN + k] = y2;
    v[0] += (double)y0 * s0 + (double)y1 * s1 + (double)y2 * s2;
    v[1] += (double)y0 * y0 + (double)y1 * y1 + (double)y2 * y2;
  }
}

// The s and t steps in one pass (fused solve, no preconditioner): s = r -
// alpha v at the block's nodes (stored), t = A^ s with the neighbours' s
// formed from their r and v (neither changes in this step); (s, s), (t, s),
// (t, t).  Same expressions and accumulation order as bi_s_body followed by
// bi_t_body.
template <int DIM, class TJ = double>
__device__ __forceinline__ void bi_st_body(const tcad_pack_t& pk, const FlatBlock& fb,
                                           const TJ* __restrict__ J, const BiVec& w,
                                           double alpha, double (&v)[3]) {
  const Inst g = load_inst(pk, fb.inst);
  int64_t off[6];
  nbr_offsets(g, off);
  const int64_t NN = pk.n_nodes;
  v[0] = 0.0; v[1] = 0.0; v[2] = 0.0;
  const double* R = w.r;
  const double* V = w.v;
  double* S = w.s;
  double* To = w.t;
  const auto sval = [&](int64_t m, int c) {
    const double rv = R[c * NN + m], vv = V[c * NN + m];
    const double sv = rv - alpha * vv;
    return sv;
  };
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
    const double s0 = sval(k, 0), s1 = sval(k, 1), s2 = sval(k, 2);
    S[k] = s0; S[NN + k] = s1; S[2 * NN + k] = s2;
    v[0] += (double)s0 * (double)s0;
    v[0] += (double)s1 * (double)s1;
    v[0] += (double)s2 * (double)s2;
    double y0, y1, y2;
    spmv_node_f<DIM, true, double>(J, sval, k, NN, off, fb.ioff, fb.iend, y0, y1, y2);
    To[k] = y0; To[NN + k] = y1; To[2 * NN + k] = y2;
    v[1] += (double)y0 * s0 + (double)y1 * s1 + (double)y2 * s2;
    v[2] += (double)y0 * y0 + (double)y1 * y1 + (double)y2 * y2;
  }
}

// x += alpha ph + omega sh; r = s - omega t; (rh, r), (r, r), (rh, rh)
template <class T>
__device__ __forceinline__ void bi_x_body(const tcad_pack_t& pk, const FlatBlock& fb,
                                          T* __restrict__ x, const BiVecT<T>& w, T alpha,
                                          T omega, double (&v)[3]) {
  const int64_t NN = pk.n_nodes;
  const T* __restrict__ PH = w.ph;
  const T* __restrict__ SH = w.sh;
  const T* __restrict__ S = w.s;
  const T* __restrict__ Tt = w.t;
  const T* __restrict__ RH = w.rh;
  T* __restrict__ R = w.r;
  v[0] = 0.0; v[1] = 0.0; v[2] = 0.0;
  for (int64_t k0 = fb.begin + threadIdx.x; k0 < fb.end; k0 += 2 * NT) {
    const int64_t k1 = k0 + NT;
    const bool two = k1 < fb.end;
    T xv[6], ph[6], sh[6], sv[6], tv[6], rh[6];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t q0 = c * NN + k0;
      xv[c] = x[q0]; ph[c] = PH[q0]; sh[c] = SH[q0]; sv[c] = S[q0]; tv[c] = Tt[q0];
      rh[c] = RH[q0];
      if (two) {
        const int64_t q1 = c * NN + k1;
        xv[3 + c] = x[q1]; ph[3 + c] = PH[q1]; sh[3 + c] = SH[q1]; sv[3 + c] = S[q1];
        tv[3 + c] = Tt[q1]; rh[3 + c] = RH[q1];
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (h == 1 && !two) break;
      const int64_t k = h ? k1 : k0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int q = 3 * h + c;
        x[c * NN + k] = xv[q] + alpha * ph[q] + omega * sh[q];
        const T r = sv[q] - omega * tv[q];
        R[c * NN + k] = r;
        v[0] += (double)rh[q] * r;
        v[1] += (double)r * r;
        v[2] += (double)rh[q] * rh[q];
      }
    }
  }
}

// r = b - A^ x; (r, r)
template <int DIM, class T, class TJ = T>
__device__ __forceinline__ double true_resid_body(const tcad_pack_t& pk, const FlatBlock& fb,
                                                  const TJ* __restrict__ J,
                                                  const T* __restrict__ b,
                                                  const T* __restrict__ x, T* __restrict__ r) {
  const Inst g = load_inst(pk, fb.inst);
  int64_t off[6];
  nbr_offsets(g, off);
  const int64_t NN = pk.n_nodes;
  double v = 0.0;
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
    T y0, y1, y2;
    spmv_node<DIM, true, T>(J, x, k, NN, off, fb.ioff, fb.iend, y0, y1, y2);
    const T a0 = b[k] - y0, a1 = b[NN + k] - y1, a2 = b[2 * NN + k] - y2;
    r[k] = a0; r[NN + k] = a1; r[2 * NN + k] = a2;
    v += (double)a0 * a0 + (double)a1 * a1 + (double)a2 * a2;
  }
  return v;
}

// ---- one launch per step (any pack; blocks of finished instances return)
template <class T>
__global__ void __launch_bounds__(NT)
k_bi_init(const tcad_pack_t pk, const T* __restrict__ b, T* __restrict__ x, BiVecT<T> w,
          KState* ks, double* partial, unsigned* ticket, double rtol, int maxit,
          const int32_t* __restrict__ pre_status, const double* __restrict__ rtol_inst) {
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  double v[1] = {bi_init_body<T>(pk, fb, b, x, w)};
  double tot[1];
  if (Reduce<1>::run(pk, blockIdx.x, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0)
    fin_init(ks[fb.inst], tot[0], rtol_inst ? rtol_inst[fb.inst] : rtol, maxit,
             pre_status ? pre_status[fb.inst] : TCAD_OK);
}

template <class T>
__global__ void __launch_bounds__(NT, 4)
k_bi_p(const tcad_pack_t pk, BiVecT<T> w, const KState* ks, const int32_t* __restrict__ blk) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pk, fbi);
  const KState s = ks[fb.inst];
  if (!s.active) return;
  bi_p_body<T>(pk, fb, w, (T)s.beta, (T)s.omega, s.restart);
}

template <int DIM, class T, class TJ = T>
__global__ void __launch_bounds__(NT)
k_bi_v(const tcad_pack_t pk, const TJ* __restrict__ J, BiVecT<T> w, KState* ks,
       double* partial, unsigned* ticket, const int32_t* __restrict__ blk) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pk, fbi);
  if (!ks[fb.inst].active) return;
  double v[1] = {bi_v_body<DIM, T, TJ>(pk, fb, J, w)};
  double tot[1];
  if (Reduce<1>::run(pk, fbi, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0)
    fin_v(ks[fb.inst], tot[0]);
}

template <class T>
__global__ void __launch_bounds__(NT, 4)
k_bi_s(const tcad_pack_t pk, BiVecT<T> w, KState* ks, double* partial, unsigned* ticket,
       const int32_t* __restrict__ blk) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pk, fbi);
  const KState s0 = ks[fb.inst];
  if (!s0.active) return;
  double v[1] = {bi_s_body<T>(pk, fb, w, (T)s0.alpha)};
  double tot[1];
  if (Reduce<1>::run(pk, fbi, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0)
    fin_s(ks[fb.inst], tot[0]);
}

template <int DIM, class T, class TJ = T>
__global__ void __launch_bounds__(NT)
k_bi_t(const tcad_pack_t pk, const TJ* __restrict__ J, BiVecT<T> w, KState* ks,
       double* partial, unsigned* ticket, const int32_t* __restrict__ blk) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pk, fbi);
  if (!ks[fb.inst].active) return;
  double v[2];
  bi_t_body<DIM, T, TJ>(pk, fb, J, w, v);
  double tot[2];
  if (Reduce<2>::run(pk, fbi, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0)
    fin_t(ks[fb.inst], tot[0], tot[1]);
}

template <class T>
__global__ void __launch_bounds__(NT, 3)
k_bi_x(const tcad_pack_t pk, T* __restrict__ x, BiVecT<T> w, KState* ks, double* partial,
       unsigned* ticket, const int32_t* __restrict__ blk) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pk, fbi);
  const KState s0 = ks[fb.inst];
  if (!s0.active) return;
  double v[3];
  bi_x_body<T>(pk, fb, x, w, (T)s0.alpha, (T)s0.omega, v);
  double tot[3];
  if (Reduce<3>::run(pk, fbi, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0)
    fin_x(ks[fb.inst], tot[0], tot[1], tot[2]);
}

// true scaled residual r = b - A^ x, its norm into the state; re-arm a restart
// when it is not within the tolerance the recursive residual claimed
template <int DIM, class T, class TJ = T>
__global__ void __launch_bounds__(NT)
k_true_resid(const tcad_pack_t pk, const TJ* __restrict__ J, const T* __restrict__ b,
             const T* __restrict__ x, T* __restrict__ r, KState* ks, double* partial,
             unsigned* ticket, int rearm) {
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  double v[1] = {true_resid_body<DIM, T, TJ>(pk, fb, J, b, x, r)};
  double tot[1];
  if (Reduce<1>::run(pk, blockIdx.x, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0)
    fin_true(ks[fb.inst], tot[0], rearm);
}

}  // namespace tcad
#include "redblack.cuh"
namespace tcad {

// ---- the whole solve in one cooperative launch (single-instance packs whose
// flat blocks all fit on the GPU at once: one CTA per flat block)
//
// Grid barrier: thread 0 of each CTA adds one arrival to the monotonic
// counter bar[0] (acquire-release, so the CTA's writes before the barrier are
// visible to every CTA after it) and waits until the counter reaches
// round x nblocks.  Every wait is bounded: past kBarrierNs of device time, or
// once another CTA has given up (bar[2] != 0), the CTA sets bar[2] and the
// barrier returns false, and the kernel returns -- the host sees bar[2] and
// solves again with one launch per step.  bar[3] is added to every round's
// target: 0 always, except under the give-up test hook
// (tcad_set_krylov_fused_test), which sets it to 1 so that the first barrier
// waits for an arrival that never comes and its time limit runs out.
constexpr unsigned long long kBarrierNs = 1000000000ull;   // 1 s

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;"
               : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned nblocks, unsigned& round) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int good = 1;
    round += 1u;
    const unsigned target = round * nblocks + ld_acquire(&bar[3]);
    const unsigned prev = atom_add_acq_rel(&bar[0], 1u);
    if (prev + 1u != target) {
      const unsigned long long t0 = globaltimer_ns();
      for (unsigned it = 0;; ++it) {
        if ((int)(ld_acquire(&bar[0]) - target) >= 0) break;
        if ((it & 255u) == 255u) {
          if (ld_acquire(&bar[2]) != 0u) { good = 0; break; }
          if (globaltimer_ns() - t0 > kBarrierNs || it > (1u << 30)) {
            atomicExch(&bar[2], 1u);
            good = 0;
            break;
          }
          __nanosleep(32);
        }
      }
    }
    __threadfence();
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// Four barriers per iteration: p; v (alpha); s and t in one pass (early,
// omega); x (rho, beta, convergence).  Block partials alternate between two
// halves of `partial` by step parity: a CTA reaches the next step's store
// only after every CTA has passed the barrier that follows its read of the
// previous totals.
template <int DIM>
__global__ void __launch_bounds__(NT, 2)
k_bicgstab_fused(const tcad_pack_t pk, const double* __restrict__ J,
                 const double* __restrict__ b, double* __restrict__ x, BiVec w, KState* ks,
                 double* partial, unsigned* bar, double rtol, int maxit,
                 const int32_t* __restrict__ pre_status, const double* __restrict__ rtol_inst,
                 int max_rechecks) {
  __shared__ KState S;
  const unsigned G = gridDim.x;
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  const int inst = fb.inst;
  double* const half[2] = {partial, partial + 4 * (int64_t)pk.n_flat};
  int ph = 0;
  unsigned round = 0;
  double tot[3];
  {
    double v[1] = {bi_init_body<double>(pk, fb, b, x, w)};
    Reduce<1>::store(blockIdx.x, v, half[ph]);
    if (!grid_barrier(bar, G, round)) return;
    Reduce<1>::total(pk, inst, half[ph], tot);
    ph ^= 1;
    if (threadIdx.x == 0)
      fin_init(S, tot[0], rtol_inst ? rtol_inst[inst] : rtol, maxit,
               pre_status ? pre_status[inst] : TCAD_OK);
    __syncthreads();
  }
  for (int rechecks = 0;; ++rechecks) {
    while (S.active) {
      bi_p_body<double>(pk, fb, w, S.beta, S.omega, S.restart);
      if (!grid_barrier(bar, G, round)) return;
      {
        double v[1] = {bi_v_body<DIM, double>(pk, fb, J, w)};
        Reduce<1>::store(blockIdx.x, v, half[ph]);
        if (!grid_barrier(bar, G, round)) return;
        Reduce<1>::total(pk, inst, half[ph], tot);
        ph ^= 1;
        if (threadIdx.x == 0) fin_v(S, tot[0]);
        __syncthreads();
      }
      if (!S.active) break;
      {
        double v[3];
        bi_st_body<DIM>(pk, fb, J, w, S.alpha, v);
        Reduce<3>::store(blockIdx.x, v, half[ph]);
        if (!grid_barrier(bar, G, round)) return;
        Reduce<3>::total(pk, inst, half[ph], tot);
        ph ^= 1;
        if (threadIdx.x == 0) {
          fin_s(S, tot[0]);
          fin_t(S, tot[1], tot[2]);
        }
        __syncthreads();
      }
      {
        double v[3];
        bi_x_body<double>(pk, fb, x, w, S.alpha, S.omega, v);
        Reduce<3>::store(blockIdx.x, v, half[ph]);
        if (!grid_barrier(bar, G, round)) return;
        Reduce<3>::total(pk, inst, half[ph], tot);
        ph ^= 1;
        if (threadIdx.x == 0) fin_x(S, tot[0], tot[1], tot[2]);
        __syncthreads();
      }
    }
    {
      double v[1] = {true_resid_body<DIM, double>(pk, fb, J, b, x, w.r)};
      Reduce<1>::store(blockIdx.x, v, half[ph]);
      if (!grid_barrier(bar, G, round)) return;
      Reduce<1>::total(pk, inst, half[ph], tot);
      ph ^= 1;
      if (threadIdx.x == 0) fin_true(S, tot[0], rechecks < max_rechecks ? 1 : 0);
      __syncthreads();
    }
    if (!S.active) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) ks[inst] = S;
}

// ---- the red-black Schur solve in one cooperative launch (single-instance
// packs whose slot blocks all fit on the GPU at once: one CTA per slot
// block).  The search direction and s are formed on the fly by the red
// passes (RbFormP / RbFormS) and stored by the black passes, so an iteration
// takes five grid barriers: red(p); p + v (alpha); red(s); s + t (early,
// omega); x (rho, beta, convergence).  Bodies, scalar updates and reduction
// order are the per-step kernels' own, so the result is bit-identical to
// launch_bicgstab_rb's one launch per step.  Every wait is bounded as in
// k_bicgstab_fused; a CTA that gives up returns and the host solves again
// one launch per step.
template <int DIM>
__global__ void __launch_bounds__(NT, 2)
k_bicgstab_rb_fused(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ JR,
                    const double* __restrict__ JB, const double* __restrict__ b,
                    double* __restrict__ x, double* __restrict__ bR, double* __restrict__ bB,
                    double* __restrict__ Tr, double* __restrict__ xb,
                    double* __restrict__ rhs, BiVec w, KState* ks, double* partial,
                    unsigned* bar, double rtol, int maxit,
                    const int32_t* __restrict__ pre_status,
                    const double* __restrict__ rtol_inst, int max_rechecks) {
  __shared__ KState S;
  const unsigned G = gridDim.x;
  const FlatBlock fb = flat_block(pkb, blockIdx.x);
  const int inst = fb.inst;
  const int64_t NS = pkb.n_nodes;
  double* const half[2] = {partial, partial + 4 * (int64_t)pkb.n_flat};
  int ph = 0;
  unsigned round = 0;
  double tot[3];
  double bb = 0.0;
  {
    double v[1] = {rb_split_body<DIM>(pkb, mp, fb, b, bR, bB)};
    Reduce<1>::store(blockIdx.x, v, half[ph]);
    if (!grid_barrier(bar, G, round)) return;
    Reduce<1>::total(pkb, inst, half[ph], tot);
    ph ^= 1;
    bb = tot[0];
  }
  {
    double v[1] = {rb_init_body<DIM>(pkb, mp, fb, JB, bR, bB, rhs, xb, w)};
    Reduce<1>::store(blockIdx.x, v, half[ph]);
    if (!grid_barrier(bar, G, round)) return;
    Reduce<1>::total(pkb, inst, half[ph], tot);
    ph ^= 1;
    if (threadIdx.x == 0)
      rb_fin_init(S, tot[0], bb, rtol_inst ? rtol_inst[inst] : rtol, maxit,
                  pre_status ? pre_status[inst] : TCAD_OK);
    __syncthreads();
  }
  for (int rechecks = 0;; ++rechecks) {
    while (S.active) {
      rb_red_body<DIM>(pkb, mp, fb, JR,
                       RbMakeP{w.r, w.p, w.v, NS, S.beta, S.omega, S.restart}, Tr);
      if (!grid_barrier(bar, G, round)) return;
      {
        double v[1] = {rb_v_body<DIM, true>(pkb, mp, fb, JB, Tr, w, S.beta, S.omega,
                                            S.restart)};
        Reduce<1>::store(blockIdx.x, v, half[ph]);
        if (!grid_barrier(bar, G, round)) return;
        Reduce<1>::total(pkb, inst, half[ph], tot);
        ph ^= 1;
        if (threadIdx.x == 0) fin_v(S, tot[0]);
        __syncthreads();
      }
      if (!S.active) break;
      rb_red_body<DIM>(pkb, mp, fb, JR, RbMakeS{w.r, w.v, NS, S.alpha}, Tr);
      if (!grid_barrier(bar, G, round)) return;
      {
        double v[3];
        rb_t_body<DIM, true>(pkb, mp, fb, JB, Tr, w, S.alpha, v);
        Reduce<3>::store(blockIdx.x, v, half[ph]);
        if (!grid_barrier(bar, G, round)) return;
        Reduce<3>::total(pkb, inst, half[ph], tot);
        ph ^= 1;
        if (threadIdx.x == 0) {
          fin_s(S, tot[0]);
          fin_t(S, tot[1], tot[2]);
        }
        __syncthreads();
      }
      {
        double v[3];
        bi_x_body<double>(pkb, fb, xb, w, S.alpha, S.omega, v);
        Reduce<3>::store(blockIdx.x, v, half[ph]);
        if (!grid_barrier(bar, G, round)) return;
        Reduce<3>::total(pkb, inst, half[ph], tot);
        ph ^= 1;
        if (threadIdx.x == 0) fin_x(S, tot[0], tot[1], tot[2]);
        __syncthreads();
      }
    }
    rb_red_body<DIM>(pkb, mp, fb, JR, RbMakeVal{xb, NS}, Tr);
    if (!grid_barrier(bar, G, round)) return;
    {
      double v[1] = {rb_true_body<DIM>(pkb, mp, fb, JB, Tr, rhs, xb, w.r)};
      Reduce<1>::store(blockIdx.x, v, half[ph]);
      if (!grid_barrier(bar, G, round)) return;
      Reduce<1>::total(pkb, inst, half[ph], tot);
      ph ^= 1;
      if (threadIdx.x == 0) fin_true(S, tot[0], rechecks < max_rechecks ? 1 : 0);
      __syncthreads();
    }
    if (!S.active) break;
  }
  rb_merge_body<DIM>(pkb, mp, fb, bR, Tr, xb, x,
                     pre_status && pre_status[inst] != TCAD_OK);
  if (blockIdx.x == 0 && threadIdx.x == 0) ks[inst] = S;
}

// --------------------------------------------------------------------------
// Newton update (device2d.py:2079-2100): per-instance max update into err
__global__ void __launch_bounds__(NT)
k_newton_update(const tcad_pack_t pk, double* __restrict__ psi, double* __restrict__ nn,
                double* __restrict__ pp, const double* __restrict__ du, double max_dpsi,
                double floor_, const uint8_t* __restrict__ active,
                unsigned long long* __restrict__ err, int relative, int dry, double sfloor,
                const double* __restrict__ sfloor_inst = nullptr) {
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  if (active && !active[fb.inst]) return;
  if (sfloor_inst) sfloor = sfloor_inst[fb.inst];  // the floor the step was scaled with
  __shared__ double sm[32];
  const int64_t NN = pk.n_nodes;
  double e = 0.0;
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
    const double n0 = nn[k], p0 = pp[k];
    const double u0 = du[k];
    // relative-update unknowns come back scaled by max(density, floor)
    const double u1 = relative ? du[NN + k] * fmax(n0, sfloor) : du[NN + k];
    const double u2 = relative ? du[2 * NN + k] * fmax(p0, sfloor) : du[2 * NN + k];
    const bool finite = isfinite(u0) && isfinite(u1) && isfinite(u2);
    double dpsi = u0 < -max_dpsi ? -max_dpsi : (u0 > max_dpsi ? max_dpsi : u0);
    double n1 = n0 + u1, p1 = p0 + u2;
    // numpy.clip(a, lo, hi) = minimum(maximum(a, lo), hi)
    n1 = fmin(fmax(n1, 0.1 * n0), 10.0 * n0);
    p1 = fmin(fmax(p1, 0.1 * p0), 10.0 * p0);
    const double rn = fabs(n1 - n0) / fmax(n0, floor_);
    const double rp = fabs(p1 - p0) / fmax(p0, floor_);
    double ek = fmax(fabs(dpsi), fmax(rn, rp));
    if (!finite || !(ek == ek)) ek = INFINITY;  // NaN update: never "converged"
    e = fmax(e, ek);
    if (!dry) {
      psi[k] = psi[k] + dpsi;
      nn[k] = n1;
      pp[k] = p1;
    }
  }
  const double m = block_max<NT>(e, sm);
  if (threadIdx.x == 0) atomicMax(&err[fb.inst], (unsigned long long)__double_as_longlong(m));
}

// --------------------------------------------------------------------------
// equilibrium Poisson: PCG on A = -J (symmetric positive definite after the
// symmetric elimination), Jacobi preconditioner, energy-norm stopping test
struct CgVec {
  double *r, *z, *p, *q;
};

template <int DIM>
__device__ __forceinline__ double pspmv(const double* __restrict__ J,
                                        const double* __restrict__ x, int64_t k, int64_t NN,
                                        const int64_t* off, int64_t lo, int64_t hi) {
  double y = J[k] * x[k];
#pragma unroll
  for (int d = 0; d < 2 * DIM; ++d) {
    const int64_t m = clampi(k + off[d], lo, hi);
    y += J[(int64_t)(1 + d) * NN + k] * x[m];
  }
  return -y;
}

__global__ void __launch_bounds__(NT)
k_cg_init(const tcad_pack_t pk, const double* __restrict__ J, const double* __restrict__ b,
          double* __restrict__ x, CgVec w, KState* ks, double* partial, unsigned* ticket,
          double rtol, int maxit, const uint8_t* __restrict__ active,
          const double* __restrict__ rtol_inst) {
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  const int64_t NN = pk.n_nodes;
  double v[2] = {0.0, 0.0};
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
    const double bv = b[k];
    const double z = bv / (-J[k]);
    x[k] = 0.0; w.r[k] = bv; w.z[k] = z; w.p[k] = z;
    v[0] += bv * z;
    v[1] += bv * bv;
  }
  (void)NN;
  double tot[2];
  if (Reduce<2>::run(pk, blockIdx.x, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0) {
    KState& s = ks[fb.inst];
    s.bb = tot[0]; s.rho = tot[0]; s.rr = tot[0];
    const double rt = rtol_inst ? rtol_inst[fb.inst] : rtol;
    s.tol2 = rt * rt * tot[0];
    s.it = 0; s.maxit = maxit; s.status = TCAD_OK; s.restart = 0; s.early = 0;
    if (!isfinite(tot[0]) || !isfinite(tot[1])) s.status = TCAD_ERR_NONFINITE;
    s.active = (s.status == TCAD_OK && tot[0] > 0.0 && (!active || active[fb.inst])) ? 1 : 0;
  }
}

template <int DIM>
__global__ void __launch_bounds__(NT)
k_cg_q(const tcad_pack_t pk, const double* __restrict__ J, CgVec w, KState* ks,
       double* partial, unsigned* ticket, const int32_t* __restrict__ blk) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pk, fbi);
  if (!ks[fb.inst].active) return;
  const Inst g = load_inst(pk, fb.inst);
  int64_t off[6];
  nbr_offsets(g, off);
  const int64_t NN = pk.n_nodes;
  double v[1] = {0.0};
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
    const double q = pspmv<DIM>(J, w.p, k, NN, off, fb.ioff, fb.iend);
    w.q[k] = q;
    v[0] += w.p[k] * q;
  }
  double tot[1];
  if (Reduce<1>::run(pk, fbi, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0) {
    KState& s = ks[fb.inst];
    if (!(tot[0] > 0.0) || !isfinite(tot[0])) {
      s.status = TCAD_ERR_BREAKDOWN;
      s.active = 0;
    } else {
      s.alpha = s.rho / tot[0];
    }
  }
}

__global__ void __launch_bounds__(NT)
k_cg_x(const tcad_pack_t pk, const double* __restrict__ J, double* __restrict__ x, CgVec w,
       KState* ks, double* partial, unsigned* ticket, const int32_t* __restrict__ blk) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pk, fbi);
  const KState s0 = ks[fb.inst];
  if (!s0.active) return;
  double v[1] = {0.0};
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
    x[k] = x[k] + s0.alpha * w.p[k];
    const double r = w.r[k] - s0.alpha * w.q[k];
    w.r[k] = r;
    const double z = r / (-J[k]);
    w.z[k] = z;
    v[0] += r * z;
  }
  double tot[1];
  if (Reduce<1>::run(pk, fbi, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0) {
    KState& s = ks[fb.inst];
    s.it += 1;
    s.rho_prev = s.rho;
    s.rho = tot[0];
    s.rr = tot[0];
    if (!isfinite(tot[0])) {
      s.status = TCAD_ERR_NONFINITE;
      s.active = 0;
    } else if (tot[0] <= s.tol2) {
      s.active = 0;
    } else if (s.it >= s.maxit) {
      s.status = TCAD_ERR_NOCONV;
      s.active = 0;
    } else {
      s.beta = s.rho / s.rho_prev;
    }
  }
}

__global__ void __launch_bounds__(NT)
k_cg_p(const tcad_pack_t pk, CgVec w, const KState* ks, const int32_t* __restrict__ blk) {
  const FlatBlock fb = flat_block(pk, blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x);
  const KState s = ks[fb.inst];
  if (!s.active) return;
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) w.p[k] = w.z[k] + s.beta * w.p[k];
}

// ---- equilibrium PCG on the red-black Schur complement (scalar Poisson)
//
// The equilibrium Newton step solves A d = F with A = -J (SPD: the box-
// integration Laplacian plus the diagonal charge derivative; eliminated
// Dirichlet rows are identity rows).  Its 5-/7-point stencil has no coupling
// inside a colour, so with the colour slot layout of redblack.cuh
//     A = [ A_rr  A_rb ]      S = A_bb - A_br A_rr^-1 A_rb   (SPD, black slots)
//         [ A_br  A_bb ]      S d_b = F_b - A_br A_rr^-1 F_r,
//                             d_r = A_rr^-1 (F_r - A_rb d_b),
// A_rr diagonal.  PCG runs on S with its exact diagonal as the Jacobi
// preconditioner: half the unknowns, the same matrix bytes per product
// (a red pass t = A_rr^-1 A_rb p and a black pass q = A_bb p - A_br t).
// The colour rows of J (1 + 2 DIM entries, the diagonal first) are stored
// entry-major per colour: JRe / JBe [1 + 2 DIM][slots].

// JRe, JBe <- colour rows of the equilibrium J; bR, bB <- colours of F
template <int DIM>
__global__ void __launch_bounds__(NT)
k_eqrb_pack(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ J,
            const double* __restrict__ F, double* __restrict__ JRe, double* __restrict__ JBe,
            double* __restrict__ bR, double* __restrict__ bB) {
  constexpr int NE = 1 + 2 * DIM;
  const FlatBlock fb = flat_block(pkb, blockIdx.x);
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes, NN = mp.n_full;
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const RbNode q = rb_node(g, slot, c);
      double* __restrict__ out = c ? JBe : JRe;
#pragma unroll
      for (int e = 0; e < NE; ++e)
        out[(int64_t)e * NS + slot] = q.real ? J[(int64_t)e * NN + q.node] : 0.0;
      (c ? bB : bR)[slot] = q.real ? F[q.node] : 0.0;
    }
  }
}

// red pass: Tr = A_rr^-1 (v_r - A_rb x) at the block's red slots (v null:
// -A_rr^-1 A_rb x); every instance when ks is null
template <int DIM>
__global__ void __launch_bounds__(NT)
k_eqrb_red(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ JRe,
           const double* __restrict__ x, const double* __restrict__ vr,
           double* __restrict__ Tr, const KState* ks, const int32_t* __restrict__ blk) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pkb, fbi);
  if (ks && !ks[fb.inst].active) return;
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes;
  const double* __restrict__ xi = x + g.soff;
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    const RbNode q = rb_node(g, slot, 0);
    double t = 0.0;
    if (q.real) {
      int m[6];
      rb_nbrs<DIM>(g, q, (int)(slot - g.soff), m);
      double a = 0.0;                         // (J_rb x): A_rb = -J_rb
#pragma unroll
      for (int d = 0; d < 2 * DIM; ++d) a += JRe[(int64_t)(1 + d) * NS + slot] * xi[m[d]];
      const double arr = -JRe[slot];
      t = ((vr ? vr[slot] : 0.0) + a) / arr;  // A_rr^-1 (v_r - A_rb x)
    }
    Tr[slot] = t;
  }
}

// black coupling at one slot: sum_d A_bd Tr(m_d) = -sum_d J_bd Tr(m_d)
template <int DIM>
__device__ __forceinline__ double eqrb_black_u(const RbGeo& g, const double* __restrict__ JBe,
                                               const double* __restrict__ Tr, int64_t slot,
                                               int64_t NS, const RbNode& q) {
  int m[6];
  rb_nbrs<DIM>(g, q, (int)(slot - g.soff), m);
  const double* __restrict__ ti = Tr + g.soff;
  double a = 0.0;
#pragma unroll
  for (int d = 0; d < 2 * DIM; ++d) a += JBe[(int64_t)(1 + d) * NS + slot] * ti[m[d]];
  return -a;
}

// Sinv = 1 / diag(S): diag(S)_b = A_bb - sum_d A_bd A_{r(d) b} / A_{r(d)}
template <int DIM>
__global__ void __launch_bounds__(NT)
k_eqrb_diag(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ JRe,
            const double* __restrict__ JBe, double* __restrict__ Sinv) {
  const FlatBlock fb = flat_block(pkb, blockIdx.x);
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes;
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    const RbNode q = rb_node(g, slot, 1);
    double sd = 0.0;
    if (q.real) {
      int m[6];
      rb_nbrs<DIM>(g, q, (int)(slot - g.soff), m);
      sd = -JBe[slot];
#pragma unroll
      for (int d = 0; d < 2 * DIM; ++d) {
        const double jbd = JBe[(int64_t)(1 + d) * NS + slot];
        if (jbd != 0.0) {                     // a real neighbour: its row holds
          const int64_t r = g.soff + m[d];    //   the coupling back, direction d ^ 1
          const double jrb = JRe[(int64_t)(1 + (d ^ 1)) * NS + r];
          sd -= (jbd * jrb) / (-JRe[r]);
        }
      }
    }
    Sinv[slot] = (q.real && sd != 0.0) ? 1.0 / sd : 0.0;
  }
}

// Schur start: rhs = F_b - A_br A_rr^-1 F_r (Tr = A_rr^-1 F_r from the red
// pass), x = 0, r = rhs, z = Sinv r, p = z; (r, z), (r, r) as k_cg_init
template <int DIM>
__global__ void __launch_bounds__(NT)
k_eqrb_init(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ JBe,
            const double* __restrict__ bB, const double* __restrict__ Tr,
            const double* __restrict__ Sinv, double* __restrict__ x, CgVec w, KState* ks,
            double* partial, unsigned* ticket, double rtol, int maxit,
            const uint8_t* __restrict__ active, const double* __restrict__ rtol_inst) {
  const FlatBlock fb = flat_block(pkb, blockIdx.x);
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes;
  double v[2] = {0.0, 0.0};
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    const RbNode q = rb_node(g, slot, 1);
    const double bv = q.real ? bB[slot] - eqrb_black_u<DIM>(g, JBe, Tr, slot, NS, q) : 0.0;
    const double z = bv * Sinv[slot];
    x[slot] = 0.0; w.r[slot] = bv; w.z[slot] = z; w.p[slot] = z;
    v[0] += bv * z;
    v[1] += bv * bv;
  }
  double tot[2];
  if (Reduce<2>::run(pkb, blockIdx.x, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0) {
    KState& s = ks[fb.inst];
    s.bb = tot[0]; s.rho = tot[0]; s.rr = tot[0];
    const double rt = rtol_inst ? rtol_inst[fb.inst] : rtol;
    s.tol2 = rt * rt * tot[0];
    s.it = 0; s.maxit = maxit; s.status = TCAD_OK; s.restart = 0; s.early = 0;
    if (!isfinite(tot[0]) || !isfinite(tot[1])) s.status = TCAD_ERR_NONFINITE;
    s.active = (s.status == TCAD_OK && tot[0] > 0.0 && (!active || active[fb.inst])) ? 1 : 0;
  }
}

// q = S p (Tr from the red pass of p); alpha = rho / (p, q)
template <int DIM>
__global__ void __launch_bounds__(NT)
k_eqrb_q(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ JBe,
         const double* __restrict__ Tr, CgVec w, KState* ks, double* partial,
         unsigned* ticket, const int32_t* __restrict__ blk) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pkb, fbi);
  if (!ks[fb.inst].active) return;
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes;
  double v[1] = {0.0};
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    const RbNode q = rb_node(g, slot, 1);
    const double pv = w.p[slot];
    // S p = A_bb p + A_br t, t = -A_rr^-1 A_rb p
    const double qv = q.real ? -JBe[slot] * pv + eqrb_black_u<DIM>(g, JBe, Tr, slot, NS, q)
                             : 0.0;
    w.q[slot] = qv;
    v[0] += pv * qv;
  }
  double tot[1];
  if (Reduce<1>::run(pkb, fbi, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0) {
    KState& s = ks[fb.inst];
    if (!(tot[0] > 0.0) || !isfinite(tot[0])) {
      s.status = TCAD_ERR_BREAKDOWN;
      s.active = 0;
    } else {
      s.alpha = s.rho / tot[0];
    }
  }
}

// x += alpha p, r -= alpha q, z = Sinv r; (r, z), convergence as k_cg_x
__global__ void __launch_bounds__(NT)
k_eqrb_x(const tcad_pack_t pkb, const double* __restrict__ Sinv, double* __restrict__ x,
         CgVec w, KState* ks, double* partial, unsigned* ticket,
         const int32_t* __restrict__ blk) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pkb, fbi);
  const KState s0 = ks[fb.inst];
  if (!s0.active) return;
  double v[1] = {0.0};
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
    x[k] = x[k] + s0.alpha * w.p[k];
    const double r = w.r[k] - s0.alpha * w.q[k];
    w.r[k] = r;
    const double z = r * Sinv[k];
    w.z[k] = z;
    v[0] += r * z;
  }
  double tot[1];
  if (Reduce<1>::run(pkb, fbi, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0) {
    KState& s = ks[fb.inst];
    s.it += 1;
    s.rho_prev = s.rho;
    s.rho = tot[0];
    s.rr = tot[0];
    if (!isfinite(tot[0])) {
      s.status = TCAD_ERR_NONFINITE;
      s.active = 0;
    } else if (tot[0] <= s.tol2) {
      s.active = 0;
    } else if (s.it >= s.maxit) {
      s.status = TCAD_ERR_NOCONV;
      s.active = 0;
    } else {
      s.beta = s.rho / s.rho_prev;
    }
  }
}

// full update: d_r = Tr (= A_rr^-1 (F_r - A_rb d_b) from the red pass), d_b = x
template <int DIM>
__global__ void __launch_bounds__(NT)
k_eqrb_merge(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ Tr,
             const double* __restrict__ xb, double* __restrict__ d) {
  const FlatBlock fb = flat_block(pkb, blockIdx.x);
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    const RbNode qr = rb_node(g, slot, 0);
    const RbNode qb = rb_node(g, slot, 1);
    if (qr.real) d[qr.node] = Tr[slot];
    if (qb.real) d[qb.node] = xb[slot];
  }
}

// equilibrium update: clip to +-max_dpsi, psi += d, err = max |d|
__global__ void __launch_bounds__(NT)
k_eq_update(const tcad_pack_t pk, double* __restrict__ psi, const double* __restrict__ d,
            double max_dpsi, const uint8_t* __restrict__ active,
            unsigned long long* __restrict__ err) {
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  if (active && !active[fb.inst]) return;
  __shared__ double sm[32];
  double e = 0.0;
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
    double v = d[k];
    v = v < -max_dpsi ? -max_dpsi : (v > max_dpsi ? max_dpsi : v);
    psi[k] = psi[k] + v;
    double a = fabs(v);
    if (!(a == a)) a = INFINITY;
    e = fmax(e, a);
  }
  const double m = block_max<NT>(e, sm);
  if (threadIdx.x == 0) atomicMax(&err[fb.inst], (unsigned long long)__double_as_longlong(m));
}

// slaved Boltzmann densities n = nie_s e^psi, p = nie_s e^-psi
__global__ void __launch_bounds__(NT)
k_slaved(const tcad_pack_t pk, const double* __restrict__ psi, double* __restrict__ nn,
         double* __restrict__ pp) {
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
    const double ps = psi[k];
    const double c = ps < -700.0 ? -700.0 : (ps > 700.0 ? 700.0 : ps);
    nn[k] = pk.nie_s[k] * exp(c);
    pp[k] = pk.nie_s[k] * exp(-c);
  }
}

// --------------------------------------------------------------------------
// mixed precision: FP32 copy of the block-scaled operator, FP64 iterative
// refinement around FP32 BiCGStab (the residual always uses the FP64 A^)
__global__ void __launch_bounds__(NT)
k_to_f32(const tcad_pack_t pk, int ne, const double* __restrict__ J, float* __restrict__ J32,
         const int32_t* __restrict__ blk) {
  const FlatBlock fb = flat_block(pk, blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x);
  const int64_t NN = pk.n_nodes;
  for (int e = 0; e < ne; ++e)
    for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT)
      J32[(int64_t)e * NN + k] = (float)J[(int64_t)e * NN + k];
}

// x = 0, ||b||^2.  The refinement keeps its residual in FP64 and hands the
// inner FP32 solve r / ||r|| (k_ir_scale): the scaled right-hand side of a
// Newton step far from the solution can exceed the FP32 range where the
// relative unknowns divide by a density at the floor; normalised, every
// entry is at most 1 and the FP32 solve sees a unit-norm system.
__global__ void __launch_bounds__(NT)
k_ir_init(const tcad_pack_t pk, const double* __restrict__ b, double* __restrict__ x,
          KState* irs, double* partial, unsigned* ticket) {
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  const int64_t NN = pk.n_nodes;
  double v[1] = {0.0};
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t q = c * NN + k;
      const double bv = b[q];
      x[q] = 0.0;
      v[0] += bv * bv;
    }
  }
  double tot[1];
  if (Reduce<1>::run(pk, blockIdx.x, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0) {
    irs[fb.inst].bb = tot[0];
    irs[fb.inst].rr = tot[0];
  }
}

// r32 = (float)(r / ||r||) for the instances still refining (||r||^2 in irs)
__global__ void __launch_bounds__(NT)
k_ir_scale(const tcad_pack_t pk, const double* __restrict__ r, float* __restrict__ r32,
           const KState* irs, const int32_t* __restrict__ pre_status) {
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  if (pre_status[fb.inst] != TCAD_OK) return;
  const int64_t NN = pk.n_nodes;
  const double nrm = sqrt(irs[fb.inst].rr);
  const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT)
#pragma unroll
    for (int c = 0; c < 3; ++c) r32[c * NN + k] = (float)(r[c * NN + k] * inv);
}

// x += ||r|| d32 for the instances still refining (d32 solves A^ d = r/||r||)
__global__ void __launch_bounds__(NT)
k_ir_axpy(const tcad_pack_t pk, double* __restrict__ x, const float* __restrict__ d,
          const KState* irs, const int32_t* __restrict__ pre_status) {
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  if (pre_status[fb.inst] != TCAD_OK) return;
  const int64_t NN = pk.n_nodes;
  const double nrm = sqrt(irs[fb.inst].rr);
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT)
#pragma unroll
    for (int c = 0; c < 3; ++c) x[c * NN + k] += nrm * (double)d[c * NN + k];
}

// r = b - A^ x in FP64 (FP64 operator) into r64, ||r||^2
template <int DIM>
__global__ void __launch_bounds__(NT)
k_ir_resid(const tcad_pack_t pk, const double* __restrict__ J, const double* __restrict__ b,
           const double* __restrict__ x, double* __restrict__ r64, KState* irs,
           const int32_t* __restrict__ pre_status, double* partial, unsigned* ticket) {
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  if (pre_status[fb.inst] != TCAD_OK) return;
  const Inst g = load_inst(pk, fb.inst);
  int64_t off[6];
  nbr_offsets(g, off);
  const int64_t NN = pk.n_nodes;
  double v[1] = {0.0};
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT) {
    double y0, y1, y2;
    spmv_node<DIM, true, double>(J, x, k, NN, off, fb.ioff, fb.iend, y0, y1, y2);
    const double a0 = b[k] - y0, a1 = b[NN + k] - y1, a2 = b[2 * NN + k] - y2;
    r64[k] = a0; r64[NN + k] = a1; r64[2 * NN + k] = a2;
    v[0] += a0 * a0 + a1 * a1 + a2 * a2;
  }
  double tot[1];
  if (Reduce<1>::run(pk, blockIdx.x, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0)
    irs[fb.inst].rr = tot[0];
}

// --------------------------------------------------------------------------
// workspace carving
struct Carve {
  char* base;
  size_t used;
  size_t cap;
  template <class T>
  T* take(size_t count) {
    const size_t bytes = (count * sizeof(T) + 255) & ~(size_t)255;
    T* p = reinterpret_cast<T*>(base + used);
    used += bytes;
    return p;
  }
};

struct Work {
  BiVec bi;
  CgVec cg;
  double* partial;  // 2 x 4 x n_flat: block partial sums (the fused solve alternates halves)
  unsigned* bar;    // fused solve's grid barrier: counter, generation, gave-up flag
  KState* ks;
  unsigned* ticket;
  int32_t* status;
  unsigned long long* err;
  double* eta;
  double* sfl;   // per-instance density floor of the relative unknowns this step
  int32_t* blk;  // compact list of the flat blocks still iterating (Krylov)
  int32_t* fl;   // flat blocks / tiles of the instances a Newton step still
  int32_t* tl;   //   solves (assembly and block-Jacobi set-up)
  size_t bytes;
};

// FP32 extension of the workspace (mixed-precision Newton), carved after Work
struct Work32 {
  BiVecT<float> bi;
  float* J32;
  float* r32;
  float* d32;
  KState* irs;
  double* eta_in;
  int32_t* pre;
  size_t bytes;
};

static Work32 carve32(const tcad_pack_t* pk, void* base) {
  Carve c{reinterpret_cast<char*>(base), 0, 0};
  Work32 w;
  const size_t v3 = 3 * (size_t)pk->n_nodes;
  w.bi.r = c.take<float>(v3);
  w.bi.rh = c.take<float>(v3);
  w.bi.p = c.take<float>(v3);
  w.bi.v = c.take<float>(v3);
  w.bi.s = c.take<float>(v3);
  w.bi.t = c.take<float>(v3);
  w.bi.ph = w.bi.p;
  w.bi.sh = w.bi.s;
  w.J32 = c.take<float>((size_t)(pk->dim == 2 ? TCAD_NE2 : TCAD_NE3) * pk->n_nodes);
  w.r32 = c.take<float>(v3);
  w.d32 = c.take<float>(v3);
  w.irs = c.take<KState>(pk->n_inst);
  w.eta_in = c.take<double>(pk->n_inst);
  w.pre = c.take<int32_t>(pk->n_inst);
  w.bytes = c.used;
  return w;
}

// ILU(0) extension: Q = D~^-1 per node, M^-1 p and M^-1 s
struct WorkIlu {
  double* Q;
  double* ph;
  double* sh;
  uint8_t* mask;    // instances preconditioned with ILU(0)
  int32_t* pre;     // factor pre-status (-1: skip)
  float* Mf;        // 2D: forward sweep data in anti-diagonal slot order [27][2n]
  float* Mb;        //     backward sweep data [18][2n]
  double* rs;       //     right-hand side in slot order [3][2n]
  double* xs;       //     sweep result in slot order [3][2n]
  size_t bytes;
};

static WorkIlu carve_ilu(const tcad_pack_t* pk, void* base) {
  Carve c{reinterpret_cast<char*>(base), 0, 0};
  WorkIlu w{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0};
  const size_t v3 = 3 * (size_t)pk->n_nodes;
  w.Q = c.take<double>(9 * (size_t)pk->n_nodes);
  w.ph = c.take<double>(v3);
  w.sh = c.take<double>(v3);
  w.mask = c.take<uint8_t>(pk->n_inst);
  w.pre = c.take<int32_t>(pk->n_inst);
  if (pk->dim == 2) {
    const size_t ns = 2 * (size_t)pk->n_nodes;
    w.Mf = c.take<float>(27 * ns);
    w.Mb = c.take<float>(18 * ns);
    w.rs = c.take<double>(3 * ns);
    w.xs = c.take<double>(3 * ns);
  }
  w.bytes = c.used;
  return w;
}

// Red-black Schur extension: the colour rows of the scaled J, the colours of
// b, the red pass result, the black iterate and right-hand side (slot arrays
// sized by n_nodes, which bounds the slot count), the full ||b||^2 and the
// slot pack's tables
struct WorkRb {
  double *JR, *JB, *bR, *bB, *tR, *xb, *rhs, *bbf;
  int32_t* shape;
  int64_t* node_off;
  int64_t* flat_off;
  int32_t* flat_inst;
  int32_t* blk;  // compact list of the slot pack's flat blocks still iterating
  size_t bytes;
};

// Slot-pack flat blocks hold pk->flat_nodes slots (measured, 200-iteration
// solves on the two-lane 983k-node tri-gate: 419 us per iteration at 512
// slots and 5 CTAs per SM, 450 at 256 slots, 511 at 256 slots and 4 CTAs,
// 774 at 128).  The count is bounded by slots / rb_flat + n_inst <=
// n_nodes / rb_flat + n_inst.
static int64_t rb_flat(const tcad_pack_t* pk) { return pk->flat_nodes; }
static size_t rb_flat_cap(const tcad_pack_t* pk) {
  return (size_t)(pk->n_nodes / rb_flat(pk)) + (size_t)pk->n_inst + 1;
}

static WorkRb carve_rb(const tcad_pack_t* pk, void* base) {
  Carve c{reinterpret_cast<char*>(base), 0, 0};
  WorkRb w;
  const size_t nn = (size_t)pk->n_nodes, v3 = 3 * nn;
  const size_t ne = pk->dim == 2 ? TCAD_NE2 : TCAD_NE3;
  w.JR = c.take<double>(ne * (nn + 32));   // warp tiles of 32 slots
  w.JB = c.take<double>(ne * (nn + 32));
  w.bR = c.take<double>(v3);
  w.bB = c.take<double>(v3);
  w.tR = c.take<double>(v3);
  w.xb = c.take<double>(v3);
  w.rhs = c.take<double>(v3);
  w.bbf = c.take<double>(pk->n_inst);
  w.shape = c.take<int32_t>(3 * (size_t)pk->n_inst);
  w.node_off = c.take<int64_t>((size_t)pk->n_inst + 1);
  w.flat_off = c.take<int64_t>((size_t)pk->n_inst + 1);
  w.flat_inst = c.take<int32_t>(rb_flat_cap(pk));
  w.blk = c.take<int32_t>(rb_flat_cap(pk));
  w.bytes = c.used;
  return w;
}

// Equilibrium red-black extension: the colour rows of the Poisson J, the
// Schur diagonal's inverse, the colours of F, the red pass result, the black
// iterate (slot arrays sized by n_nodes) and the slot pack's tables.  Part of
// every workspace (about 15 doubles a node in 3D).
struct WorkEq {
  double *JRe, *JBe, *Sinv, *bR, *bB, *tR, *xb;
  int32_t* shape;
  int64_t* node_off;
  int64_t* flat_off;
  int32_t* flat_inst;
  int32_t* blk;
  size_t bytes;
};

static WorkEq carve_eq(const tcad_pack_t* pk, void* base) {
  Carve c{reinterpret_cast<char*>(base), 0, 0};
  WorkEq w;
  const size_t nn = (size_t)pk->n_nodes;
  const size_t ne = 1 + 2 * (size_t)pk->dim;
  w.JRe = c.take<double>(ne * nn);
  w.JBe = c.take<double>(ne * nn);
  w.Sinv = c.take<double>(nn);
  w.bR = c.take<double>(nn);
  w.bB = c.take<double>(nn);
  w.tR = c.take<double>(nn);
  w.xb = c.take<double>(nn);
  w.shape = c.take<int32_t>(3 * (size_t)pk->n_inst);
  w.node_off = c.take<int64_t>((size_t)pk->n_inst + 1);
  w.flat_off = c.take<int64_t>((size_t)pk->n_inst + 1);
  w.flat_inst = c.take<int32_t>(rb_flat_cap(pk));
  w.blk = c.take<int32_t>(rb_flat_cap(pk));
  w.bytes = c.used;
  return w;
}

// The slot pack of a pack (host tables; see redblack.cuh): per instance
// (ceil(Nx/2), Ny Nz, 1) slots of each colour, flat blocks of pk->flat_nodes
struct RbLayout {
  tcad_pack_t pkb;
  RbMap mp;
  std::vector<int64_t> hfoff;
};

template <class W>   // WorkRb or WorkEq: the slot pack's table arrays
static int rb_layout(const tcad_pack_t* pk, const W& wr, RbLayout& L, cudaStream_t s) {
  const int ni = pk->n_inst;
  std::vector<int32_t> shp(3 * (size_t)ni), sb(3 * (size_t)ni), fi;
  TCAD_CUDA_CHECK(cudaMemcpyAsync(shp.data(), pk->shape, sizeof(int32_t) * shp.size(),
                                  cudaMemcpyDeviceToHost, s));
  TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
  std::vector<int64_t> noff(ni + 1), foff(ni + 1);
  noff[0] = 0; foff[0] = 0;
  const int64_t fn = rb_flat(pk);
  for (int i = 0; i < ni; ++i) {
    const int64_t hx = (shp[3 * i] + 1) / 2, rows = (int64_t)shp[3 * i + 1] * shp[3 * i + 2];
    sb[3 * i] = (int32_t)hx; sb[3 * i + 1] = (int32_t)rows; sb[3 * i + 2] = 1;
    noff[i + 1] = noff[i] + hx * rows;
    const int64_t nf = (hx * rows + fn - 1) / fn;
    foff[i + 1] = foff[i] + nf;
    for (int64_t b = 0; b < nf; ++b) fi.push_back(i);
  }
  // (the Krylov partials hold 8 n_flat doubles: 4 per slot block fit, as
  // n_flat >= max(n_inst, n_nodes / flat_nodes))
  if (noff[ni] > pk->n_nodes || (size_t)foff[ni] > rb_flat_cap(pk) ||
      4 * foff[ni] > 8 * pk->n_flat)
    return TCAD_ERR_ARG;
  TCAD_CUDA_CHECK(cudaMemcpyAsync(wr.shape, sb.data(), sizeof(int32_t) * sb.size(),
                                  cudaMemcpyHostToDevice, s));
  TCAD_CUDA_CHECK(cudaMemcpyAsync(wr.node_off, noff.data(), sizeof(int64_t) * noff.size(),
                                  cudaMemcpyHostToDevice, s));
  TCAD_CUDA_CHECK(cudaMemcpyAsync(wr.flat_off, foff.data(), sizeof(int64_t) * foff.size(),
                                  cudaMemcpyHostToDevice, s));
  TCAD_CUDA_CHECK(cudaMemcpyAsync(wr.flat_inst, fi.data(), sizeof(int32_t) * fi.size(),
                                  cudaMemcpyHostToDevice, s));
  TCAD_CUDA_CHECK(cudaStreamSynchronize(s));   // the host vectors go out of scope
  L.pkb = *pk;
  L.pkb.n_nodes = noff[ni];
  L.pkb.n_flat = foff[ni];
  L.pkb.shape = wr.shape;
  L.pkb.node_off = wr.node_off;
  L.pkb.flat_off = wr.flat_off;
  L.pkb.flat_inst = wr.flat_inst;
  L.pkb.flat_nodes = (int32_t)fn;
  L.mp.shape = pk->shape;
  L.mp.node_off = pk->node_off;
  L.mp.n_full = pk->n_nodes;
  L.hfoff = foff;
  return TCAD_OK;
}

static Work carve(const tcad_pack_t* pk, void* base, size_t cap) {
  Carve c{reinterpret_cast<char*>(base), 0, cap};
  Work w;
  const size_t v3 = 3 * (size_t)pk->n_nodes;
  w.bi.r = c.take<double>(v3);
  w.bi.rh = c.take<double>(v3);
  w.bi.p = c.take<double>(v3);
  w.bi.v = c.take<double>(v3);
  w.bi.s = c.take<double>(v3);
  w.bi.t = c.take<double>(v3);
  w.bi.ph = w.bi.p;
  w.bi.sh = w.bi.s;
  // the scalar PCG reuses the first vector's storage (3 x n_nodes)
  w.cg.r = w.bi.r;
  w.cg.z = w.bi.r + pk->n_nodes;
  w.cg.p = w.bi.r + 2 * pk->n_nodes;
  w.cg.q = w.bi.rh;
  w.partial = c.take<double>(8 * (size_t)pk->n_flat);
  w.bar = c.take<unsigned>(4);
  w.ks = c.take<KState>(pk->n_inst);
  w.ticket = c.take<unsigned>(pk->n_inst);
  w.status = c.take<int32_t>(pk->n_inst);
  w.err = c.take<unsigned long long>(pk->n_inst);
  w.eta = c.take<double>(pk->n_inst);
  w.sfl = c.take<double>(pk->n_inst);
  w.blk = c.take<int32_t>(pk->n_flat);
  w.fl = c.take<int32_t>(pk->n_flat);
  w.tl = c.take<int32_t>(pk->n_tiles);
  w.bytes = c.used;
  return w;
}

// out = M^-1 r: the coalesced slot-order sweeps when the factor wrote them
// (2D, every shorter side <= kIluThreads), else the node-order sweeps
template <class T>
static void ilu_apply_t(const tcad_pack_t* pk, const double* J, const double* Q, const T* r,
                        T* out, const Work& w, const uint8_t* mask, int nzmax,
                        const WorkIlu* ilc, unsigned ng, const int32_t* dlist,
                        cudaStream_t s) {
  const int ni = pk->n_inst;
  if (ilc && ilc->Mf) {
    const int64_t NS = 2 * pk->n_nodes;
    k_ilu_perm<T><<<ng, NT_ILU_FLAT, 0, s>>>(*pk, r, ilc->rs, w.ks, mask, dlist, NS);
    k_ilu_sweep<<<(unsigned)ni, kIluThreads, 0, s>>>(*pk, ilc->Mf, ilc->Mb, ilc->rs, ilc->xs,
                                                     w.ks, mask, NS);
    k_ilu_unperm<T><<<ng, NT_ILU_FLAT, 0, s>>>(*pk, ilc->xs, r, out, w.ks, mask, dlist, NS);
    note_launch(3);
    return;
  }
  k_ilu2d_apply<T><<<(unsigned)(ni * nzmax), kIluThreads, 0, s>>>(*pk, J, Q, r, out, w.ks, mask,
                                                                  nzmax);
  note_launch();
}

// ---- fused (one cooperative launch) BiCGStab: when and how
static std::atomic<int> g_fused_mode{1};   // 0: one launch per step always
static std::atomic<int> g_fused_test_hold{0};        // give-up test hook (bar[3] = 1)
static std::atomic<uint64_t> g_fused_gave_up{0};     // fused launches that gave up

// k_bicgstab_fused<DIM> needs every flat block resident at once
template <int DIM>
static bool fused_fits(unsigned nb) {
  int dev = 0, coop = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop)
    return false;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return false;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_bicgstab_fused<DIM>, NT, 0) !=
      cudaSuccess)
    return false;
  return nb >= 1 && (long long)nb <= (long long)per * sms;
}

// The whole solve of a single-instance pack in one launch (same arithmetic
// as the launch-per-step path).  Returns TCAD_OK with hks[0] filled, or 1
// when the launch was refused or a grid barrier gave up (the caller then
// solves with one launch per step).
// Launch grid of a per-step Krylov loop: every flat block, or -- once the
// instances still iterating cover under 3/4 of them -- only those instances'
// blocks (a compact list rebuilt whenever the active set changes), so a
// batch's stragglers do not pay for launches over finished instances.
struct ActiveGrid {
  unsigned nb = 0, ng = 0;
  const int32_t* dlist = nullptr;
  int ni = 0;
  std::vector<int64_t> hfoff;
  std::vector<int32_t> hlist;
  std::vector<uint8_t> was_active;

  // hfoff_host: the pack's flat_off on the host (read from the device if null)
  int init(const tcad_pack_t* pk, cudaStream_t s, const std::vector<int64_t>* hfoff_host) {
    nb = (unsigned)pk->n_flat;
    ng = nb;
    ni = pk->n_inst;
    if (ni > 1) {
      if (hfoff_host) {
        hfoff = *hfoff_host;
      } else {
        hfoff.resize(ni + 1);
        TCAD_CUDA_CHECK(cudaMemcpyAsync(hfoff.data(), pk->flat_off,
                                        sizeof(int64_t) * (ni + 1), cudaMemcpyDeviceToHost, s));
        TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
      }
      was_active.assign(ni, 1);
    }
    return TCAD_OK;
  }

  int update(const std::vector<KState>& hks, int32_t* dev_list, cudaStream_t s) {
    if (ni <= 1) return TCAD_OK;
    bool changed = false;
    int64_t act_blocks = 0;
    for (int i = 0; i < ni; ++i) {
      changed = changed || (was_active[i] != (hks[i].active ? 1 : 0));
      if (hks[i].active) act_blocks += hfoff[i + 1] - hfoff[i];
    }
    if (!changed) return TCAD_OK;
    for (int i = 0; i < ni; ++i) was_active[i] = hks[i].active ? 1 : 0;
    if (4 * act_blocks < 3 * (int64_t)nb) {
      hlist.clear();
      for (int i = 0; i < ni; ++i)
        if (hks[i].active)
          for (int64_t b = hfoff[i]; b < hfoff[i + 1]; ++b) hlist.push_back((int32_t)b);
      TCAD_CUDA_CHECK(cudaMemcpyAsync(dev_list, hlist.data(), sizeof(int32_t) * hlist.size(),
                                      cudaMemcpyHostToDevice, s));
      ng = (unsigned)hlist.size();
      dlist = dev_list;
    } else {
      ng = nb;
      dlist = nullptr;
    }
    return TCAD_OK;
  }
};

static int launch_bicgstab_fused(const tcad_pack_t* pk, const double* J, const double* b,
                                 double* x, double rtol, int maxiter, const BiVec& bi,
                                 const Work& w, const int32_t* pre_status,
                                 std::vector<KState>& hks, cudaStream_t s,
                                 const double* rtol_inst) {
  TCAD_CUDA_CHECK(cudaMemsetAsync(w.bar, 0, 4 * sizeof(unsigned), s));
  if (g_fused_test_hold.load()) {
    static const unsigned kPhantom = 1u;
    TCAD_CUDA_CHECK(cudaMemcpyAsync(w.bar + 3, &kPhantom, sizeof(unsigned),
                                    cudaMemcpyHostToDevice, s));
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)pk->n_flat);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const int rechecks = 8;
  cudaError_t e =
      pk->dim == 2
          ? cudaLaunchKernelEx(&cfg, k_bicgstab_fused<2>, *pk, J, b, x, bi, w.ks, w.partial,
                               w.bar, rtol, maxiter, pre_status, rtol_inst, rechecks)
          : cudaLaunchKernelEx(&cfg, k_bicgstab_fused<3>, *pk, J, b, x, bi, w.ks, w.partial,
                               w.bar, rtol, maxiter, pre_status, rtol_inst, rechecks);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return 1;
  }
  note_launch();
  hks.resize(1);
  unsigned hbar[4] = {0u, 0u, 0u, 0u};
  TCAD_CUDA_CHECK(cudaMemcpyAsync(hks.data(), w.ks, sizeof(KState), cudaMemcpyDeviceToHost, s));
  TCAD_CUDA_CHECK(cudaMemcpyAsync(hbar, w.bar, sizeof(hbar), cudaMemcpyDeviceToHost, s));
  TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
  if (hbar[2] != 0u) {
    g_fused_gave_up.fetch_add(1);
    return 1;
  }
  return TCAD_OK;
}

template <class T, class TJ = T>
static int launch_bicgstab_t(const tcad_pack_t* pk, const TJ* J, const T* b, T* x, double rtol,
                             int maxiter, const BiVecT<T>& bi, const Work& w,
                             const int32_t* pre_status, std::vector<KState>& hks,
                             cudaStream_t s, const double* rtol_inst,
                             const double* Jilu = nullptr, const double* Qilu = nullptr,
                             const uint8_t* ilu_mask = nullptr, int nzmax = 1,
                             const WorkIlu* ilc = nullptr) {
  const unsigned nb = (unsigned)pk->n_flat;
  const int ni = pk->n_inst;
  if constexpr (std::is_same<T, double>::value && std::is_same<TJ, double>::value) {
    if (g_fused_mode.load() && ni == 1 && Qilu == nullptr &&
        (pk->dim == 2 ? fused_fits<2>(nb) : fused_fits<3>(nb)) &&
        launch_bicgstab_fused(pk, J, b, x, rtol, maxiter, bi, w, pre_status, hks, s,
                              rtol_inst) == TCAD_OK)
      return TCAD_OK;
  }
  TCAD_CUDA_CHECK(cudaMemsetAsync(w.ticket, 0, sizeof(unsigned) * ni, s));
  k_bi_init<<<nb, NT, 0, s>>>(*pk, b, x, bi, w.ks, w.partial, w.ticket, rtol, maxiter,
                              pre_status, rtol_inst);
  note_launch();
  TCAD_LAUNCH_CHECK();
  hks.resize(ni);
  int check = 4;
  int done_iters = 0;
  int rechecks = 0;
  ActiveGrid grid;
  if (int rc = grid.init(pk, s, nullptr)) return rc;
  for (;;) {
    const unsigned ng = grid.ng;
    const int32_t* dlist = grid.dlist;
    for (int q = 0; q < check; ++q) {
      k_bi_p<<<ng, NT, 0, s>>>(*pk, bi, w.ks, dlist);
      note_launch();
      if (Qilu) {  // ph = M^-1 p
        ilu_apply_t<T>(pk, Jilu, Qilu, bi.p, bi.ph, w, ilu_mask, nzmax, ilc, ng, dlist, s);
      }
      if (pk->dim == 2)
        k_bi_v<2><<<ng, NT, 0, s>>>(*pk, J, bi, w.ks, w.partial, w.ticket, dlist);
      else
        k_bi_v<3><<<ng, NT, 0, s>>>(*pk, J, bi, w.ks, w.partial, w.ticket, dlist);
      note_launch();
      // (The s and t steps stay two launches here: k_bi_st, which forms the
      // neighbours' s from their r and v, measured 120 us against 20 + 80 us
      // for k_bi_s + k_bi_t on the 983k-node tri-gate -- two loads per
      // neighbour value instead of one; the single-launch solve of small
      // packs, which is latency-bound, keeps the fused form.)
      {
        k_bi_s<<<ng, NT, 0, s>>>(*pk, bi, w.ks, w.partial, w.ticket, dlist);
        note_launch();
        if (Qilu) {  // sh = M^-1 s
          ilu_apply_t<T>(pk, Jilu, Qilu, bi.s, bi.sh, w, ilu_mask, nzmax, ilc, ng, dlist, s);
        }
        if (pk->dim == 2)
          k_bi_t<2><<<ng, NT, 0, s>>>(*pk, J, bi, w.ks, w.partial, w.ticket, dlist);
        else
          k_bi_t<3><<<ng, NT, 0, s>>>(*pk, J, bi, w.ks, w.partial, w.ticket, dlist);
        note_launch();
      }
      k_bi_x<<<ng, NT, 0, s>>>(*pk, x, bi, w.ks, w.partial, w.ticket, dlist);
      note_launch();
    }
    TCAD_LAUNCH_CHECK();
    done_iters += check;
    TCAD_CUDA_CHECK(cudaMemcpyAsync(hks.data(), w.ks, sizeof(KState) * ni,
                                    cudaMemcpyDeviceToHost, s));
    TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
    bool any = false;
    for (int i = 0; i < ni; ++i) any = any || hks[i].active;
    if (any)
      if (int rc = grid.update(hks, w.blk, s)) return rc;
    if (!any) {
      // true-residual check; instances whose recursive residual drifted are
      // re-armed from the true residual (bounded number of re-checks)
      const int rearm = rechecks < 8 ? 1 : 0;
      if (pk->dim == 2)
        k_true_resid<2><<<nb, NT, 0, s>>>(*pk, J, b, x, bi.r, w.ks, w.partial, w.ticket, rearm);
      else
        k_true_resid<3><<<nb, NT, 0, s>>>(*pk, J, b, x, bi.r, w.ks, w.partial, w.ticket, rearm);
      note_launch();
      TCAD_LAUNCH_CHECK();
      TCAD_CUDA_CHECK(cudaMemcpyAsync(hks.data(), w.ks, sizeof(KState) * ni,
                                      cudaMemcpyDeviceToHost, s));
      TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
      for (int i = 0; i < ni; ++i) any = any || hks[i].active;
      ++rechecks;
      if (!any) break;
    }
    if (done_iters > 64) check = 16;
    if (done_iters > 1024) check = 32;
  }
  return TCAD_OK;
}

template <int DIM>
static bool rb_fused_fits(unsigned nb) {
  int dev = 0, coop = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop)
    return false;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return false;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_bicgstab_rb_fused<DIM>, NT, 0) !=
      cudaSuccess)
    return false;
  return nb >= 1 && (long long)nb <= (long long)per * sms;
}

// The whole red-black solve of a single-instance pack in one launch (same
// arithmetic as launch_bicgstab_rb's per-step loop).  Returns TCAD_OK with
// hks[0] filled, or 1 when the launch was refused or a grid barrier gave up
// (the caller then solves one launch per step).
static int launch_bicgstab_rb_fused(const tcad_pack_t* pk, const RbLayout& L,
                                    const WorkRb& wr, const double* b, double* x,
                                    double rtol, int maxiter, const BiVec& bi, const Work& w,
                                    const int32_t* pre_status, std::vector<KState>& hks,
                                    cudaStream_t s, const double* rtol_inst) {
  TCAD_CUDA_CHECK(cudaMemsetAsync(w.bar, 0, 4 * sizeof(unsigned), s));
  if (g_fused_test_hold.load()) {
    static const unsigned kPhantom = 1u;
    TCAD_CUDA_CHECK(cudaMemcpyAsync(w.bar + 3, &kPhantom, sizeof(unsigned),
                                    cudaMemcpyHostToDevice, s));
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)L.pkb.n_flat);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const int rechecks = 8;
  cudaError_t e =
      pk->dim == 2
          ? cudaLaunchKernelEx(&cfg, k_bicgstab_rb_fused<2>, L.pkb, L.mp, (const double*)wr.JR,
                               (const double*)wr.JB, b, x, wr.bR, wr.bB, wr.tR, wr.xb, wr.rhs,
                               bi, w.ks, w.partial, w.bar, rtol, maxiter, pre_status,
                               rtol_inst, rechecks)
          : cudaLaunchKernelEx(&cfg, k_bicgstab_rb_fused<3>, L.pkb, L.mp, (const double*)wr.JR,
                               (const double*)wr.JB, b, x, wr.bR, wr.bB, wr.tR, wr.xb, wr.rhs,
                               bi, w.ks, w.partial, w.bar, rtol, maxiter, pre_status,
                               rtol_inst, rechecks);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return 1;
  }
  note_launch();
  hks.resize(1);
  unsigned hbar[4] = {0u, 0u, 0u, 0u};
  TCAD_CUDA_CHECK(cudaMemcpyAsync(hks.data(), w.ks, sizeof(KState), cudaMemcpyDeviceToHost, s));
  TCAD_CUDA_CHECK(cudaMemcpyAsync(hbar, w.bar, sizeof(hbar), cudaMemcpyDeviceToHost, s));
  TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
  if (hbar[2] != 0u) {
    g_fused_gave_up.fetch_add(1);
    return 1;
  }
  return TCAD_OK;
}

// BiCGStab on the red-black Schur complement of A^ (redblack.cuh): the same
// per-instance stopping test ||b - A^ x|| <= rtol ||b|| as launch_bicgstab_t,
// the same vector kernels on the black slot pack, and the full solution x
// (node layout) at the end.  JR / JB must hold the colour rows of the current
// J (k_rb_pack after the block-Jacobi set-up).
static int launch_bicgstab_rb(const tcad_pack_t* pk, const RbLayout& L, const WorkRb& wr,
                              const double* b, double* x, double rtol, int maxiter,
                              const Work& w, const int32_t* pre_status,
                              std::vector<KState>& hks, cudaStream_t s,
                              const double* rtol_inst) {
  const tcad_pack_t& pkb = L.pkb;
  const unsigned nbb = (unsigned)pkb.n_flat;
  const int ni = pk->n_inst;
  const bool d2 = pk->dim == 2;
  BiVec bi = w.bi;   // black vectors (stride: the slot count)
  bi.ph = bi.p;
  bi.sh = bi.s;
  if (g_fused_mode.load() && ni == 1 &&
      (d2 ? rb_fused_fits<2>(nbb) : rb_fused_fits<3>(nbb)) &&
      launch_bicgstab_rb_fused(pk, L, wr, b, x, rtol, maxiter, bi, w, pre_status, hks, s,
                               rtol_inst) == TCAD_OK)
    return TCAD_OK;
  TCAD_CUDA_CHECK(cudaMemsetAsync(w.ticket, 0, sizeof(unsigned) * ni, s));
  if (d2) k_rb_split<2><<<nbb, NT, 0, s>>>(pkb, L.mp, b, wr.bR, wr.bB, wr.bbf, w.partial, w.ticket);
  else    k_rb_split<3><<<nbb, NT, 0, s>>>(pkb, L.mp, b, wr.bR, wr.bB, wr.bbf, w.partial, w.ticket);
  note_launch();
  if (d2)
    k_rb_init<2><<<nbb, NT, 0, s>>>(pkb, L.mp, wr.JB, wr.bR, wr.bB, wr.rhs, wr.xb, bi, wr.bbf,
                                    w.ks, w.partial, w.ticket, rtol, maxiter, pre_status,
                                    rtol_inst);
  else
    k_rb_init<3><<<nbb, NT, 0, s>>>(pkb, L.mp, wr.JB, wr.bR, wr.bB, wr.rhs, wr.xb, bi, wr.bbf,
                                    w.ks, w.partial, w.ticket, rtol, maxiter, pre_status,
                                    rtol_inst);
  note_launch();
  TCAD_LAUNCH_CHECK();
  hks.resize(ni);
  int check = 4, done_iters = 0, rechecks = 0;
  ActiveGrid grid;
  if (int rc = grid.init(&pkb, s, &L.hfoff)) return rc;
  for (;;) {
    const unsigned ng = grid.ng;
    const int32_t* dlist = grid.dlist;
    for (int q = 0; q < check; ++q) {
      k_bi_p<<<ng, NT, 0, s>>>(pkb, bi, w.ks, dlist);
      if (d2) {
        k_rb_red<2><<<ng, NT, 0, s>>>(pkb, L.mp, wr.JR, bi.p, wr.tR, w.ks, dlist);
        k_rb_v<2><<<ng, NT, 0, s>>>(pkb, L.mp, wr.JB, wr.tR, bi, w.ks, w.partial, w.ticket,
                                    dlist);
      } else {
        k_rb_red<3><<<ng, NT, 0, s>>>(pkb, L.mp, wr.JR, bi.p, wr.tR, w.ks, dlist);
        k_rb_v<3><<<ng, NT, 0, s>>>(pkb, L.mp, wr.JB, wr.tR, bi, w.ks, w.partial, w.ticket,
                                    dlist);
      }
      k_bi_s<<<ng, NT, 0, s>>>(pkb, bi, w.ks, w.partial, w.ticket, dlist);
      if (d2) {
        k_rb_red<2><<<ng, NT, 0, s>>>(pkb, L.mp, wr.JR, bi.s, wr.tR, w.ks, dlist);
        k_rb_t<2><<<ng, NT, 0, s>>>(pkb, L.mp, wr.JB, wr.tR, bi, w.ks, w.partial, w.ticket,
                                    dlist);
      } else {
        k_rb_red<3><<<ng, NT, 0, s>>>(pkb, L.mp, wr.JR, bi.s, wr.tR, w.ks, dlist);
        k_rb_t<3><<<ng, NT, 0, s>>>(pkb, L.mp, wr.JB, wr.tR, bi, w.ks, w.partial, w.ticket,
                                    dlist);
      }
      k_bi_x<<<ng, NT, 0, s>>>(pkb, wr.xb, bi, w.ks, w.partial, w.ticket, dlist);
      for (int l = 0; l < 7; ++l) note_launch();
    }
    TCAD_LAUNCH_CHECK();
    done_iters += check;
    TCAD_CUDA_CHECK(cudaMemcpyAsync(hks.data(), w.ks, sizeof(KState) * ni,
                                    cudaMemcpyDeviceToHost, s));
    TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
    bool any = false;
    for (int i = 0; i < ni; ++i) any = any || hks[i].active;
    if (any)
      if (int rc = grid.update(hks, wr.blk, s)) return rc;
    if (!any) {
      // true Schur residual (= the full residual); re-arm drifted instances
      const int rearm = rechecks < 8 ? 1 : 0;
      if (d2) {
        k_rb_red<2><<<nbb, NT, 0, s>>>(pkb, L.mp, wr.JR, wr.xb, wr.tR, nullptr, nullptr);
        k_rb_true<2><<<nbb, NT, 0, s>>>(pkb, L.mp, wr.JB, wr.tR, wr.rhs, wr.xb, bi.r, w.ks,
                                        w.partial, w.ticket, rearm);
      } else {
        k_rb_red<3><<<nbb, NT, 0, s>>>(pkb, L.mp, wr.JR, wr.xb, wr.tR, nullptr, nullptr);
        k_rb_true<3><<<nbb, NT, 0, s>>>(pkb, L.mp, wr.JB, wr.tR, wr.rhs, wr.xb, bi.r, w.ks,
                                        w.partial, w.ticket, rearm);
      }
      note_launch();
      note_launch();
      TCAD_LAUNCH_CHECK();
      TCAD_CUDA_CHECK(cudaMemcpyAsync(hks.data(), w.ks, sizeof(KState) * ni,
                                      cudaMemcpyDeviceToHost, s));
      TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
      for (int i = 0; i < ni; ++i) any = any || hks[i].active;
      ++rechecks;
      if (!any) break;
      if (int rc = grid.update(hks, wr.blk, s)) return rc;
    }
    if (done_iters > 64) check = 16;
    if (done_iters > 1024) check = 32;
  }
  // x_r = b_r - E x_b (tR from the last true-residual pass holds E x_b)
  if (d2) k_rb_merge<2><<<nbb, NT, 0, s>>>(pkb, L.mp, wr.bR, wr.tR, wr.xb, x, pre_status);
  else    k_rb_merge<3><<<nbb, NT, 0, s>>>(pkb, L.mp, wr.bR, wr.tR, wr.xb, x, pre_status);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

static int launch_bicgstab(const tcad_pack_t* pk, const double* J, const double* b,
                           double* x, double rtol, int maxiter, const Work& w,
                           const int32_t* pre_status, std::vector<KState>& hks,
                           cudaStream_t s, const double* rtol_inst = nullptr,
                           const WorkIlu* ilu = nullptr, int nzmax = 1) {
  if (ilu && ilu->Q) {
    BiVec bi = w.bi;
    bi.ph = ilu->ph;
    bi.sh = ilu->sh;
    return launch_bicgstab_t<double>(pk, J, b, x, rtol, maxiter, bi, w, pre_status, hks, s,
                                     rtol_inst, J, ilu->Q, ilu->mask, nzmax, ilu);
  }
  return launch_bicgstab_t<double>(pk, J, b, x, rtol, maxiter, w.bi, w, pre_status, hks, s,
                                   rtol_inst);
}

// FP64 iterative refinement of A^ x = b (both FP64) with FP32 BiCGStab inner
// solves on the FP32 copy of A^: per instance, stop when the FP64 residual is
// within eta[i] ||b|| (instances whose pre_status is not OK stay idle).  Inner
// tolerance max(1e-4, min(0.5, eta / current relative residual)).  Returns the
// summed inner iterations, final relative residuals and statuses in res_*.
static int solve_mixed(const tcad_pack_t* pk, const double* J, const double* b, double* x,
                       const double* eta, int inner_maxiter, int max_ir, const Work& w,
                       const Work32& w32, const int32_t* pre_status_host,
                       std::vector<KState>& hks, int32_t* res_iters, int32_t* res_status,
                       double* res_relres, cudaStream_t s, const int32_t* fl = nullptr,
                       unsigned nfl = 0) {
  const unsigned nb = (unsigned)pk->n_flat;
  const int ni = pk->n_inst;
  const int ne = pk->dim == 2 ? TCAD_NE2 : TCAD_NE3;
  k_to_f32<<<fl ? nfl : nb, NT, 0, s>>>(*pk, ne, J, w32.J32, fl);
  note_launch();
  TCAD_CUDA_CHECK(cudaMemsetAsync(w.ticket, 0, sizeof(unsigned) * ni, s));
  k_ir_init<<<nb, NT, 0, s>>>(*pk, b, x, w32.irs, w.partial, w.ticket);
  note_launch();
  TCAD_LAUNCH_CHECK();
  std::vector<KState> irs(ni);
  std::vector<int32_t> pre(ni);
  std::vector<double> eta_in(ni);
  if ((int)hks.size() < ni) hks.resize(ni);
  for (int i = 0; i < ni; ++i) {
    res_iters[i] = 0;
    res_status[i] = pre_status_host[i];
    res_relres[i] = 1.0;
  }
  for (int ir = 0;; ++ir) {
    TCAD_CUDA_CHECK(cudaMemcpyAsync(irs.data(), w32.irs, sizeof(KState) * ni,
                                    cudaMemcpyDeviceToHost, s));
    TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
    bool any = false;
    for (int i = 0; i < ni; ++i) {
      if (pre_status_host[i] != TCAD_OK) { pre[i] = -1; continue; }
      const double rel = irs[i].bb > 0.0 ? std::sqrt(irs[i].rr / irs[i].bb) : 0.0;
      res_relres[i] = rel;
      const bool done = !(rel > eta[i]) || res_status[i] == TCAD_ERR_NONFINITE ||
                        res_status[i] == TCAD_ERR_BREAKDOWN || !std::isfinite(rel);
      if (!done && ir >= max_ir) { res_status[i] = TCAD_ERR_NOCONV; pre[i] = -1; continue; }
      if (!done) res_status[i] = TCAD_OK;
      pre[i] = done ? -1 : TCAD_OK;
      eta_in[i] = std::max(1e-4, std::min(0.5, eta[i] / std::max(rel, 1e-300)));
      any = any || !done;
    }
    if (!any) break;
    TCAD_CUDA_CHECK(cudaMemcpyAsync(w32.pre, pre.data(), sizeof(int32_t) * ni,
                                    cudaMemcpyHostToDevice, s));
    TCAD_CUDA_CHECK(cudaMemcpyAsync(w32.eta_in, eta_in.data(), sizeof(double) * ni,
                                    cudaMemcpyHostToDevice, s));
    // the FP64 residual lives in the (idle) first FP64 Krylov vector
    k_ir_scale<<<nb, NT, 0, s>>>(*pk, ir == 0 ? b : w.bi.r, w32.r32, w32.irs, w32.pre);
    note_launch();
    int rc = launch_bicgstab_t<float>(pk, w32.J32, w32.r32, w32.d32, 1e-4, inner_maxiter,
                                      w32.bi, w, w32.pre, hks, s, w32.eta_in);
    if (rc != TCAD_OK) return rc;
    for (int i = 0; i < ni; ++i) {
      if (pre[i] != TCAD_OK) continue;
      res_iters[i] += hks[i].it;
      if (hks[i].status == TCAD_ERR_NONFINITE || hks[i].status == TCAD_ERR_BREAKDOWN)
        res_status[i] = hks[i].status;
    }
    k_ir_axpy<<<nb, NT, 0, s>>>(*pk, x, w32.d32, w32.irs, w32.pre);
    note_launch();
    if (pk->dim == 2)
      k_ir_resid<2><<<nb, NT, 0, s>>>(*pk, J, b, x, w.bi.r, w32.irs, w32.pre, w.partial,
                                      w.ticket);
    else
      k_ir_resid<3><<<nb, NT, 0, s>>>(*pk, J, b, x, w.bi.r, w32.irs, w32.pre, w.partial,
                                      w.ticket);
    note_launch();
    TCAD_LAUNCH_CHECK();
  }
  return TCAD_OK;
}

static int launch_cg(const tcad_pack_t* pk, const double* J, const double* b, double* x,
                     double rtol, int maxiter, const Work& w, const uint8_t* active,
                     std::vector<KState>& hks, cudaStream_t s,
                     const double* rtol_inst = nullptr) {
  const unsigned nb = (unsigned)pk->n_flat;
  const int ni = pk->n_inst;
  TCAD_CUDA_CHECK(cudaMemsetAsync(w.ticket, 0, sizeof(unsigned) * ni, s));
  k_cg_init<<<nb, NT, 0, s>>>(*pk, J, b, x, w.cg, w.ks, w.partial, w.ticket, rtol, maxiter,
                              active, rtol_inst);
  note_launch();
  TCAD_LAUNCH_CHECK();
  hks.resize(ni);
  int check = 8;
  int done_iters = 0;
  // a batch's stragglers (the graded-mesh devices of a serving round can
  // need tens of thousands of iterations) launch only their own blocks
  ActiveGrid grid;
  if (int rc = grid.init(pk, s, nullptr)) return rc;
  for (;;) {
    const unsigned ng = grid.ng;
    const int32_t* dlist = grid.dlist;
    for (int q = 0; q < check; ++q) {
      if (pk->dim == 2)
        k_cg_q<2><<<ng, NT, 0, s>>>(*pk, J, w.cg, w.ks, w.partial, w.ticket, dlist);
      else
        k_cg_q<3><<<ng, NT, 0, s>>>(*pk, J, w.cg, w.ks, w.partial, w.ticket, dlist);
      note_launch();
      k_cg_x<<<ng, NT, 0, s>>>(*pk, J, x, w.cg, w.ks, w.partial, w.ticket, dlist);
      note_launch();
      k_cg_p<<<ng, NT, 0, s>>>(*pk, w.cg, w.ks, dlist);
      note_launch();
    }
    TCAD_LAUNCH_CHECK();
    done_iters += check;
    TCAD_CUDA_CHECK(cudaMemcpyAsync(hks.data(), w.ks, sizeof(KState) * ni,
                                    cudaMemcpyDeviceToHost, s));
    TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
    bool any = false;
    for (int i = 0; i < ni; ++i) any = any || hks[i].active;
    if (!any) break;
    if (int rc = grid.update(hks, w.blk, s)) return rc;
    if (done_iters > 64) check = 32;
  }
  return TCAD_OK;
}

// Equilibrium PCG on the red-black Schur complement (k_eqrb_*): the same
// per-instance loop, masks and compaction as launch_cg, on the black slots;
// d is the full update.  L: the slot pack (rb_layout over we's tables).
static int launch_cg_rb(const tcad_pack_t* pk, const RbLayout& L, const WorkEq& we,
                        const double* J, const double* b, double* d, double rtol,
                        int maxiter, const Work& w, const uint8_t* active,
                        std::vector<KState>& hks, cudaStream_t s,
                        const double* rtol_inst = nullptr) {
  const tcad_pack_t& pkb = L.pkb;
  const unsigned nbb = (unsigned)pkb.n_flat;
  const int ni = pk->n_inst;
  const bool d2 = pk->dim == 2;
  CgVec cg = w.cg;   // black slot vectors
  TCAD_CUDA_CHECK(cudaMemsetAsync(w.ticket, 0, sizeof(unsigned) * ni, s));
  TCAD_CUDA_CHECK(cudaMemsetAsync(we.xb, 0, sizeof(double) * (size_t)pkb.n_nodes, s));
  if (d2) {
    k_eqrb_pack<2><<<nbb, NT, 0, s>>>(pkb, L.mp, J, b, we.JRe, we.JBe, we.bR, we.bB);
    k_eqrb_diag<2><<<nbb, NT, 0, s>>>(pkb, L.mp, we.JRe, we.JBe, we.Sinv);
    k_eqrb_red<2><<<nbb, NT, 0, s>>>(pkb, L.mp, we.JRe, we.xb, we.bR, we.tR, nullptr, nullptr);
    k_eqrb_init<2><<<nbb, NT, 0, s>>>(pkb, L.mp, we.JBe, we.bB, we.tR, we.Sinv, we.xb, cg,
                                      w.ks, w.partial, w.ticket, rtol, maxiter, active,
                                      rtol_inst);
  } else {
    k_eqrb_pack<3><<<nbb, NT, 0, s>>>(pkb, L.mp, J, b, we.JRe, we.JBe, we.bR, we.bB);
    k_eqrb_diag<3><<<nbb, NT, 0, s>>>(pkb, L.mp, we.JRe, we.JBe, we.Sinv);
    k_eqrb_red<3><<<nbb, NT, 0, s>>>(pkb, L.mp, we.JRe, we.xb, we.bR, we.tR, nullptr, nullptr);
    k_eqrb_init<3><<<nbb, NT, 0, s>>>(pkb, L.mp, we.JBe, we.bB, we.tR, we.Sinv, we.xb, cg,
                                      w.ks, w.partial, w.ticket, rtol, maxiter, active,
                                      rtol_inst);
  }
  for (int l = 0; l < 4; ++l) note_launch();
  TCAD_LAUNCH_CHECK();
  hks.resize(ni);
  int check = 8;
  int done_iters = 0;
  ActiveGrid grid;
  if (int rc = grid.init(&pkb, s, &L.hfoff)) return rc;
  for (;;) {
    const unsigned ng = grid.ng;
    const int32_t* dlist = grid.dlist;
    for (int q = 0; q < check; ++q) {
      if (d2) {
        k_eqrb_red<2><<<ng, NT, 0, s>>>(pkb, L.mp, we.JRe, cg.p, nullptr, we.tR, w.ks, dlist);
        k_eqrb_q<2><<<ng, NT, 0, s>>>(pkb, L.mp, we.JBe, we.tR, cg, w.ks, w.partial, w.ticket,
                                      dlist);
      } else {
        k_eqrb_red<3><<<ng, NT, 0, s>>>(pkb, L.mp, we.JRe, cg.p, nullptr, we.tR, w.ks, dlist);
        k_eqrb_q<3><<<ng, NT, 0, s>>>(pkb, L.mp, we.JBe, we.tR, cg, w.ks, w.partial, w.ticket,
                                      dlist);
      }
      k_eqrb_x<<<ng, NT, 0, s>>>(pkb, we.Sinv, we.xb, cg, w.ks, w.partial, w.ticket, dlist);
      k_cg_p<<<ng, NT, 0, s>>>(pkb, cg, w.ks, dlist);
      for (int l = 0; l < 4; ++l) note_launch();
    }
    TCAD_LAUNCH_CHECK();
    done_iters += check;
    TCAD_CUDA_CHECK(cudaMemcpyAsync(hks.data(), w.ks, sizeof(KState) * ni,
                                    cudaMemcpyDeviceToHost, s));
    TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
    bool any = false;
    for (int i = 0; i < ni; ++i) any = any || hks[i].active;
    if (!any) break;
    if (int rc = grid.update(hks, we.blk, s)) return rc;
    if (done_iters > 64) check = 32;
  }
  // d_r = A_rr^-1 (F_r - A_rb d_b), then the full update
  if (d2) {
    k_eqrb_red<2><<<nbb, NT, 0, s>>>(pkb, L.mp, we.JRe, we.xb, we.bR, we.tR, nullptr, nullptr);
    k_eqrb_merge<2><<<nbb, NT, 0, s>>>(pkb, L.mp, we.tR, we.xb, d);
  } else {
    k_eqrb_red<3><<<nbb, NT, 0, s>>>(pkb, L.mp, we.JRe, we.xb, we.bR, we.tR, nullptr, nullptr);
    k_eqrb_merge<3><<<nbb, NT, 0, s>>>(pkb, L.mp, we.tR, we.xb, d);
  }
  note_launch();
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

}  // namespace tcad

using namespace tcad;

extern "C" int tcad_set_krylov_fused_test(int hold) {
  return g_fused_test_hold.exchange(hold ? 1 : 0);
}

extern "C" uint64_t tcad_krylov_fused_gave_up(void) { return g_fused_gave_up.load(); }

extern "C" int tcad_set_krylov_fused(int on) {
  return g_fused_mode.exchange(on ? 1 : 0);
}

// offsets of the workspace's extensions: FP64 work, then the FP32 extension,
// the ILU(0) extension, the equilibrium red-black extension and the
// red-black Schur extension of the coupled solves
static size_t rnd256(size_t b) { return (b + 255) & ~(size_t)255; }
static size_t off_w32(const tcad_pack_t* pk) { return rnd256(carve(pk, nullptr, 0).bytes); }
static size_t off_ilu(const tcad_pack_t* pk) {
  return off_w32(pk) + rnd256(carve32(pk, nullptr).bytes);
}
static size_t off_eq(const tcad_pack_t* pk) {
  return off_ilu(pk) + rnd256(carve_ilu(pk, nullptr).bytes);
}
static size_t off_rb(const tcad_pack_t* pk) {
  return off_eq(pk) + rnd256(carve_eq(pk, nullptr).bytes);
}

extern "C" size_t tcad_block_workspace_bytes(const tcad_pack_t* pk, int method, int restart) {
  if (!pk) return 0;
  (void)restart;
  // the red-black extension (two colour copies of J and five slot vectors,
  // about as much again as J) only for method 2
  return off_rb(pk) + (method == 2 ? carve_rb(pk, nullptr).bytes : 0) + 512;
}

extern "C" int tcad_block_jacobi_setup(const tcad_pack_t* pk, double* J, double* F,
                                       int32_t* status, void* stream) {
  if (!pack_ok(pk) || !J || !F || !status) return TCAD_ERR_ARG;
  if (pk->dim == 2)
    k_bj_setup<2><<<(unsigned)pk->n_flat, NT, 0, (cudaStream_t)stream>>>(*pk, J, F, status,
                                                                         nullptr, nullptr, 0.0,
                                                                         nullptr);
  else
    k_bj_setup<3><<<(unsigned)pk->n_flat, NT, 0, (cudaStream_t)stream>>>(*pk, J, F, status,
                                                                         nullptr, nullptr, 0.0,
                                                                         nullptr);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

extern "C" int tcad_block_jacobi_setup_rel(const tcad_pack_t* pk, double* J, double* F,
                                           int32_t* status, const double* n, const double* p,
                                           double dens_floor, void* stream) {
  if (!pack_ok(pk) || !J || !F || !status || !n || !p || !(dens_floor > 0.0))
    return TCAD_ERR_ARG;
  if (pk->dim == 2)
    k_bj_setup<2><<<(unsigned)pk->n_flat, NT, 0, (cudaStream_t)stream>>>(*pk, J, F, status, n,
                                                                         p, dens_floor, nullptr);
  else
    k_bj_setup<3><<<(unsigned)pk->n_flat, NT, 0, (cudaStream_t)stream>>>(*pk, J, F, status, n,
                                                                         p, dens_floor, nullptr);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

extern "C" size_t tcad_block_ilu_bytes(const tcad_pack_t* pk) {
  if (!pack_ok(pk)) return 0;
  return 9 * sizeof(double) * (size_t)pk->n_nodes;
}

// largest shorter side min(Nx, Ny) of the pack's instances (host read)
static int pack_max_short_side(const tcad_pack_t* pk, cudaStream_t s) {
  if (pk->n_inst < 1) return 0;
  std::vector<int32_t> shp(3 * (size_t)pk->n_inst);
  if (cudaMemcpyAsync(shp.data(), pk->shape, sizeof(int32_t) * shp.size(),
                      cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return 1 << 30;
  int m = 0;
  for (int i = 0; i < pk->n_inst; ++i) m = std::max(m, std::min((int)shp[3 * i], (int)shp[3 * i + 1]));
  return m;
}

// largest Nz of the pack's instances (host read of the shape table)
static int pack_nzmax(const tcad_pack_t* pk, cudaStream_t s) {
  if (pk->dim == 2 || pk->n_inst < 1) return 1;
  std::vector<int32_t> shp(3 * (size_t)pk->n_inst);
  if (cudaMemcpyAsync(shp.data(), pk->shape, sizeof(int32_t) * shp.size(),
                      cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return -1;
  int m = 1;
  for (int i = 0; i < pk->n_inst; ++i) m = std::max(m, (int)shp[3 * i + 2]);
  return m;
}

extern "C" int tcad_block_ilu_setup(const tcad_pack_t* pk, const double* J, double* Q,
                                    int32_t* status, void* stream) {
  if (!pack_ok(pk) || !J || !Q || !status) return TCAD_ERR_ARG;
  if (pk->n_inst < 1) return TCAD_OK;
  const int nzm = pack_nzmax(pk, (cudaStream_t)stream);
  if (nzm < 1) return TCAD_ERR_CUDA;
  k_ilu2d_factor<<<(unsigned)(pk->n_inst * nzm), kIluThreads, 0, (cudaStream_t)stream>>>(
      *pk, J, Q, nullptr, status, nzm, nullptr, nullptr);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

extern "C" int tcad_block_ilu_apply(const tcad_pack_t* pk, const double* J, const double* Q,
                                    const double* r, double* out, void* stream) {
  if (!pack_ok(pk) || !J || !Q || !r || !out || r == out) return TCAD_ERR_ARG;
  if (pk->n_inst < 1) return TCAD_OK;
  const int nzm = pack_nzmax(pk, (cudaStream_t)stream);
  if (nzm < 1) return TCAD_ERR_CUDA;
  k_ilu2d_apply<double><<<(unsigned)(pk->n_inst * nzm), kIluThreads, 0,
                          (cudaStream_t)stream>>>(*pk, J, Q, r, out, nullptr, nullptr, nzm);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

extern "C" int tcad_block_spmv(const tcad_pack_t* pk, const double* J, const double* x,
                               double* y, void* stream) {
  if (!pack_ok(pk)) return TCAD_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (pk->dim == 2)
    k_spmv<2, true><<<(unsigned)pk->n_flat, NT, 0, s>>>(*pk, J, x, y);
  else
    k_spmv<3, true><<<(unsigned)pk->n_flat, NT, 0, s>>>(*pk, J, x, y);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

extern "C" int tcad_block_krylov(const tcad_pack_t* pk, const double* J, const double* b,
                                 double* x, int method, double rtol, int maxiter,
                                 int restart, void* work, size_t work_bytes, int32_t* iters,
                                 int32_t* status, double* relres, void* stream) {
  if (!pack_ok(pk) || !work) return TCAD_ERR_ARG;
  if (method != 0 && method != 2) return TCAD_ERR_ARG;  // GMRES: the CSR entry point
  (void)restart;
  Work w = carve(pk, work, work_bytes);
  if (w.bytes > work_bytes) return TCAD_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<KState> hks;
  int rc;
  if (method == 2) {
    if (work_bytes < tcad_block_workspace_bytes(pk, 2, 0)) return TCAD_ERR_ARG;
    const WorkRb wrb = carve_rb(pk, reinterpret_cast<char*>(work) + off_rb(pk));
    RbLayout rbl;
    if ((rc = rb_layout(pk, wrb, rbl, s)) != TCAD_OK) return rc;
    const unsigned nbb = (unsigned)rbl.pkb.n_flat;
    if (pk->dim == 2)
      k_rb_pack<2><<<nbb, NT, 0, s>>>(rbl.pkb, rbl.mp, J, wrb.JR, wrb.JB);
    else
      k_rb_pack<3><<<nbb, NT, 0, s>>>(rbl.pkb, rbl.mp, J, wrb.JR, wrb.JB);
    note_launch();
    TCAD_LAUNCH_CHECK();
    rc = launch_bicgstab_rb(pk, rbl, wrb, b, x, rtol, maxiter, w, nullptr, hks, s, nullptr);
  } else {
    rc = launch_bicgstab(pk, J, b, x, rtol, maxiter, w, nullptr, hks, s);
  }
  if (rc != TCAD_OK) return rc;
  for (int i = 0; i < pk->n_inst; ++i) {
    if (iters) iters[i] = hks[i].it;
    if (status) status[i] = hks[i].status;
    if (relres) relres[i] = hks[i].bb > 0.0 ? std::sqrt(hks[i].rr / hks[i].bb) : 0.0;
  }
  return TCAD_OK;
}

extern "C" int tcad_newton_update(const tcad_pack_t* pk, double* psi, double* n, double* p,
                                  const double* du, double max_dpsi, double dens_floor,
                                  const uint8_t* active, double* partial, double* err,
                                  void* stream) {
  if (!pack_ok(pk)) return TCAD_ERR_ARG;
  (void)partial;
  cudaStream_t s = (cudaStream_t)stream;
  TCAD_CUDA_CHECK(cudaMemsetAsync(err, 0, sizeof(double) * pk->n_inst, s));
  k_newton_update<<<(unsigned)pk->n_flat, NT, 0, s>>>(
      *pk, psi, n, p, du, max_dpsi, dens_floor, active,
      reinterpret_cast<unsigned long long*>(err), 0, 0, dens_floor);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

extern "C" int tcad_newton_solve(const tcad_pack_t* pk, double* psi, double* n, double* p,
                                 double* F, double* J, double* du,
                                 const tcad_newton_opts_t* opts, uint8_t* active,
                                 void* work, size_t work_bytes,
                                 tcad_newton_result_t* result, void* stream) {
  if (!pack_ok(pk) || !opts || !active || !result || !work) return TCAD_ERR_ARG;
  if (opts->method != 0) return TCAD_ERR_ARG;
  Work w = carve(pk, work, work_bytes);
  if (w.bytes > work_bytes) return TCAD_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int ni = pk->n_inst;
  const unsigned nb = (unsigned)pk->n_flat;
  std::vector<uint8_t> hact(ni);
  TCAD_CUDA_CHECK(cudaMemcpyAsync(hact.data(), active, ni, cudaMemcpyDeviceToHost, s));
  TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
  for (int i = 0; i < ni; ++i) {
    result[i].iters = 0; result[i].converged = 0; result[i].krylov_iters = 0;
    result[i].status = TCAD_OK; result[i].err = INFINITY; result[i].relres = 0.0;
    result[i].fp64_from = -1; result[i].polish_iters = 0;
  }
  std::vector<KState> hks(ni);  // sized up front: a solve may end before any inner launch
  std::vector<unsigned long long> herr(ni);
  std::vector<int32_t> hstat(ni);
  std::vector<int> polish_left(ni, -1);  // -1: not yet converged
  if (opts->precision != 64 && opts->precision != 32 && opts->precision != TCAD_PRECISION_J32)
    return TCAD_ERR_ARG;
  if (opts->precision != 64 && work_bytes < tcad_block_workspace_bytes(pk, 0, 0))
    return TCAD_ERR_ARG;
  const Work32 w32 = carve32(pk, reinterpret_cast<char*>(work) + ((w.bytes + 255) & ~(size_t)255));
  // ILU(0) right preconditioner (2D): its region follows the FP32 extension.
  // precond 1: every instance; 2 (automatic): the instances of a batch
  // (more than one), and any instance whose node-block-Jacobi solve fails
  const bool use_ilu = opts->precond == 1 || (opts->precond == 2 && pk->dim == 2);
  std::vector<uint8_t> ilu_on(ni, 0);
  const int nzmax = use_ilu ? pack_nzmax(pk, s) : 1;
  if (nzmax < 1) return TCAD_ERR_CUDA;
  if (use_ilu)
    for (int i = 0; i < ni; ++i) ilu_on[i] = (opts->precond == 1 || ni > 1) ? 1 : 0;
  if (use_ilu && work_bytes < tcad_block_workspace_bytes(pk, 0, 0)) return TCAD_ERR_ARG;
  const WorkIlu wilu = use_ilu ? carve_ilu(pk, reinterpret_cast<char*>(work) +
                                                   ((w.bytes + 255) & ~(size_t)255) +
                                                   ((w32.bytes + 255) & ~(size_t)255))
                               : WorkIlu{nullptr, nullptr, nullptr, nullptr, nullptr,
                                         nullptr, nullptr, nullptr, nullptr, 0};
  WorkIlu wilu_use = wilu;
  if (use_ilu && (pk->dim != 2 || pack_max_short_side(pk, s) > kIluThreads)) {
    wilu_use.Mf = nullptr;  // node-order sweeps
    wilu_use.Mb = nullptr;
  }
  // red-black Schur solves: the slot pack's tables, once per call (a
  // single-instance pack small enough is solved in one cooperative launch,
  // k_bicgstab_rb_fused, by launch_bicgstab_rb itself)
  // (a workspace sized without the red-black extension -- method 0 -- solves
  // the whole system)
  const bool use_rb = opts->red_black != 0 && work_bytes >= tcad_block_workspace_bytes(pk, 2, 0);
  WorkRb wrb{};
  RbLayout rbl;
  if (use_rb) {
    wrb = carve_rb(pk, reinterpret_cast<char*>(work) + off_rb(pk));
    if (int rc = rb_layout(pk, wrb, rbl, s)) return rc;
  }
  std::vector<int32_t> mix_it(ni), mix_st(ni), mix_grew(ni, 0), mix_steps(ni, 0);
  std::vector<double> mix_rr(ni), mix_prev(ni, -1.0);
  std::vector<uint8_t> use64(ni, 0);  // precision 32: instances switched to FP64
  std::vector<int32_t> last_kit(ni, 0);
  std::vector<double> heta(ni, opts->forcing ? std::max(opts->eta_max, opts->rtol) : opts->rtol);
  const double sfloor = opts->scale_floor > 0.0 ? opts->scale_floor : opts->dens_floor;
  std::vector<double> hsfl(ni, sfloor);
  const double eta_lo = std::max(opts->rtol, opts->eta_min);
  // Per-step launch lists: once the instances still iterating cover under
  // 3/4 of the pack, the assembly and the block-Jacobi set-up cover only
  // their tiles / flat blocks (rebuilt when that set changes).
  std::vector<int64_t> hfoff;
  std::vector<int32_t> htile_inst, lt, lf;
  std::vector<uint8_t> listed;
  const int32_t* tl = nullptr;
  const int32_t* fl = nullptr;
  int64_t ntl = 0, nfl = 0;
  if (ni > 1) {
    hfoff.resize(ni + 1);
    std::vector<int32_t> htile(4 * (size_t)pk->n_tiles);
    TCAD_CUDA_CHECK(cudaMemcpyAsync(hfoff.data(), pk->flat_off, sizeof(int64_t) * (ni + 1),
                                    cudaMemcpyDeviceToHost, s));
    TCAD_CUDA_CHECK(cudaMemcpyAsync(htile.data(), pk->tile, sizeof(int32_t) * htile.size(),
                                    cudaMemcpyDeviceToHost, s));
    TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
    htile_inst.resize(pk->n_tiles);
    for (int64_t t = 0; t < pk->n_tiles; ++t) htile_inst[t] = htile[4 * t];
    listed.assign(ni, 2);  // forces a first decision
  }
  for (int it = 0; it < opts->max_iter; ++it) {
    if (ni > 1 && listed != hact) {
      listed = hact;
      int64_t act_blocks = 0;
      for (int i = 0; i < ni; ++i)
        if (hact[i]) act_blocks += hfoff[i + 1] - hfoff[i];
      if (4 * act_blocks < 3 * (int64_t)nb) {
        lt.clear();
        lf.clear();
        for (int64_t t = 0; t < pk->n_tiles; ++t)
          if (hact[htile_inst[t]]) lt.push_back((int32_t)t);
        for (int i = 0; i < ni; ++i)
          if (hact[i])
            for (int64_t b = hfoff[i]; b < hfoff[i + 1]; ++b) lf.push_back((int32_t)b);
        if (!lt.empty())
          TCAD_CUDA_CHECK(cudaMemcpyAsync(w.tl, lt.data(), sizeof(int32_t) * lt.size(),
                                          cudaMemcpyHostToDevice, s));
        if (!lf.empty())
          TCAD_CUDA_CHECK(cudaMemcpyAsync(w.fl, lf.data(), sizeof(int32_t) * lf.size(),
                                          cudaMemcpyHostToDevice, s));
        tl = w.tl; ntl = (int64_t)lt.size();
        fl = w.fl; nfl = (int64_t)lf.size();
      } else {
        tl = nullptr; fl = nullptr; ntl = 0; nfl = 0;
      }
    }
    int rc = sg_assemble_tiles(pk, psi, n, p, F, J, TCAD_MODE_ELIMINATE, tl, ntl, s);
    if (rc != TCAD_OK) return rc;
    if (opts->dt > 0.0) {  // one step of the theta scheme: storage term
      rc = storage_terms(pk, n, p, opts->n_old, opts->p_old, opts->fn_old, opts->fp_old,
                         opts->dt, opts->theta, F, J, fl, nfl, s);
      if (rc != TCAD_OK) return rc;
    }
    TCAD_CUDA_CHECK(cudaMemsetAsync(w.status, 0, sizeof(int32_t) * ni, s));
    // density floor of each instance's relative unknowns: the polishing
    // steps use their own (far below the densities), the others sfloor
    for (int i = 0; i < ni; ++i)
      hsfl[i] = (polish_left[i] > 0 && opts->polish_scale_floor > 0.0)
                    ? opts->polish_scale_floor : sfloor;
    TCAD_CUDA_CHECK(cudaMemcpyAsync(w.sfl, hsfl.data(), sizeof(double) * ni,
                                    cudaMemcpyHostToDevice, s));
    if (!fl || nfl > 0) {
      const bool rel = opts->density_scaling != 0;
      const double* sn_ = rel ? n : nullptr;
      const double* sp_ = rel ? p : nullptr;
      const unsigned g = fl ? (unsigned)nfl : nb;
      if (pk->dim == 2)
        k_bj_setup<2><<<g, NT, 0, s>>>(*pk, J, F, w.status, sn_, sp_, sfloor, fl, w.sfl);
      else
        k_bj_setup<3><<<g, NT, 0, s>>>(*pk, J, F, w.status, sn_, sp_, sfloor, fl, w.sfl);
    }
    note_launch();
    TCAD_LAUNCH_CHECK();
    // inactive instances: pre-mark so their Krylov stays idle
    TCAD_CUDA_CHECK(cudaMemcpyAsync(hstat.data(), w.status, sizeof(int32_t) * ni,
                                    cudaMemcpyDeviceToHost, s));
    TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
    for (int i = 0; i < ni; ++i)
      if (!hact[i] && hstat[i] == TCAD_OK) hstat[i] = -1;  // idle marker
    TCAD_CUDA_CHECK(cudaMemcpyAsync(w.status, hstat.data(), sizeof(int32_t) * ni,
                                    cudaMemcpyHostToDevice, s));
    TCAD_CUDA_CHECK(cudaMemcpyAsync(w.eta, heta.data(), sizeof(double) * ni,
                                    cudaMemcpyHostToDevice, s));
    // instances whose step is solved in FP64 this iteration, and those whose
    // (FP32-solved) step is applied before the FP64 solve starts
    std::vector<uint8_t> grp64(ni, 0), grp32(ni, 0);
    for (int i = 0; i < ni; ++i) {
      if (!hact[i]) continue;
      if (opts->precision == 32 && !use64[i] && hstat[i] == TCAD_OK) grp32[i] = 1;
      else grp64[i] = 1;  // includes failed block set-ups: their update is zero
    }
    bool any32 = false, any64 = false;
    for (int i = 0; i < ni; ++i) { any32 = any32 || grp32[i]; }
    TCAD_CUDA_CHECK(cudaMemsetAsync(w.err, 0, sizeof(unsigned long long) * ni, s));
    if (any32) {
      // FP32 inner Krylov inside FP64 iterative refinement
      std::vector<int32_t> st32(ni);
      for (int i = 0; i < ni; ++i) st32[i] = grp32[i] ? TCAD_OK : -1;
      rc = solve_mixed(pk, J, F, du, heta.data(), opts->krylov_maxiter, 30, w, w32,
                       st32.data(), hks, mix_it.data(), mix_st.data(), mix_rr.data(), s, fl,
                       (unsigned)nfl);
      if (rc != TCAD_OK) return rc;
      // Acceptance test before the step is applied (a dry-run update): an
      // FP32-solved step is rejected when its refinement failed (breakdown,
      // no convergence), when the update is non-finite, when it hits the
      // 10x density clip, when the update norm grew on two mixed steps in a
      // row, or when the instance has taken max_iter/3 mixed steps without
      // converging.  A rejected instance re-solves this step in FP64 and
      // stays in FP64 for the rest of the call.
      TCAD_CUDA_CHECK(cudaMemcpyAsync(active, grp32.data(), ni, cudaMemcpyHostToDevice, s));
      k_newton_update<<<nb, NT, 0, s>>>(*pk, psi, n, p, du, opts->max_dpsi, opts->dens_floor,
                                        active, w.err, opts->density_scaling, 1, sfloor,
                                        w.sfl);
      note_launch();
      TCAD_LAUNCH_CHECK();
      TCAD_CUDA_CHECK(cudaMemcpyAsync(herr.data(), w.err, sizeof(unsigned long long) * ni,
                                      cudaMemcpyDeviceToHost, s));
      TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
      TCAD_CUDA_CHECK(cudaMemsetAsync(w.err, 0, sizeof(unsigned long long) * ni, s));
      bool acc_any = false;
      for (int i = 0; i < ni; ++i) {
        if (!grp32[i]) continue;
        double e;
        std::memcpy(&e, &herr[i], sizeof(double));
        const bool grew = mix_prev[i] >= 0.0 && e >= mix_prev[i];
        mix_grew[i] = grew ? mix_grew[i] + 1 : 0;
        ++mix_steps[i];
        const bool reject = mix_st[i] != TCAD_OK || !std::isfinite(e) || e >= 8.999 ||
                            mix_grew[i] >= 2 ||
                            mix_steps[i] > std::max(4, opts->max_iter / 3);
        mix_prev[i] = e;
        if (opts->verbose && reject)
          std::fprintf(stderr, "    [gpu] inst %d it %2d  fp32 step rejected (err=%.3e st=%d)"
                               " -> fp64\n", i, it, e, mix_st[i]);
        result[i].krylov_iters += mix_it[i];
        if (reject) {
          grp32[i] = 0;
          grp64[i] = 1;
          use64[i] = 1;
          result[i].fp64_from = it;
        } else {
          result[i].status = mix_st[i];
          result[i].relres = mix_rr[i];
          last_kit[i] = mix_it[i];
          acc_any = true;
        }
      }
      if (acc_any) {
        TCAD_CUDA_CHECK(cudaMemcpyAsync(active, grp32.data(), ni, cudaMemcpyHostToDevice, s));
        k_newton_update<<<nb, NT, 0, s>>>(*pk, psi, n, p, du, opts->max_dpsi,
                                          opts->dens_floor, active, w.err,
                                          opts->density_scaling, 0, sfloor, w.sfl);
        note_launch();
        TCAD_LAUNCH_CHECK();
      }
    }
    for (int i = 0; i < ni; ++i) { any64 = any64 || grp64[i]; }
    // FP64 BiCGStab for the FP64 group (the other instances stay idle); in
    // automatic preconditioning an instance whose node-block-Jacobi solve
    // failed is solved again with ILU(0) before its update is applied
    std::vector<uint8_t> solve_set(grp64), done_set(ni, 0);
    for (int pass = 0; pass < 2 && any64; ++pass) {
      std::vector<int32_t> st64(ni);
      bool any_ilu = false;
      for (int i = 0; i < ni; ++i) {
        st64[i] = solve_set[i] ? hstat[i] : -1;
        any_ilu = any_ilu || (solve_set[i] && ilu_on[i]);
      }
      TCAD_CUDA_CHECK(cudaMemcpyAsync(w.status, st64.data(), sizeof(int32_t) * ni,
                                      cudaMemcpyHostToDevice, s));
      if (any_ilu) {  // factor the ILU instances of this solve
        std::vector<int32_t> pre(ni);
        std::vector<uint8_t> msk(ni);
        for (int i = 0; i < ni; ++i) {
          msk[i] = (solve_set[i] && ilu_on[i]) ? 1 : 0;
          pre[i] = msk[i] ? st64[i] : -1;
        }
        TCAD_CUDA_CHECK(cudaMemcpyAsync(wilu.pre, pre.data(), sizeof(int32_t) * ni,
                                        cudaMemcpyHostToDevice, s));
        TCAD_CUDA_CHECK(cudaMemcpyAsync(wilu.mask, msk.data(), ni, cudaMemcpyHostToDevice, s));
        k_ilu2d_factor<<<(unsigned)(ni * nzmax), kIluThreads, 0, s>>>(
            *pk, J, wilu.Q, wilu.pre, nullptr, nzmax, wilu_use.Mf, wilu_use.Mb);
        note_launch();
        TCAD_LAUNCH_CHECK();
      }
      // precision 33: the Newton steps before the update test passes run the
      // FP64 BiCGStab on an FP32 copy of the scaled operator (half the
      // operator bytes); the polishing steps, and any solve with ILU(0),
      // keep the FP64 operator
      bool any_polish = false;
      for (int i = 0; i < ni; ++i) any_polish = any_polish || (solve_set[i] && polish_left[i] > 0);
      if (opts->precision == TCAD_PRECISION_J32 && !any_ilu && !any_polish) {
        const int ne = pk->dim == 2 ? TCAD_NE2 : TCAD_NE3;
        k_to_f32<<<fl ? (unsigned)nfl : nb, NT, 0, s>>>(*pk, ne, J, w32.J32, fl);
        note_launch();
        TCAD_LAUNCH_CHECK();
        rc = launch_bicgstab_t<double, float>(pk, w32.J32, F, du, opts->rtol,
                                              opts->krylov_maxiter, w.bi, w, w.status, hks, s,
                                              w.eta);
      } else if (use_rb && !any_ilu) {
        const unsigned nbb = (unsigned)rbl.pkb.n_flat;
        if (pk->dim == 2)
          k_rb_pack<2><<<nbb, NT, 0, s>>>(rbl.pkb, rbl.mp, J, wrb.JR, wrb.JB);
        else
          k_rb_pack<3><<<nbb, NT, 0, s>>>(rbl.pkb, rbl.mp, J, wrb.JR, wrb.JB);
        note_launch();
        TCAD_LAUNCH_CHECK();
        rc = launch_bicgstab_rb(pk, rbl, wrb, F, du, opts->rtol, opts->krylov_maxiter, w,
                                w.status, hks, s, w.eta);
      } else {
        rc = launch_bicgstab(pk, J, F, du, opts->rtol, opts->krylov_maxiter, w, w.status, hks,
                             s, w.eta, any_ilu ? &wilu_use : nullptr, nzmax);
      }
      if (rc != TCAD_OK) return rc;
      std::vector<uint8_t> apply(ni, 0), retry(ni, 0);
      bool any_retry = false;
      for (int i = 0; i < ni; ++i) {
        if (!solve_set[i]) continue;
        last_kit[i] = hks[i].it;
        result[i].krylov_iters += hks[i].it;
        result[i].status = hks[i].status;
        result[i].relres = hks[i].bb > 0.0 ? std::sqrt(hks[i].rr / hks[i].bb) : 0.0;
        const bool failed = hks[i].status == TCAD_ERR_NOCONV ||
                            hks[i].status == TCAD_ERR_BREAKDOWN;
        if (pass == 0 && failed && opts->precond == 2 && use_ilu && !ilu_on[i]) {
          ilu_on[i] = 1;  // from now on this instance is ILU-preconditioned
          retry[i] = 1;
          any_retry = true;
          if (opts->verbose)
            std::fprintf(stderr, "    [gpu] inst %d it %2d  block-Jacobi solve failed (st=%d)"
                                 " -> ILU(0)\n", i, it, hks[i].status);
        } else {
          apply[i] = 1;  // instances whose solve broke down keep the partial step
        }
      }
      // apply this pass's accepted steps (the retried ones are solved again;
      // their du is overwritten by the next pass)
      TCAD_CUDA_CHECK(cudaMemcpyAsync(active, apply.data(), ni, cudaMemcpyHostToDevice, s));
      k_newton_update<<<nb, NT, 0, s>>>(*pk, psi, n, p, du, opts->max_dpsi, opts->dens_floor,
                                        active, w.err, opts->density_scaling, 0, sfloor,
                                        w.sfl);
      note_launch();
      TCAD_LAUNCH_CHECK();
      if (!any_retry) break;
      solve_set = retry;
    }
    TCAD_CUDA_CHECK(cudaMemcpyAsync(herr.data(), w.err, sizeof(unsigned long long) * ni,
                                    cudaMemcpyDeviceToHost, s));
    TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
    bool any = false;
    for (int i = 0; i < ni; ++i) {
      if (!hact[i]) continue;
      double e;
      std::memcpy(&e, &herr[i], sizeof(double));
      result[i].iters = it + 1;
      result[i].err = e;
      const bool lin_ok = result[i].status == TCAD_OK;
      const bool hard = result[i].status == TCAD_ERR_SINGULAR ||
                        result[i].status == TCAD_ERR_NONFINITE;
      if (opts->verbose)
        std::fprintf(stderr, "    [gpu] inst %d it %2d  err=%.3e  krylov=%d relres=%.2e eta=%.1e st=%d\n",
                    i, it, e, last_kit[i], result[i].relres, heta[i], result[i].status);
      // forcing term of the next step (inexact Newton): quadratic convergence
      // is kept while the linear tolerance tracks the update size
      if (opts->forcing)
        heta[i] = std::min(std::max(opts->eta_max, eta_lo),
                           std::max(eta_lo, 0.1 * (std::isfinite(e) ? e : 1.0)));
      if (polish_left[i] > 0) {
        // post-convergence polishing step (already counted as converged)
        ++result[i].polish_iters;
        if (--polish_left[i] == 0) hact[i] = 0;
      } else if (e < opts->tol_update && lin_ok) {
        result[i].converged = 1;
        polish_left[i] = opts->polish > 0 ? opts->polish : 0;
        if (polish_left[i] == 0) hact[i] = 0;
        // the polishing steps resolve what the floored update test cannot
        // see (sub-floor densities, low-bias currents): their own tolerance
        else if (opts->forcing && opts->polish_eta > 0.0)
          heta[i] = std::max(opts->rtol, opts->polish_eta);
      } else if (hard || !(e == e) || e == INFINITY) {
        hact[i] = 0;  // singular block / non-finite state: this instance failed
      }
      any = any || hact[i];
    }
    if (!any) break;
  }
  TCAD_CUDA_CHECK(cudaMemcpyAsync(active, hact.data(), ni, cudaMemcpyHostToDevice, s));
  TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
  return TCAD_OK;
}

extern "C" int tcad_equilibrium_solve(const tcad_pack_t* pk, double* psi, double* n,
                                      double* p, double* F, double* J, double* d,
                                      const tcad_newton_opts_t* opts, void* work,
                                      size_t work_bytes, tcad_newton_result_t* result,
                                      void* stream) {
  if (!pack_ok(pk) || !opts || !result || !work) return TCAD_ERR_ARG;
  Work w = carve(pk, work, work_bytes);
  if (w.bytes > work_bytes) return TCAD_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const int ni = pk->n_inst;
  const unsigned nb = (unsigned)pk->n_flat;
  std::vector<uint8_t> hact(ni, 1);
  uint8_t* dact = reinterpret_cast<uint8_t*>(w.status);  // reuse: n_inst bytes
  for (int i = 0; i < ni; ++i) {
    result[i].iters = 0; result[i].converged = 0; result[i].krylov_iters = 0;
    result[i].status = TCAD_OK; result[i].err = INFINITY; result[i].relres = 0.0;
    result[i].fp64_from = -1; result[i].polish_iters = 0;
  }
  std::vector<KState> hks;
  std::vector<unsigned long long> herr(ni);
  // inexact-Newton forcing (opts->forcing): step k's PCG is solved to
  // eta_k = clamp(0.1 |d_{k-1}|, rtol, eta_max), so the early steps from the
  // bulk guess stop at eta_max while the last ones, with |d| near the update
  // test, are solved to rtol; quadratic convergence is kept and the
  // converged potential is the same discrete solution
  std::vector<double> heta(ni, opts->forcing ? std::max(opts->eta_max, opts->rtol) : opts->rtol);
  // PCG on the red-black Schur complement (opts->red_black; the workspace's
  // equilibrium extension): the slot pack's tables once per call
  const bool use_rb = opts->red_black != 0 && work_bytes >= tcad_block_workspace_bytes(pk, 0, 0);
  WorkEq we{};
  RbLayout rbl;
  if (use_rb) {
    we = carve_eq(pk, reinterpret_cast<char*>(work) + off_eq(pk));
    if (int rc = rb_layout(pk, we, rbl, s)) return rc;
  }
  for (int it = 0; it < opts->max_iter; ++it) {
    TCAD_CUDA_CHECK(cudaMemcpyAsync(dact, hact.data(), ni, cudaMemcpyHostToDevice, s));
    TCAD_CUDA_CHECK(cudaMemcpyAsync(w.eta, heta.data(), sizeof(double) * ni,
                                    cudaMemcpyHostToDevice, s));
    int rc = tcad_poisson_assemble(pk, psi, F, J, TCAD_MODE_ELIMINATE, stream);
    if (rc != TCAD_OK) return rc;
    rc = use_rb ? launch_cg_rb(pk, rbl, we, J, F, d, opts->rtol, opts->krylov_maxiter, w, dact,
                               hks, s, w.eta)
                : launch_cg(pk, J, F, d, opts->rtol, opts->krylov_maxiter, w, dact, hks, s,
                            w.eta);
    if (rc != TCAD_OK) return rc;
    TCAD_CUDA_CHECK(cudaMemsetAsync(w.err, 0, sizeof(unsigned long long) * ni, s));
    k_eq_update<<<nb, NT, 0, s>>>(*pk, psi, d, opts->max_dpsi, dact, w.err);
    note_launch();
    TCAD_LAUNCH_CHECK();
    TCAD_CUDA_CHECK(cudaMemcpyAsync(herr.data(), w.err, sizeof(unsigned long long) * ni,
                                    cudaMemcpyDeviceToHost, s));
    TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
    bool any = false;
    for (int i = 0; i < ni; ++i) {
      if (!hact[i]) continue;
      double e;
      std::memcpy(&e, &herr[i], sizeof(double));
      result[i].iters = it + 1;
      result[i].err = e;
      result[i].krylov_iters += hks[i].it;
      result[i].status = hks[i].status;
      result[i].relres = hks[i].bb > 0.0 ? std::sqrt(hks[i].rr / hks[i].bb) : 0.0;
      if (opts->verbose)
        std::fprintf(stderr, "    [gpu] eq inst %d it %2d  |d|=%.3e  cg=%d st=%d\n", i, it, e,
                    hks[i].it, hks[i].status);
      if (e < opts->tol_update && result[i].status == TCAD_OK) {
        result[i].converged = 1;
        hact[i] = 0;
      } else if (!(e == e) || e == INFINITY) {
        hact[i] = 0;
      }
      if (opts->forcing)
        heta[i] = std::min(std::max(opts->eta_max, opts->rtol),
                           std::max(opts->rtol, 0.1 * (std::isfinite(e) ? e : 1.0)));
      any = any || hact[i];
    }
    if (!any) break;
  }
  k_slaved<<<nb, NT, 0, s>>>(*pk, psi, n, p);
  note_launch();
  TCAD_LAUNCH_CHECK();
  TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
  return TCAD_OK;
}

// ---------------------------------------------------------------------------
// Node-block BiCGStab that allocates nothing.
//
// Some callers cannot allocate device memory on demand: a serving process
// whose HBM is carved up by its own pool allocator up front, a foreign-
// language host (cgo, JNI, N-API) that has no device allocator to hand over
// scratch, or a latency-critical loop that must not pay cudaMalloc's implicit
// device-wide synchronisation.  For them the Krylov scratch lives in the
// file-scope device array below: TCAD_STATIC_SCRATCH_BYTES, which every GPU
// that loads this library keeps reserved until the process exits.  The
// caller passes only inputs (pack, prepared J, b) and outputs (x, per-
// instance results).
//
// Set-up: the array's host-side name is only a stand-in for the symbol, not
// a device address, so the first call on each device (with that device
// current) looks the address up with cudaGetSymbolAddress and caches it; make
// that first call before any stream capture.  All calls share the one array:
// the solver clears what must start at zero (reduction tickets) and
// initialises its vectors itself, and two calls whose work overlaps on the GPU
// (different streams, or different host threads) race on the scratch.
namespace tcad {

static __device__ __align__(256) unsigned char g_noalloc_scratch[TCAD_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
// Per-device address of the array, looked up once per device.  Host threads
// that race on the first call store the same value; the atomics make that
// well defined.  The address belongs to the device's context: after a
// cudaDeviceReset the library must be reloaded before this entry point is
// used again.
static std::atomic<void*> g_noalloc_addr[kMaxDevices];

static int noalloc_scratch(void** out) {
  int dev = -1;
  TCAD_CUDA_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return TCAD_ERR_ARG;
  void* p = g_noalloc_addr[dev].load(std::memory_order_acquire);
  if (p == nullptr) {
    TCAD_CUDA_CHECK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[dev].store(p, std::memory_order_release);
  }
  *out = p;
  return TCAD_OK;
}

}  // namespace tcad

extern "C" int tcad_block_krylov_noalloc(const tcad_pack_t* pk, const double* J,
                                         const double* b, double* x, double rtol,
                                         int maxiter, int32_t* iters, int32_t* status,
                                         double* relres, void* stream) {
  if (!pack_ok(pk) || !J || !b || !x) return TCAD_ERR_ARG;
  if (pk->n_nodes > TCAD_STATIC_MAX_NODES || pk->n_inst > TCAD_STATIC_MAX_INST ||
      pk->n_inst < 1)
    return TCAD_ERR_ARG;  // beyond the static scratch: use tcad_block_krylov
  void* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc != TCAD_OK) return rc;
  Work w = carve(pk, base, TCAD_STATIC_SCRATCH_BYTES);
  if (w.bytes > TCAD_STATIC_SCRATCH_BYTES) return TCAD_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned nb = (unsigned)pk->n_flat;
  const int ni = pk->n_inst;
  KState hks[TCAD_STATIC_MAX_INST];  // host mirror on the stack, no heap
  TCAD_CUDA_CHECK(cudaMemsetAsync(w.ticket, 0, sizeof(unsigned) * ni, s));
  k_bi_init<<<nb, NT, 0, s>>>(*pk, b, x, w.bi, w.ks, w.partial, w.ticket, rtol, maxiter,
                              nullptr, nullptr);
  note_launch();
  TCAD_LAUNCH_CHECK();
  int check = 4, done_iters = 0, rechecks = 0;
  for (;;) {
    for (int q = 0; q < check; ++q) {
      k_bi_p<<<nb, NT, 0, s>>>(*pk, w.bi, w.ks, nullptr);
      if (pk->dim == 2)
        k_bi_v<2><<<nb, NT, 0, s>>>(*pk, J, w.bi, w.ks, w.partial, w.ticket, nullptr);
      else
        k_bi_v<3><<<nb, NT, 0, s>>>(*pk, J, w.bi, w.ks, w.partial, w.ticket, nullptr);
      k_bi_s<<<nb, NT, 0, s>>>(*pk, w.bi, w.ks, w.partial, w.ticket, nullptr);
      if (pk->dim == 2)
        k_bi_t<2><<<nb, NT, 0, s>>>(*pk, J, w.bi, w.ks, w.partial, w.ticket, nullptr);
      else
        k_bi_t<3><<<nb, NT, 0, s>>>(*pk, J, w.bi, w.ks, w.partial, w.ticket, nullptr);
      k_bi_x<<<nb, NT, 0, s>>>(*pk, x, w.bi, w.ks, w.partial, w.ticket, nullptr);
      note_launch(5);
    }
    TCAD_LAUNCH_CHECK();
    done_iters += check;
    TCAD_CUDA_CHECK(cudaMemcpyAsync(hks, w.ks, sizeof(KState) * ni, cudaMemcpyDeviceToHost, s));
    TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
    bool any = false;
    for (int i = 0; i < ni; ++i) any = any || hks[i].active;
    if (!any) {
      const int rearm = rechecks < 8 ? 1 : 0;
      if (pk->dim == 2)
        k_true_resid<2><<<nb, NT, 0, s>>>(*pk, J, b, x, w.bi.r, w.ks, w.partial, w.ticket, rearm);
      else
        k_true_resid<3><<<nb, NT, 0, s>>>(*pk, J, b, x, w.bi.r, w.ks, w.partial, w.ticket, rearm);
      note_launch();
      TCAD_LAUNCH_CHECK();
      TCAD_CUDA_CHECK(cudaMemcpyAsync(hks, w.ks, sizeof(KState) * ni, cudaMemcpyDeviceToHost,
                                      s));
      TCAD_CUDA_CHECK(cudaStreamSynchronize(s));
      for (int i = 0; i < ni; ++i) any = any || hks[i].active;
      ++rechecks;
      if (!any) break;
    }
    if (done_iters > 64) check = 16;
    if (done_iters > 1024) check = 32;
  }
  for (int i = 0; i < ni; ++i) {
    if (iters) iters[i] = hks[i].it;
    if (status) status[i] = hks[i].status;
    if (relres) relres[i] = hks[i].bb > 0.0 ? std::sqrt(hks[i].rr / hks[i].bb) : 0.0;
  }
  return TCAD_OK;
}
