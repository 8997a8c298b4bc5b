// Block ILU(0) of the node-block-scaled 2D operator, as a right
// preconditioner of the BiCGStab in krylov.cu.  On 3D packs the same
// factorisation is taken plane by plane (the in-plane W/E/S/N couplings of
// each z-plane; the D/U couplings are left to the Krylov iteration): a
// block-diagonal-over-planes preconditioner, one CTA per (instance, plane).
//
// The scaled operator is A^ = I + G_k sum_d B_kd (node k, neighbours
// d = W, E, S, N): G_k is the (row-scaled) inverse diagonal block stored in
// J entries 0..8, B_kd the 5-entry neighbour block (psi<-psi, n<-psi, n<-n,
// p<-psi, p<-p) in entries 9 + 5d + m.  For the 5-point block stencil
// ILU(0) keeps the off-diagonal blocks of A^ and changes only the diagonal
// ones (no fill survives), i.e. M = (D~ + L^) D~^-1 (D~ + U^) with
//   D~_k = I - G_k (B_kW D~_W^-1 G_W B_WE + B_kS D~_S^-1 G_S B_SN)
// (W, S the lower neighbours in the x-fastest natural order).  Q_k = D~_k^-1
// is stored (9 doubles per node).  Applying M^-1 r:
//   forward  a_k = Q_k (r_k - G_k (B_kW a_W + B_kS a_S))
//   backward x_k = a_k - Q_k G_k (B_kE x_E + B_kN x_N)
// Node (i, j) depends on (i-1, j) and (i, j-1) only, so all nodes of an
// anti-diagonal i + j = d are independent: one CTA per instance sweeps the
// nx + ny - 1 anti-diagonals with a block barrier between them (global
// writes of a level are visible to the block after the barrier).
#pragma once

namespace tcad {

constexpr int kIluThreads = 256;

// C = M * B with B the sparse neighbour block (b0..b4)
__device__ __forceinline__ void mul_dense_nb(const double* M, const double* b, double* C) {
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    C[3 * r + 0] = M[3 * r + 0] * b[0] + M[3 * r + 1] * b[1] + M[3 * r + 2] * b[3];
    C[3 * r + 1] = M[3 * r + 1] * b[2];
    C[3 * r + 2] = M[3 * r + 2] * b[4];
  }
}

// C = B * M with B the sparse neighbour block
__device__ __forceinline__ void mul_nb_dense(const double* b, const double* M, double* C) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    C[0 + c] = b[0] * M[0 + c];
    C[3 + c] = b[1] * M[0 + c] + b[2] * M[3 + c];
    C[6 + c] = b[3] * M[0 + c] + b[4] * M[6 + c];
  }
}

__device__ __forceinline__ void mul33(const double* A, const double* B, double* C) {
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      C[3 * r + c] = A[3 * r + 0] * B[0 + c] + A[3 * r + 1] * B[3 + c] + A[3 * r + 2] * B[6 + c];
}

__device__ __forceinline__ void load9(const double* __restrict__ X, int64_t NN, int64_t k,
                                      int e0, double* out) {
#pragma unroll
  for (int e = 0; e < 9; ++e) out[e] = X[(int64_t)(e0 + e) * NN + k];
}

__device__ __forceinline__ void load_nb(const double* __restrict__ J, int64_t NN, int64_t k,
                                        int d, double* b) {
#pragma unroll
  for (int m = 0; m < 5; ++m) b[m] = J[(int64_t)(9 + 5 * d + m) * NN + k];
}

// y += B v (sparse neighbour block)
__device__ __forceinline__ void add_nb_vec(const double* b, double v0, double v1, double v2,
                                           double& y0, double& y1, double& y2) {
  y0 += b[0] * v0;
  y1 += b[1] * v0 + b[2] * v1;
  y2 += b[3] * v0 + b[4] * v2;
}

// ---------------------------------------------------------------------------
// Coalesced sweep (2D packs whose shorter side fits the block).
//
// The sweeps touch one node per row per anti-diagonal level, so in node
// order every access of a level is a separate memory sector.  The factor
// therefore also writes what the sweeps read in ANTI-DIAGONAL-MAJOR order:
// node (c, w) -- row c of the shorter side, position w along it -- of the
// plane whose first node is `base` sits in slot 2*base + (c + w)*Lc + c.
// A plane with Lc <= Lw rows has (Lc + Lw - 1) Lc <= 2 Lc Lw slots, so the
// slots of all planes fit in 2 * n_nodes.  Per slot (FP32, a preconditioner
// needs no more): forward Q, Q G B_walk, Q G B_cross (27 values),
// backward Q G B_walk', Q G B_cross' (18) -- G folded in, so
//   forward  a = Q r - (Q G B_walk) a_prev - (Q G B_cross) a_cross
//   backward x = a - (Q G B_walk') x_next - (Q G B_cross') x_cross'.
// The right-hand side is permuted into slot order and the result back by
// two node-parallel kernels.
struct IluGeo {
  bool byj;      // rows are j (ny <= nx), walk along i
  int Lc, Lw;    // rows, positions per row
  int64_t soff;  // first slot of the plane
};

__device__ __forceinline__ IluGeo ilu_geo(const Inst& g, int64_t base) {
  IluGeo q;
  q.byj = g.ny <= g.nx;
  q.Lc = q.byj ? g.ny : g.nx;
  q.Lw = q.byj ? g.nx : g.ny;
  q.soff = 2 * base;
  return q;
}

// slot of node (i, j) of the plane
__device__ __forceinline__ int64_t ilu_slot(const IluGeo& q, int i, int j) {
  const int c = q.byj ? j : i, w = q.byj ? i : j;
  return q.soff + (int64_t)(c + w) * q.Lc + c;
}

// store the forward / backward sweep data of node k (FP32, slot order)
__device__ __forceinline__ void ilu_store_slot(const double* __restrict__ J, int64_t NN,
                                               int64_t k, const IluGeo& q, int i, int j,
                                               int nx, int ny, const double* Qk,
                                               float* __restrict__ Mf, float* __restrict__ Mb,
                                               int64_t NS) {
  double G[9], QG[9], b[5], T1[9];
  load9(J, NN, k, 0, G);
  mul33(Qk, G, QG);
  const int64_t sl = ilu_slot(q, i, j);
  const int c = q.byj ? j : i, w = q.byj ? i : j;
  // direction indices: W 0, E 1, S 2, N 3
  const int dwp = q.byj ? 0 : 2, dcp = q.byj ? 2 : 0;
  const int dwn = q.byj ? 1 : 3, dcn = q.byj ? 3 : 1;
#pragma unroll
  for (int e = 0; e < 9; ++e) Mf[(int64_t)e * NS + sl] = (float)Qk[e];
  const bool has[4] = {w > 0, c > 0, w < q.Lw - 1, c < q.Lc - 1};
  const int dir[4] = {dwp, dcp, dwn, dcn};
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    if (has[m]) {
      load_nb(J, NN, k, dir[m], b);
      mul_dense_nb(QG, b, T1);
    } else {
#pragma unroll
      for (int e = 0; e < 9; ++e) T1[e] = 0.0;
    }
    float* dst = m < 2 ? Mf + (int64_t)(9 + 9 * m) * NS : Mb + (int64_t)(9 * (m - 2)) * NS;
#pragma unroll
    for (int e = 0; e < 9; ++e) dst[(int64_t)e * NS + sl] = (float)T1[e];
  }
  (void)nx; (void)ny;
}

// r (node order) -> rs (slot order) for the instances preconditioned here;
// the others' ph = p is written by k_ilu_unperm.
// Factor: Q_k for every node of each instance whose pre_status is TCAD_OK;
// status[inst] = TCAD_ERR_SINGULAR when a D~ block is singular.
__global__ void __launch_bounds__(kIluThreads)
k_ilu2d_factor(const tcad_pack_t pk, const double* __restrict__ J, double* __restrict__ Q,
               const int32_t* __restrict__ pre_status, int32_t* __restrict__ status,
               int nzmax, float* __restrict__ Mf, float* __restrict__ Mb) {
  const int inst = blockIdx.x / nzmax, z = blockIdx.x % nzmax;
  if (pre_status && pre_status[inst] != TCAD_OK) return;
  const Inst g = load_inst(pk, inst);
  if (z >= g.nz) return;
  const int64_t base = g.off + (int64_t)z * g.nx * g.ny;  // this z-plane (2D: the instance)
  const int64_t NN = pk.n_nodes;
  const int nx = g.nx, ny = g.ny;
  for (int d = 0; d < nx + ny - 1; ++d) {
    const int jlo = d - (nx - 1) > 0 ? d - (nx - 1) : 0;
    const int jhi = d < ny - 1 ? d : ny - 1;
    for (int j = jlo + threadIdx.x; j <= jhi; j += kIluThreads) {
      const int i = d - j;
      const int64_t k = base + (int64_t)j * nx + i;
      double S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      double b[5], G[9], Qm[9], T1[9], T2[9], T3[9];
      if (i > 0) {  // W: term B_kW Q_W G_W B_WE
        const int64_t m = k - 1;
        load9(J, NN, m, 0, G);
        load_nb(J, NN, m, 1, b);
        mul_dense_nb(G, b, T1);
        load9(Q, NN, m, 0, Qm);
        mul33(Qm, T1, T2);
        load_nb(J, NN, k, 0, b);
        mul_nb_dense(b, T2, T3);
#pragma unroll
        for (int e = 0; e < 9; ++e) S[e] += T3[e];
      }
      if (j > 0) {  // S: term B_kS Q_S G_S B_SN
        const int64_t m = k - nx;
        load9(J, NN, m, 0, G);
        load_nb(J, NN, m, 3, b);
        mul_dense_nb(G, b, T1);
        load9(Q, NN, m, 0, Qm);
        mul33(Qm, T1, T2);
        load_nb(J, NN, k, 2, b);
        mul_nb_dense(b, T2, T3);
#pragma unroll
        for (int e = 0; e < 9; ++e) S[e] += T3[e];
      }
      load9(J, NN, k, 0, G);
      double D[9];
      mul33(G, S, D);
#pragma unroll
      for (int e = 0; e < 9; ++e) D[e] = (e % 4 == 0 ? 1.0 : 0.0) - D[e];
      const double c00 = D[4] * D[8] - D[5] * D[7];
      const double c01 = D[5] * D[6] - D[3] * D[8];
      const double c02 = D[3] * D[7] - D[4] * D[6];
      const double det = D[0] * c00 + D[1] * c01 + D[2] * c02;
      double inv[9];
      if (isfinite(det) && fabs(det) >= 1e-300) {
        const double id = 1.0 / det;
        inv[0] = c00 * id;
        inv[1] = (D[2] * D[7] - D[1] * D[8]) * id;
        inv[2] = (D[1] * D[5] - D[2] * D[4]) * id;
        inv[3] = c01 * id;
        inv[4] = (D[0] * D[8] - D[2] * D[6]) * id;
        inv[5] = (D[2] * D[3] - D[0] * D[5]) * id;
        inv[6] = c02 * id;
        inv[7] = (D[1] * D[6] - D[0] * D[7]) * id;
        inv[8] = (D[0] * D[4] - D[1] * D[3]) * id;
      } else {
        if (status) atomicExch(&status[inst], TCAD_ERR_SINGULAR);
#pragma unroll
        for (int e = 0; e < 9; ++e) inv[e] = (e % 4 == 0) ? 1.0 : 0.0;
      }
#pragma unroll
      for (int e = 0; e < 9; ++e) Q[(int64_t)e * NN + k] = inv[e];
      if (Mf) ilu_store_slot(J, NN, k, ilu_geo(g, base), i, j, nx, ny, inv, Mf, Mb, 2 * NN);
    }
    __syncthreads();
  }
}

// out = M^-1 rin for every instance still iterating (ks[inst].active);
// instances with mask[inst] == 0 are not preconditioned (out = rin).
template <class T>
__global__ void __launch_bounds__(kIluThreads)
k_ilu2d_apply(const tcad_pack_t pk, const double* __restrict__ J, const double* __restrict__ Q,
              const T* __restrict__ rin, T* __restrict__ out, const KState* ks,
              const uint8_t* __restrict__ mask, int nzmax) {
  const int inst = blockIdx.x / nzmax, z = blockIdx.x % nzmax;
  if (ks && !ks[inst].active) return;
  const Inst g = load_inst(pk, inst);
  if (z >= g.nz) return;
  const int64_t base = g.off + (int64_t)z * g.nx * g.ny;  // this z-plane (2D: the instance)
  const int64_t NN = pk.n_nodes;
  if (mask && !mask[inst]) {
    const int64_t end = base + (int64_t)g.nx * g.ny;
    for (int64_t k = base + threadIdx.x; k < end; k += kIluThreads) {
      out[k] = rin[k];
      out[NN + k] = rin[NN + k];
      out[2 * NN + k] = rin[2 * NN + k];
    }
    return;
  }
  const int nx = g.nx, ny = g.ny;
  const int nd = nx + ny - 1;
  // Fast path when every anti-diagonal fits the block (min(nx, ny) <=
  // threads).  Each thread owns one row c of the shorter dimension (j, or i
  // when nx < ny) and walks along it, one node per anti-diagonal level: the
  // previous node of its own row is in a register, the other lower
  // neighbour (row c-1, same position) comes from a shared-memory front,
  // and the node data of the next two positions of its row is already in
  // flight, so each level costs only the dependent arithmetic and a barrier.
  const bool byj = ny <= nx;
  const int Lc = byj ? ny : nx, Lw = byj ? nx : ny;
  if (Lc <= kIluThreads) {
    __shared__ double fr[2][kIluThreads][3];
    // rows by parity: warps 0..3 own the even rows, warps 4..7 the odd ones,
    // so (d - c) has one parity across a warp and the slot choice below
    // never diverges inside a warp
    const int tid = threadIdx.x, half = kIluThreads / 2;
    const int c = tid < half ? 2 * tid : 2 * (tid - half) + 1;
    const bool lane = c < Lc;
    // neighbour directions: along the row (walk) and across rows (cross)
    const int dwp = byj ? 0 : 2, dcp = byj ? 2 : 0;   // forward: W/S
    const int dwn = byj ? 1 : 3, dcn = byj ? 3 : 1;   // backward: E/N
    auto node = [&](int w) -> int64_t {
      return byj ? base + (int64_t)c * nx + w : base + (int64_t)w * nx + c;
    };
    struct Nd {
      double G[9], Q[9], bw[5], bc[5], v[3];
    };
    // forward data of position w (v = r)
    auto load_f = [&](int w, Nd& o) {
      if (!lane || w < 0 || w >= Lw) return;
      const int64_t k = node(w);
      load9(J, NN, k, 0, o.G);
      load9(Q, NN, k, 0, o.Q);
      if (w > 0) load_nb(J, NN, k, dwp, o.bw);
      if (c > 0) load_nb(J, NN, k, dcp, o.bc);
      o.v[0] = rin[k]; o.v[1] = rin[NN + k]; o.v[2] = rin[2 * NN + k];
    };
    // backward data of position w (v = a from the forward sweep)
    auto load_b = [&](int w, Nd& o) {
      if (!lane || w < 0 || w >= Lw) return;
      const int64_t k = node(w);
      load9(J, NN, k, 0, o.G);
      load9(Q, NN, k, 0, o.Q);
      if (w < Lw - 1) load_nb(J, NN, k, dwn, o.bw);
      if (c < Lc - 1) load_nb(J, NN, k, dcn, o.bc);
      o.v[0] = out[k]; o.v[1] = out[NN + k]; o.v[2] = out[2 * NN + k];
    };
    // two register slots: position w lives in slot (w & 1); after a
    // position is used its slot is reloaded with position w + 2 (no copies,
    // so a pending load is waited for only where its data is used)
    Nd A, B;
    double p0 = 0.0, p1 = 0.0, p2 = 0.0;   // own previous result
    int cur = 0;
    auto fstep = [&](const Nd& X, int w) {
      const int pv = cur ^ 1;
      double u0 = 0.0, u1 = 0.0, u2 = 0.0;
      if (w > 0) add_nb_vec(X.bw, p0, p1, p2, u0, u1, u2);
      if (c > 0) {
        const double* f = fr[pv][c - 1];
        add_nb_vec(X.bc, f[0], f[1], f[2], u0, u1, u2);
      }
      const double t0 = X.v[0] - (X.G[0] * u0 + X.G[1] * u1 + X.G[2] * u2);
      const double t1 = X.v[1] - (X.G[3] * u0 + X.G[4] * u1 + X.G[5] * u2);
      const double t2 = X.v[2] - (X.G[6] * u0 + X.G[7] * u1 + X.G[8] * u2);
      p0 = X.Q[0] * t0 + X.Q[1] * t1 + X.Q[2] * t2;
      p1 = X.Q[3] * t0 + X.Q[4] * t1 + X.Q[5] * t2;
      p2 = X.Q[6] * t0 + X.Q[7] * t1 + X.Q[8] * t2;
      double* f = fr[cur][c];
      f[0] = p0; f[1] = p1; f[2] = p2;
      const int64_t k = node(w);
      out[k] = (T)p0; out[NN + k] = (T)p1; out[2 * NN + k] = (T)p2;
    };
    auto bstep = [&](const Nd& X, int w) {
      const int pv = cur ^ 1;
      double u0 = 0.0, u1 = 0.0, u2 = 0.0;
      if (w < Lw - 1) add_nb_vec(X.bw, p0, p1, p2, u0, u1, u2);
      if (c < Lc - 1) {
        const double* f = fr[pv][c + 1];
        add_nb_vec(X.bc, f[0], f[1], f[2], u0, u1, u2);
      }
      const double t0 = X.G[0] * u0 + X.G[1] * u1 + X.G[2] * u2;
      const double t1 = X.G[3] * u0 + X.G[4] * u1 + X.G[5] * u2;
      const double t2 = X.G[6] * u0 + X.G[7] * u1 + X.G[8] * u2;
      p0 = X.v[0] - (X.Q[0] * t0 + X.Q[1] * t1 + X.Q[2] * t2);
      p1 = X.v[1] - (X.Q[3] * t0 + X.Q[4] * t1 + X.Q[5] * t2);
      p2 = X.v[2] - (X.Q[6] * t0 + X.Q[7] * t1 + X.Q[8] * t2);
      double* f = fr[cur][c];
      f[0] = p0; f[1] = p1; f[2] = p2;
      const int64_t k = node(w);
      out[k] = (T)p0; out[NN + k] = (T)p1; out[2 * NN + k] = (T)p2;
    };
    // ---- forward: a_k = Q_k (r_k - G_k (B_walk a_prev + B_cross a_cross))
    load_f(0, A);
    load_f(1, B);
    for (int d = 0; d < nd; ++d) {
      const int w = d - c;
      if (lane && w >= 0 && w < Lw) {
        if ((w & 1) == 0) {
          fstep(A, w);
          load_f(w + 2, A);
        } else {
          fstep(B, w);
          load_f(w + 2, B);
        }
      }
      __syncthreads();
      cur ^= 1;
    }
    // ---- backward: x_k = a_k - Q_k G_k (B_walk x_next + B_cross x_cross)
    if (((Lw - 1) & 1) == 0) {
      load_b(Lw - 1, A);
      load_b(Lw - 2, B);
    } else {
      load_b(Lw - 1, B);
      load_b(Lw - 2, A);
    }
    for (int d = nd - 1; d >= 0; --d) {
      const int w = d - c;
      if (lane && w >= 0 && w < Lw) {
        if ((w & 1) == 0) {
          bstep(A, w);
          load_b(w - 2, A);
        } else {
          bstep(B, w);
          load_b(w - 2, B);
        }
      }
      __syncthreads();
      cur ^= 1;
    }
    return;
  }
  // forward: a_k = Q_k (r_k - G_k (B_kW a_W + B_kS a_S))
  for (int d = 0; d < nd; ++d) {
    const int jlo = d - (nx - 1) > 0 ? d - (nx - 1) : 0;
    const int jhi = d < ny - 1 ? d : ny - 1;
    for (int j = jlo + threadIdx.x; j <= jhi; j += kIluThreads) {
      const int i = d - j;
      const int64_t k = base + (int64_t)j * nx + i;
      double u0 = 0.0, u1 = 0.0, u2 = 0.0, b[5];
      if (i > 0) {
        load_nb(J, NN, k, 0, b);
        add_nb_vec(b, out[k - 1], out[NN + k - 1], out[2 * NN + k - 1], u0, u1, u2);
      }
      if (j > 0) {
        load_nb(J, NN, k, 2, b);
        add_nb_vec(b, out[k - nx], out[NN + k - nx], out[2 * NN + k - nx], u0, u1, u2);
      }
      double G[9], Qk[9];
      load9(J, NN, k, 0, G);
      load9(Q, NN, k, 0, Qk);
      const double t0 = rin[k] - (G[0] * u0 + G[1] * u1 + G[2] * u2);
      const double t1 = rin[NN + k] - (G[3] * u0 + G[4] * u1 + G[5] * u2);
      const double t2 = rin[2 * NN + k] - (G[6] * u0 + G[7] * u1 + G[8] * u2);
      out[k] = (T)(Qk[0] * t0 + Qk[1] * t1 + Qk[2] * t2);
      out[NN + k] = (T)(Qk[3] * t0 + Qk[4] * t1 + Qk[5] * t2);
      out[2 * NN + k] = (T)(Qk[6] * t0 + Qk[7] * t1 + Qk[8] * t2);
    }
    __syncthreads();
  }
  // backward: x_k = a_k - Q_k G_k (B_kE x_E + B_kN x_N), in place
  for (int d = nd - 1; d >= 0; --d) {
    const int jlo = d - (nx - 1) > 0 ? d - (nx - 1) : 0;
    const int jhi = d < ny - 1 ? d : ny - 1;
    for (int j = jlo + threadIdx.x; j <= jhi; j += kIluThreads) {
      const int i = d - j;
      const int64_t k = base + (int64_t)j * nx + i;
      double u0 = 0.0, u1 = 0.0, u2 = 0.0, b[5];
      if (i < nx - 1) {
        load_nb(J, NN, k, 1, b);
        add_nb_vec(b, out[k + 1], out[NN + k + 1], out[2 * NN + k + 1], u0, u1, u2);
      }
      if (j < ny - 1) {
        load_nb(J, NN, k, 3, b);
        add_nb_vec(b, out[k + nx], out[NN + k + nx], out[2 * NN + k + nx], u0, u1, u2);
      }
      double G[9], Qk[9];
      load9(J, NN, k, 0, G);
      load9(Q, NN, k, 0, Qk);
      const double t0 = G[0] * u0 + G[1] * u1 + G[2] * u2;
      const double t1 = G[3] * u0 + G[4] * u1 + G[5] * u2;
      const double t2 = G[6] * u0 + G[7] * u1 + G[8] * u2;
      out[k] = (T)((double)out[k] - (Qk[0] * t0 + Qk[1] * t1 + Qk[2] * t2));
      out[NN + k] = (T)((double)out[NN + k] - (Qk[3] * t0 + Qk[4] * t1 + Qk[5] * t2));
      out[2 * NN + k] = (T)((double)out[2 * NN + k] - (Qk[6] * t0 + Qk[7] * t1 + Qk[8] * t2));
    }
    __syncthreads();
  }
}

}  // namespace tcad

namespace tcad {

constexpr int NT_ILU_FLAT = 256;  // flat (node-parallel) permutation kernels

template <class T>
__global__ void __launch_bounds__(NT_ILU_FLAT)
k_ilu_perm(const tcad_pack_t pk, const T* __restrict__ r, double* __restrict__ rs,
           const KState* ks, const uint8_t* __restrict__ mask, const int32_t* __restrict__ blk,
           int64_t NS) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pk, fbi);
  if (ks && !ks[fb.inst].active) return;
  if (mask && !mask[fb.inst]) return;
  const Inst g = load_inst(pk, fb.inst);
  const IluGeo q = ilu_geo(g, g.off);
  const int64_t NN = pk.n_nodes;
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT_ILU_FLAT) {
    const int64_t loc = k - g.off;
    const int i = (int)(loc % g.nx), j = (int)(loc / g.nx);
    const int64_t sl = ilu_slot(q, i, j);
    rs[sl] = (double)r[k];
    rs[NS + sl] = (double)r[NN + k];
    rs[2 * NS + sl] = (double)r[2 * NN + k];
  }
}

// out (node order) = xs (slot order); instances not preconditioned: out = r
template <class T>
__global__ void __launch_bounds__(NT_ILU_FLAT)
k_ilu_unperm(const tcad_pack_t pk, const double* __restrict__ xs, const T* __restrict__ r,
             T* __restrict__ out, const KState* ks, const uint8_t* __restrict__ mask,
             const int32_t* __restrict__ blk, int64_t NS) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pk, fbi);
  if (ks && !ks[fb.inst].active) return;
  const int64_t NN = pk.n_nodes;
  if (mask && !mask[fb.inst]) {
    for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT_ILU_FLAT) {
      out[k] = r[k]; out[NN + k] = r[NN + k]; out[2 * NN + k] = r[2 * NN + k];
    }
    return;
  }
  const Inst g = load_inst(pk, fb.inst);
  const IluGeo q = ilu_geo(g, g.off);
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += NT_ILU_FLAT) {
    const int64_t loc = k - g.off;
    const int i = (int)(loc % g.nx), j = (int)(loc / g.nx);
    const int64_t sl = ilu_slot(q, i, j);
    out[k] = (T)xs[sl]; out[NN + k] = (T)xs[NS + sl]; out[2 * NN + k] = (T)xs[2 * NS + sl];
  }
}

// The sweeps, one CTA per 2D instance (Lc <= kIluThreads): thread c owns
// row c.  Level d's data of thread c is slot soff + d Lc + c, so a level's
// loads are coalesced across the block; they are issued two levels ahead
// into one of three register sets chosen by d mod 3 (uniform in the block).
// xs holds a after the forward sweep and x after the backward one.
__global__ void __launch_bounds__(kIluThreads)
k_ilu_sweep(const tcad_pack_t pk, const float* __restrict__ Mf, const float* __restrict__ Mb,
            const double* __restrict__ rs, double* __restrict__ xs, const KState* ks,
            const uint8_t* __restrict__ mask, int64_t NS) {
  const int inst = blockIdx.x;
  if (ks && !ks[inst].active) return;
  if (mask && !mask[inst]) return;
  const Inst g = load_inst(pk, inst);
  const IluGeo q = ilu_geo(g, g.off);
  const int Lc = q.Lc, Lw = q.Lw, nd = Lc + Lw - 1;
  const int c = threadIdx.x;
  const bool lane = c < Lc;
  __shared__ double fr[2][kIluThreads][3];
  struct Fd {
    float q[9], mw[9], mc[9];
    double r[3];
  };
  struct Bd {
    float mw[9], mc[9];
    double a[3];
  };
  auto valid = [&](int d) { const int w = d - c; return lane && d >= 0 && d < nd && w >= 0 && w < Lw; };
  auto fload = [&](int d, Fd& o) {
    if (!valid(d)) return;
    const int64_t sl = q.soff + (int64_t)d * Lc + c;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      o.q[e] = Mf[(int64_t)e * NS + sl];
      o.mw[e] = Mf[(int64_t)(9 + e) * NS + sl];
      o.mc[e] = Mf[(int64_t)(18 + e) * NS + sl];
    }
    o.r[0] = rs[sl]; o.r[1] = rs[NS + sl]; o.r[2] = rs[2 * NS + sl];
  };
  auto bload = [&](int d, Bd& o) {
    if (!valid(d)) return;
    const int64_t sl = q.soff + (int64_t)d * Lc + c;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      o.mw[e] = Mb[(int64_t)e * NS + sl];
      o.mc[e] = Mb[(int64_t)(9 + e) * NS + sl];
    }
    o.a[0] = xs[sl]; o.a[1] = xs[NS + sl]; o.a[2] = xs[2 * NS + sl];
  };
  double p0 = 0.0, p1 = 0.0, p2 = 0.0;  // own previous result (same row)
  int cur = 0;
  auto fstep = [&](int d, const Fd& X) {
    if (valid(d)) {
      const int w = d - c;
      const double* fc = fr[cur ^ 1][c > 0 ? c - 1 : 0];
      const double c0 = c > 0 ? fc[0] : 0.0, c1 = c > 0 ? fc[1] : 0.0, c2 = c > 0 ? fc[2] : 0.0;
      const double w0 = w > 0 ? p0 : 0.0, w1 = w > 0 ? p1 : 0.0, w2 = w > 0 ? p2 : 0.0;
      double a[3];
#pragma unroll
      for (int r = 0; r < 3; ++r)
        a[r] = ((double)X.q[3 * r] * X.r[0] + (double)X.q[3 * r + 1] * X.r[1] +
                (double)X.q[3 * r + 2] * X.r[2]) -
               ((double)X.mw[3 * r] * w0 + (double)X.mw[3 * r + 1] * w1 +
                (double)X.mw[3 * r + 2] * w2) -
               ((double)X.mc[3 * r] * c0 + (double)X.mc[3 * r + 1] * c1 +
                (double)X.mc[3 * r + 2] * c2);
      p0 = a[0]; p1 = a[1]; p2 = a[2];
      double* f = fr[cur][c];
      f[0] = a[0]; f[1] = a[1]; f[2] = a[2];
      const int64_t sl = q.soff + (int64_t)d * Lc + c;
      xs[sl] = a[0]; xs[NS + sl] = a[1]; xs[2 * NS + sl] = a[2];
    }
    __syncthreads();
    cur ^= 1;
  };
  auto bstep = [&](int d, const Bd& X) {
    if (valid(d)) {
      const int w = d - c;
      const double* fc = fr[cur ^ 1][c < Lc - 1 ? c + 1 : c];
      const bool hc = c < Lc - 1, hw = w < Lw - 1;
      const double c0 = hc ? fc[0] : 0.0, c1 = hc ? fc[1] : 0.0, c2 = hc ? fc[2] : 0.0;
      const double w0 = hw ? p0 : 0.0, w1 = hw ? p1 : 0.0, w2 = hw ? p2 : 0.0;
      double x[3];
#pragma unroll
      for (int r = 0; r < 3; ++r)
        x[r] = X.a[r] -
               ((double)X.mw[3 * r] * w0 + (double)X.mw[3 * r + 1] * w1 +
                (double)X.mw[3 * r + 2] * w2) -
               ((double)X.mc[3 * r] * c0 + (double)X.mc[3 * r + 1] * c1 +
                (double)X.mc[3 * r + 2] * c2);
      p0 = x[0]; p1 = x[1]; p2 = x[2];
      double* f = fr[cur][c];
      f[0] = x[0]; f[1] = x[1]; f[2] = x[2];
      const int64_t sl = q.soff + (int64_t)d * Lc + c;
      xs[sl] = x[0]; xs[NS + sl] = x[1]; xs[2 * NS + sl] = x[2];
    }
    __syncthreads();
    cur ^= 1;
  };
  {  // forward, levels 0 .. nd-1, data two levels ahead
    Fd S0, S1, S2;
    fload(0, S0);
    fload(1, S1);
    for (int d = 0; d < nd; d += 3) {
      fload(d + 2, S2);
      fstep(d, S0);
      if (d + 1 >= nd) break;
      fload(d + 3, S0);
      fstep(d + 1, S1);
      if (d + 2 >= nd) break;
      fload(d + 4, S1);
      fstep(d + 2, S2);
    }
  }
  {  // backward, levels nd-1 .. 0
    Bd S0, S1, S2;
    bload(nd - 1, S0);
    bload(nd - 2, S1);
    for (int d = nd - 1; d >= 0; d -= 3) {
      bload(d - 2, S2);
      bstep(d, S0);
      if (d - 1 < 0) break;
      bload(d - 3, S0);
      bstep(d - 1, S1);
      if (d - 2 < 0) break;
      bload(d - 4, S1);
      bstep(d - 2, S2);
    }
  }
}

}  // namespace tcad
