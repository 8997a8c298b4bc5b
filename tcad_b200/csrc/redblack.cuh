// Red-black reduction of the block-scaled node system.
//
// The stencils couple a node only to its face neighbours (5 points in 2D, 7
// in 3D), so colouring node (i, j, k) by (i + j + k) & 1 -- red 0, black 1 --
// leaves no coupling inside a colour.  After the block-Jacobi set-up every
// diagonal block of A^ is the identity, and
//
//     A^ = [ I  E ]      x_r = b_r - E x_b,
//          [ F  I ]      (I - F E) x_b = b_b - F b_r.
//
// BiCGStab runs on the Schur complement I - F E over the black nodes: half
// the unknowns, one red pass (t = E x: the red rows of A^ on black values)
// and one black pass (x - F t) per operator product -- the same matrix bytes
// as one product with A^ -- and measured on the tri-gate Newton systems
// about half the iterations of the full system (the reduction is the exact
// elimination that red-black ILU(0) approximates).  The full residual of a
// black iterate is (0, r_schur), so the stopping test is the full system's
// own: ||b - A^ x|| <= rtol ||b||, with ||b|| the full right-hand side.
//
// Compact colour layout ("slots"): each instance row (j, k) holds
// hx = ceil(nx / 2) slots of each colour; the colour-c node (i, j, k) sits at
// slot soff + (j + ny k) hx + (i >> 1) of that colour's arrays, so a warp's
// consecutive slots are consecutive nodes of one colour along x and every
// neighbour is at a coalesced slot of the other colour.  Rows with nx odd
// have one pad slot in one colour; pad slots hold zeros in every matrix and
// vector, which every kernel here keeps.  The slot arrays are described by a
// derived pack (pkb): n_nodes = slots, shape (hx, ny nz, 1) per instance, its
// own flat blocks -- so the generic vector kernels (k_bi_p, k_bi_s, k_bi_x)
// and the per-instance reductions run on it unchanged.

namespace tcad {

struct RbMap {
  const int32_t* shape;     // the original pack's [3 n_inst] Nx, Ny, Nz
  const int64_t* node_off;  // the original pack's first node of each instance
  int64_t n_full;           // the original pack's n_nodes (vector stride)
};

struct RbGeo {
  int nx, ny, nz, hx;
  int64_t soff, ooff;  // first slot, first node
};

__device__ __forceinline__ RbGeo rb_geo(const tcad_pack_t& pkb, const RbMap& mp, int inst) {
  RbGeo g;
  g.nx = mp.shape[3 * inst];
  g.ny = mp.shape[3 * inst + 1];
  g.nz = mp.shape[3 * inst + 2];
  g.hx = (g.nx + 1) >> 1;
  g.soff = pkb.node_off[inst];
  g.ooff = mp.node_off[inst];
  return g;
}

struct RbNode {
  int i, j, k;
  int row;       // j + ny k
  int64_t node;  // index in the original pack
  bool real;     // false: a pad slot
};

// Index arithmetic is 32-bit and instance-local (an instance has far fewer
// than 2^31 slots): 64-bit division is a long instruction sequence and its
// registers halved the occupancy of the passes.  The passes that run every
// iteration are held to 5 CTAs per SM (51 registers; the black passes spill
// 44 bytes): they are latency-bound -- under ncu the 3-CTA black pass waited
// 33 long-scoreboard stalls per issue at 34 % warps active, DRAM 33 % busy
// -- and a whole iteration went from 511 us at 4 CTAs to 419 at 5.
__device__ __forceinline__ RbNode rb_node(const RbGeo& g, int64_t slot, int colour) {
  RbNode q;
  const unsigned local = (unsigned)(slot - g.soff);
  const unsigned row = local / (unsigned)g.hx;
  const int hi = (int)(local - row * (unsigned)g.hx);
  const unsigned k = row / (unsigned)g.ny;
  q.row = (int)row;
  q.k = (int)k;
  q.j = (int)(row - k * (unsigned)g.ny);
  q.i = 2 * hi + (((q.j + q.k) & 1) ^ colour);
  q.real = q.i < g.nx;
  q.node = g.ooff + (int64_t)row * g.nx + q.i;
  return q;
}

// instance-local slots (in the other colour's arrays) of the face neighbours
// x-, x+, y-, y+, z-, z+ -- the order of the Jacobian's neighbour entries; a
// missing neighbour gets the node's own slot (its Jacobian entries are zero)
template <int DIM>
__device__ __forceinline__ void rb_nbrs(const RbGeo& g, const RbNode& q, int self, int* m) {
  const int base = q.row * g.hx;
  const int h = q.i >> 1;
  m[0] = q.i > 0 ? base + ((q.i - 1) >> 1) : self;
  m[1] = q.i + 1 < g.nx ? base + ((q.i + 1) >> 1) : self;
  m[2] = q.j > 0 ? base - g.hx + h : self;
  m[3] = q.j + 1 < g.ny ? base + g.hx + h : self;
  if (DIM == 3) {
    const int plane = g.ny * g.hx;
    m[4] = q.k > 0 ? base - plane + h : self;
    m[5] = q.k + 1 < g.nz ? base + plane + h : self;
  }
}

// Colour rows of J are stored in warp tiles: the NE entries of 32
// consecutive slots are one contiguous run of NE x 32 doubles (entry e of
// slot s at ((s / 32) NE + e) 32 + s % 32), so a warp's loads of a slot row
// stay inside one 10 KB (3D) span instead of touching NE arrays a whole
// colour apart.
template <int NE>
__device__ __forceinline__ int64_t rb_jidx(int e, int64_t slot) {
  return (((slot >> 5) * NE + e) << 5) + (slot & 31);
}

// y = D (sum_d A_d x_m(d)) at one slot of a colour array Jc (warp tiles; the
// set-up's D^-1 in entries 0..8, the raw neighbour entries after them): the
// coupling part of A^ on the other colour's values; xi = that colour's
// vector from the instance's first slot, m instance-local
template <int DIM>
__device__ __forceinline__ void rb_couple(const double* __restrict__ Jc,
                                          const double* __restrict__ xi, int64_t slot,
                                          int64_t NS, const int* m, double& y0, double& y1,
                                          double& y2) {
  constexpr int NE = Stencil<DIM>::NE;
  const double* __restrict__ Jt = Jc + rb_jidx<NE>(0, slot);   // entry e at Jt[32 e]
  double t0 = 0.0, t1 = 0.0, t2 = 0.0;
#pragma unroll
  for (int d = 0; d < 2 * DIM; ++d) {
    const int e = 9 + 5 * d;
    const double xs = xi[m[d]], xn = xi[NS + m[d]], xp = xi[2 * NS + m[d]];
    t0 += Jt[32 * e] * xs;
    t1 += Jt[32 * (e + 1)] * xs + Jt[32 * (e + 2)] * xn;
    t2 += Jt[32 * (e + 3)] * xs + Jt[32 * (e + 4)] * xp;
  }
  double d[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) d[e] = Jt[32 * e];
  y0 = d[0] * t0 + d[1] * t1 + d[2] * t2;
  y1 = d[3] * t0 + d[4] * t1 + d[5] * t2;
  y2 = d[6] * t0 + d[7] * t1 + d[8] * t2;
}

// JR, JB <- the red and black rows of the block-scaled J in warp tiles
// (zeros at pads; the tile tail past the last slot is never read)
template <int DIM>
__global__ void __launch_bounds__(NT)
k_rb_pack(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ J,
          double* __restrict__ JR, double* __restrict__ JB) {
  constexpr int NE = Stencil<DIM>::NE;
  const FlatBlock fb = flat_block(pkb, blockIdx.x);
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes, NN = mp.n_full;
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const RbNode q = rb_node(g, slot, c);
      double* __restrict__ out = c ? JB : JR;
#pragma unroll 13
      for (int e = 0; e < NE; ++e)
        out[rb_jidx<NE>(e, slot)] = q.real ? J[(int64_t)e * NN + q.node] : 0.0;
    }
  }
}

// bR, bB <- the colours of b; per instance (b, b) of the full vector
template <int DIM>
__global__ void __launch_bounds__(NT)
k_rb_split(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ b,
           double* __restrict__ bR, double* __restrict__ bB, double* __restrict__ bbf,
           double* partial, unsigned* ticket) {
  const FlatBlock fb = flat_block(pkb, blockIdx.x);
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes, NN = mp.n_full;
  double v = 0.0;
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const RbNode q = rb_node(g, slot, c);
      double* __restrict__ out = c ? bB : bR;
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const double bv = q.real ? b[r * NN + q.node] : 0.0;
        out[r * NS + slot] = bv;
        v += bv * bv;
      }
    }
  }
  double vv[1] = {v};
  double tot[1];
  if (Reduce<1>::run(pkb, blockIdx.x, fb.inst, vv, partial, ticket, tot) && threadIdx.x == 0)
    bbf[fb.inst] = tot[0];
}

// red pass: Tr = E x (the red rows' coupling to black values x); every
// instance when ks is null, else only those still iterating
template <int DIM>
__global__ void __launch_bounds__(NT, 5)
k_rb_red(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ JR,
         const double* __restrict__ x, double* __restrict__ Tr, const KState* ks,
         const int32_t* __restrict__ blk) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pkb, fbi);
  if (ks && !ks[fb.inst].active) return;
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes;
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    const RbNode q = rb_node(g, slot, 0);
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    if (q.real) {
      int m[6];
      rb_nbrs<DIM>(g, q, (int)(slot - g.soff), m);
      rb_couple<DIM>(JR, x + g.soff, slot, NS, m, y0, y1, y2);
    }
    Tr[slot] = y0; Tr[NS + slot] = y1; Tr[2 * NS + slot] = y2;
  }
}

// black pass at one slot: y = x_b - F Tr (0 at a pad)
template <int DIM>
__device__ __forceinline__ void rb_black(const RbGeo& g, const double* __restrict__ JB,
                                         const double* __restrict__ Tr,
                                         const double* __restrict__ X, int64_t slot,
                                         int64_t NS, double& y0, double& y1, double& y2) {
  const RbNode q = rb_node(g, slot, 1);
  y0 = 0.0; y1 = 0.0; y2 = 0.0;
  if (!q.real) return;
  int m[6];
  rb_nbrs<DIM>(g, q, (int)(slot - g.soff), m);
  double u0, u1, u2;
  rb_couple<DIM>(JB, Tr + g.soff, slot, NS, m, u0, u1, u2);
  y0 = X[slot] - u0;
  y1 = X[NS + slot] - u1;
  y2 = X[2 * NS + slot] - u2;
}

// Schur right-hand side and BiCGStab start: rhs = bB - F bR; x = 0,
// r = rh = rhs, p = v = 0; the tolerance is on the full ||b|| (bbf)
template <int DIM>
__global__ void __launch_bounds__(NT, 3)
k_rb_init(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ JB,
          const double* __restrict__ bR, const double* __restrict__ bB,
          double* __restrict__ rhs, double* __restrict__ x, BiVec w,
          const double* __restrict__ bbf, KState* ks, double* partial, unsigned* ticket,
          double rtol, int maxit, const int32_t* __restrict__ pre_status,
          const double* __restrict__ rtol_inst) {
  const FlatBlock fb = flat_block(pkb, blockIdx.x);
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes;
  double v = 0.0;
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    double y[3];
    rb_black<DIM>(g, JB, bR, bB, slot, NS, y[0], y[1], y[2]);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t q = c * NS + slot;
      rhs[q] = y[c];
      x[q] = 0.0; w.r[q] = y[c]; w.rh[q] = y[c]; w.p[q] = 0.0; w.v[q] = 0.0;
      v += y[c] * y[c];
    }
  }
  double vv[1] = {v};
  double tot[1];
  if (Reduce<1>::run(pkb, blockIdx.x, fb.inst, vv, partial, ticket, tot) &&
      threadIdx.x == 0) {
    KState& s = ks[fb.inst];
    const double rt = rtol_inst ? rtol_inst[fb.inst] : rtol;
    fin_init(s, tot[0], rt, maxit, pre_status ? pre_status[fb.inst] : TCAD_OK);
    const double bb = bbf[fb.inst];
    s.bb = bb;
    s.tol2 = rt * rt * bb;
    if (s.status == TCAD_OK && !isfinite(bb)) {
      s.status = TCAD_ERR_NONFINITE;
      s.active = 0;
    }
  }
}

// v = S p (S = I - F E; Tr = E p from the red pass); (rh, v)
template <int DIM>
__global__ void __launch_bounds__(NT, 5)
k_rb_v(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ JB,
       const double* __restrict__ Tr, BiVec w, KState* ks, double* partial, unsigned* ticket,
       const int32_t* __restrict__ blk) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pkb, fbi);
  if (!ks[fb.inst].active) return;
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes;
  const double* __restrict__ RH = w.rh;
  double* __restrict__ Vo = w.v;
  double v = 0.0;
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    double y0, y1, y2;
    rb_black<DIM>(g, JB, Tr, w.p, slot, NS, y0, y1, y2);
    const double h0 = RH[slot], h1 = RH[NS + slot], h2 = RH[2 * NS + slot];
    Vo[slot] = y0; Vo[NS + slot] = y1; Vo[2 * NS + slot] = y2;
    v += h0 * y0 + h1 * y1 + h2 * y2;
  }
  double vv[1] = {v};
  double tot[1];
  if (Reduce<1>::run(pkb, fbi, fb.inst, vv, partial, ticket, tot) && threadIdx.x == 0)
    fin_v(ks[fb.inst], tot[0]);
}

// t = S s (Tr = E s); (t, s), (t, t)
template <int DIM>
__global__ void __launch_bounds__(NT, 5)
k_rb_t(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ JB,
       const double* __restrict__ Tr, BiVec w, KState* ks, double* partial, unsigned* ticket,
       const int32_t* __restrict__ blk) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pkb, fbi);
  if (!ks[fb.inst].active) return;
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes;
  const double* __restrict__ S = w.s;
  double* __restrict__ To = w.t;
  double v[2] = {0.0, 0.0};
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    double y0, y1, y2;
    rb_black<DIM>(g, JB, Tr, S, slot, NS, y0, y1, y2);
    const double s0 = S[slot], s1 = S[NS + slot], s2 = S[2 * NS + slot];
    To[slot] = y0; To[NS + slot] = y1; To[2 * NS + slot] = y2;
    v[0] += y0 * s0 + y1 * s1 + y2 * s2;
    v[1] += y0 * y0 + y1 * y1 + y2 * y2;
  }
  double tot[2];
  if (Reduce<2>::run(pkb, fbi, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0)
    fin_t(ks[fb.inst], tot[0], tot[1]);
}

// true Schur residual r = rhs - S x (Tr = E x), which is the black part of
// the full residual (its red part is zero); (r, r); re-arm as k_true_resid
template <int DIM>
__global__ void __launch_bounds__(NT, 3)
k_rb_true(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ JB,
          const double* __restrict__ Tr, const double* __restrict__ rhs,
          const double* __restrict__ x, double* __restrict__ r, KState* ks, double* partial,
          unsigned* ticket, int rearm) {
  const FlatBlock fb = flat_block(pkb, blockIdx.x);
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes;
  double v = 0.0;
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    double y[3];
    rb_black<DIM>(g, JB, Tr, x, slot, NS, y[0], y[1], y[2]);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double a = rhs[c * NS + slot] - y[c];
      r[c * NS + slot] = a;
      v += a * a;
    }
  }
  double vv[1] = {v};
  double tot[1];
  if (Reduce<1>::run(pkb, blockIdx.x, fb.inst, vv, partial, ticket, tot) && threadIdx.x == 0)
    fin_true(ks[fb.inst], tot[0], rearm);
}

// full solution: x_r = bR - Tr (Tr = E x_b), x_b; zero for the instances
// whose pre-status kept them idle
template <int DIM>
__global__ void __launch_bounds__(NT)
k_rb_merge(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ bR,
           const double* __restrict__ Tr, const double* __restrict__ xb,
           double* __restrict__ x, const int32_t* __restrict__ pre_status) {
  const FlatBlock fb = flat_block(pkb, blockIdx.x);
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes, NN = mp.n_full;
  const bool idle = pre_status && pre_status[fb.inst] != TCAD_OK;
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    const RbNode qr = rb_node(g, slot, 0);
    const RbNode qb = rb_node(g, slot, 1);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t q = c * NS + slot;
      if (qr.real) x[c * NN + qr.node] = idle ? 0.0 : bR[q] - Tr[q];
      if (qb.real) x[c * NN + qb.node] = idle ? 0.0 : xb[q];
    }
  }
}

}  // namespace tcad
