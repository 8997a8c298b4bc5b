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
// iteration are held to 5 CTAs per SM (48 registers; the t pass spills 72
// bytes): they are latency-bound -- under ncu the 3-CTA black pass waited 33
// long-scoreboard stalls per issue at 34 % warps active, DRAM 33 % busy --
// and a two-lane tri-gate iteration went from 511 us at 4 CTAs to 419 at 5
// (about 410 with J in warp tiles).
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
// coupling part of A^ on the other colour's values X(m, c), m instance-local
template <int DIM, class XF>
__device__ __forceinline__ void rb_couple_f(const double* __restrict__ Jc, const XF& X,
                                            int64_t slot, const int* m, double& y0,
                                            double& y1, double& y2) {
  constexpr int NE = Stencil<DIM>::NE;
  const double* __restrict__ Jt = Jc + rb_jidx<NE>(0, slot);   // entry e at Jt[32 e]
  double t0 = 0.0, t1 = 0.0, t2 = 0.0;
#pragma unroll
  for (int d = 0; d < 2 * DIM; ++d) {
    const int e = 9 + 5 * d;
    const double xs = X(m[d], 0), xn = X(m[d], 1), xp = X(m[d], 2);
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

// a stored vector of the other colour (xi: from the instance's first slot)
struct RbVal {
  const double* __restrict__ xi;
  int64_t NS;
  __device__ __forceinline__ double operator()(int m, int c) const { return xi[c * NS + m]; }
};

// The search direction p = r + beta (p - omega v) (p = r on a restart) and
// s = r - alpha v formed on the fly at the other colour's slots, from vectors
// no CTA writes meanwhile -- the expressions of bi_p_body and bi_s_body (the
// single-launch solve forms them where the per-step solve stores them)
struct RbFormP {
  const double* __restrict__ r;
  const double* __restrict__ p;
  const double* __restrict__ v;
  int64_t NS;
  double beta, omega;
  int restart;
  __device__ __forceinline__ double operator()(int m, int c) const {
    const double rv = r[c * NS + m];
    return restart ? rv : rv + beta * (p[c * NS + m] - omega * v[c * NS + m]);
  }
};
struct RbFormS {
  const double* __restrict__ r;
  const double* __restrict__ v;
  int64_t NS;
  double alpha;
  __device__ __forceinline__ double operator()(int m, int c) const {
    return r[c * NS + m] - alpha * v[c * NS + m];
  }
};

template <int DIM>
__device__ __forceinline__ void rb_couple(const double* __restrict__ Jc,
                                          const double* __restrict__ xi, int64_t slot,
                                          int64_t NS, const int* m, double& y0, double& y1,
                                          double& y2) {
  rb_couple_f<DIM>(Jc, RbVal{xi, NS}, slot, m, y0, y1, y2);
}

// ---- per-block bodies, shared by the per-step kernels below and the
// single-launch solve (k_bicgstab_rb_fused), so both run the same
// arithmetic in the same order

// bR, bB <- the colours of b at the block's slots; returns the thread's
// share of (b, b)
template <int DIM>
__device__ __forceinline__ double rb_split_body(const tcad_pack_t& pkb, const RbMap& mp,
                                                const FlatBlock& fb,
                                                const double* __restrict__ b,
                                                double* __restrict__ bR,
                                                double* __restrict__ bB) {
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
  return v;
}

// black pass coupling at one slot: u = F Tr; false at a pad (u = 0).  The
// callers load the slot's own vectors after it (y = X - u), which keeps them
// out of the registers the gathers need.
template <int DIM>
__device__ __forceinline__ bool rb_black_u(const RbGeo& g, const double* __restrict__ JB,
                                           const double* __restrict__ Tr, int64_t slot,
                                           int64_t NS, double* u) {
  const RbNode q = rb_node(g, slot, 1);
  u[0] = 0.0; u[1] = 0.0; u[2] = 0.0;
  if (!q.real) return false;
  int m[6];
  rb_nbrs<DIM>(g, q, (int)(slot - g.soff), m);
  rb_couple<DIM>(JB, Tr + g.soff, slot, NS, m, u[0], u[1], u[2]);
  return true;
}

// rhs = bB - F bR; x = 0, r = rh = rhs, p = v = 0; returns (rhs, rhs) share
template <int DIM>
__device__ __forceinline__ double rb_init_body(const tcad_pack_t& pkb, const RbMap& mp,
                                               const FlatBlock& fb,
                                               const double* __restrict__ JB,
                                               const double* __restrict__ bR,
                                               const double* __restrict__ bB,
                                               double* __restrict__ rhs,
                                               double* __restrict__ x, const BiVec& w) {
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes;
  double v = 0.0;
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    double u[3];
    const bool real = rb_black_u<DIM>(g, JB, bR, slot, NS, u);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t q = c * NS + slot;
      const double y = real ? bB[q] - u[c] : 0.0;
      rhs[q] = y;
      x[q] = 0.0; w.r[q] = y; w.rh[q] = y; w.p[q] = 0.0; w.v[q] = 0.0;
      v += y * y;
    }
  }
  return v;
}

// red pass: Tr = E X at the block's red slots, X a value functor factory
// (instance base offset -> functor)
template <int DIM, class MK>
__device__ __forceinline__ void rb_red_body(const tcad_pack_t& pkb, const RbMap& mp,
                                            const FlatBlock& fb,
                                            const double* __restrict__ JR, const MK& make,
                                            double* __restrict__ Tr) {
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes;
  const auto X = make(g.soff);
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    const RbNode q = rb_node(g, slot, 0);
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    if (q.real) {
      int m[6];
      rb_nbrs<DIM>(g, q, (int)(slot - g.soff), m);
      rb_couple_f<DIM>(JR, X, slot, m, y0, y1, y2);
    }
    Tr[slot] = y0; Tr[NS + slot] = y1; Tr[2 * NS + slot] = y2;
  }
}

// v = S p (Tr = E p); FORM: p formed and stored first (p = r + beta (p -
// omega v); restart: rh = p = r), else p as stored; returns (rh, v) share
template <int DIM, bool FORM>
__device__ __forceinline__ double rb_v_body(const tcad_pack_t& pkb, const RbMap& mp,
                                            const FlatBlock& fb,
                                            const double* __restrict__ JB,
                                            const double* __restrict__ Tr, const BiVec& w,
                                            double beta, double omega, int restart) {
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes;
  double* __restrict__ P = w.p;
  double* __restrict__ RH = w.rh;
  double* __restrict__ Vo = w.v;
  const double* __restrict__ R = w.r;
  double v = 0.0;
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    double u[3];
    const bool real = rb_black_u<DIM>(g, JB, Tr, slot, NS, u);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t i = c * NS + slot;
      double pn, h;
      if (FORM) {
        const double rv = R[i];
        pn = restart ? rv : rv + beta * (P[i] - omega * Vo[i]);
        P[i] = pn;
        if (restart) RH[i] = rv;
        h = restart ? rv : RH[i];
      } else {
        pn = P[i];
        h = RH[i];
      }
      const double y = real ? pn - u[c] : 0.0;
      Vo[i] = y;
      v += h * y;
    }
  }
  return v;
}

// t = S s (Tr = E s); FORM: s = r - alpha v formed and stored first (its
// (s, s) share in v[0], accumulated as bi_s_body does), else s as stored;
// v[1] = (t, s), v[2] = (t, t) shares
template <int DIM, bool FORM>
__device__ __forceinline__ void rb_t_body(const tcad_pack_t& pkb, const RbMap& mp,
                                          const FlatBlock& fb, const double* __restrict__ JB,
                                          const double* __restrict__ Tr, const BiVec& w,
                                          double alpha, double (&v)[3]) {
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes;
  double* __restrict__ S = w.s;
  double* __restrict__ To = w.t;
  const double* __restrict__ R = w.r;
  const double* __restrict__ V = w.v;
  v[0] = 0.0; v[1] = 0.0; v[2] = 0.0;
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    double u[3];
    const bool real = rb_black_u<DIM>(g, JB, Tr, slot, NS, u);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t i = c * NS + slot;
      double sv;
      if (FORM) {
        sv = R[i] - alpha * V[i];
        v[0] += sv * sv;
        S[i] = sv;
      } else {
        sv = S[i];
      }
      const double y = real ? sv - u[c] : 0.0;
      To[i] = y;
      v[1] += y * sv;
      v[2] += y * y;
    }
  }
}

// true Schur residual r = rhs - S x (Tr = E x), the black part of the full
// residual (its red part is zero); returns (r, r) share
template <int DIM>
__device__ __forceinline__ double rb_true_body(const tcad_pack_t& pkb, const RbMap& mp,
                                               const FlatBlock& fb,
                                               const double* __restrict__ JB,
                                               const double* __restrict__ Tr,
                                               const double* __restrict__ rhs,
                                               const double* __restrict__ x,
                                               double* __restrict__ r) {
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes;
  double v = 0.0;
  for (int64_t slot = fb.begin + threadIdx.x; slot < fb.end; slot += NT) {
    double u[3];
    const bool real = rb_black_u<DIM>(g, JB, Tr, slot, NS, u);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double y = real ? x[c * NS + slot] - u[c] : 0.0;
      const double a = rhs[c * NS + slot] - y;
      r[c * NS + slot] = a;
      v += a * a;
    }
  }
  return v;
}

// full solution at the block's slots: x_r = bR - Tr (Tr = E x_b), x_b; zero
// when idle
template <int DIM>
__device__ __forceinline__ void rb_merge_body(const tcad_pack_t& pkb, const RbMap& mp,
                                              const FlatBlock& fb,
                                              const double* __restrict__ bR,
                                              const double* __restrict__ Tr,
                                              const double* __restrict__ xb,
                                              double* __restrict__ x, bool idle) {
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NS = pkb.n_nodes, NN = mp.n_full;
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

// functor factories for rb_red_body
struct RbMakeVal {
  const double* x;
  int64_t NS;
  __device__ __forceinline__ RbVal operator()(int64_t soff) const { return RbVal{x + soff, NS}; }
};
struct RbMakeP {
  const double *r, *p, *v;
  int64_t NS;
  double beta, omega;
  int restart;
  __device__ __forceinline__ RbFormP operator()(int64_t soff) const {
    return RbFormP{r + soff, p + soff, v + soff, NS, beta, omega, restart};
  }
};
struct RbMakeS {
  const double *r, *v;
  int64_t NS;
  double alpha;
  __device__ __forceinline__ RbFormS operator()(int64_t soff) const {
    return RbFormS{r + soff, v + soff, NS, alpha};
  }
};

// ---- one launch per step

// JR, JB <- the red and black rows of the block-scaled J in warp tiles
// (zeros at pads; the tile tail past the last slot is never read)
template <int DIM>
__global__ void __launch_bounds__(NT)
k_rb_pack(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ J,
          double* __restrict__ JR, double* __restrict__ JB) {
  constexpr int NE = Stencil<DIM>::NE;
  const FlatBlock fb = flat_block(pkb, blockIdx.x);
  const RbGeo g = rb_geo(pkb, mp, fb.inst);
  const int64_t NN = mp.n_full;
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
  double vv[1] = {rb_split_body<DIM>(pkb, mp, fb, b, bR, bB)};
  double tot[1];
  if (Reduce<1>::run(pkb, blockIdx.x, fb.inst, vv, partial, ticket, tot) && threadIdx.x == 0)
    bbf[fb.inst] = tot[0];
}

// the Schur start: the tolerance is on the full ||b|| (bbf)
__device__ __forceinline__ void rb_fin_init(KState& s, double tot, double bb, double rt,
                                            int maxit, int pre) {
  fin_init(s, tot, rt, maxit, pre);
  s.bb = bb;
  s.tol2 = rt * rt * bb;
  if (s.status == TCAD_OK && !isfinite(bb)) {
    s.status = TCAD_ERR_NONFINITE;
    s.active = 0;
  }
}

template <int DIM>
__global__ void __launch_bounds__(NT, 3)
k_rb_init(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ JB,
          const double* __restrict__ bR, const double* __restrict__ bB,
          double* __restrict__ rhs, double* __restrict__ x, BiVec w,
          const double* __restrict__ bbf, KState* ks, double* partial, unsigned* ticket,
          double rtol, int maxit, const int32_t* __restrict__ pre_status,
          const double* __restrict__ rtol_inst) {
  const FlatBlock fb = flat_block(pkb, blockIdx.x);
  double vv[1] = {rb_init_body<DIM>(pkb, mp, fb, JB, bR, bB, rhs, x, w)};
  double tot[1];
  if (Reduce<1>::run(pkb, blockIdx.x, fb.inst, vv, partial, ticket, tot) && threadIdx.x == 0)
    rb_fin_init(ks[fb.inst], tot[0], bbf[fb.inst], rtol_inst ? rtol_inst[fb.inst] : rtol,
                maxit, pre_status ? pre_status[fb.inst] : TCAD_OK);
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
  rb_red_body<DIM>(pkb, mp, fb, JR, RbMakeVal{x, pkb.n_nodes}, Tr);
}

// v = S p (Tr = E p from the red pass); (rh, v)
template <int DIM>
__global__ void __launch_bounds__(NT, 5)
k_rb_v(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ JB,
       const double* __restrict__ Tr, BiVec w, KState* ks, double* partial, unsigned* ticket,
       const int32_t* __restrict__ blk) {
  const int64_t fbi = blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x;
  const FlatBlock fb = flat_block(pkb, fbi);
  if (!ks[fb.inst].active) return;
  double vv[1] = {rb_v_body<DIM, false>(pkb, mp, fb, JB, Tr, w, 0.0, 0.0, 0)};
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
  double v3[3];
  rb_t_body<DIM, false>(pkb, mp, fb, JB, Tr, w, 0.0, v3);
  double v[2] = {v3[1], v3[2]};
  double tot[2];
  if (Reduce<2>::run(pkb, fbi, fb.inst, v, partial, ticket, tot) && threadIdx.x == 0)
    fin_t(ks[fb.inst], tot[0], tot[1]);
}

// true Schur residual; (r, r); re-arm as k_true_resid
template <int DIM>
__global__ void __launch_bounds__(NT, 3)
k_rb_true(const tcad_pack_t pkb, const RbMap mp, const double* __restrict__ JB,
          const double* __restrict__ Tr, const double* __restrict__ rhs,
          const double* __restrict__ x, double* __restrict__ r, KState* ks, double* partial,
          unsigned* ticket, int rearm) {
  const FlatBlock fb = flat_block(pkb, blockIdx.x);
  double vv[1] = {rb_true_body<DIM>(pkb, mp, fb, JB, Tr, rhs, x, r)};
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
  rb_merge_body<DIM>(pkb, mp, fb, bR, Tr, xb, x,
                     pre_status && pre_status[fb.inst] != TCAD_OK);
}

}  // namespace tcad
