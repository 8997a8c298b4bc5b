// Fused SG residual/Jacobian assembly (coupled psi/n/p) and the equilibrium
// Poisson assembly, written straight into the fixed node-block layout of
// include/tcad_b200.h.  Built with -fmad=false (see sg_edge.cuh).
//
// One CTA owns a 32 x 8 tile of nodes (x fastest, so a warp is one row of 32
// consecutive nodes and every node-array access is a coalesced 256-byte
// line).  The tile's plane values plus a one-node halo are staged in shared
// memory; every x- and y-edge touching the tile is evaluated ONCE (Bernoulli
// functions included) into shared memory and read by both endpoint nodes.
// In 3D the CTA marches up to pk.tile_z planes in z, carrying the z-edge
// between consecutive planes in registers (the up-edge of plane k is the
// down-edge of plane k+1), so z-edges are also evaluated once.
#include "sg_edge.cuh"

namespace tcad {

constexpr int TX = TCAD_TILE_X, TY = TCAD_TILE_Y;

struct NodeVals {
  double psi, n, p;
};

// Neighbour-block entry offsets: 9 + 5*d + m.
__device__ __forceinline__ int nb(int d, int m) { return 9 + 5 * d + m; }

// ---- asynchronous staging of a z-plane's coefficients (3D, asm_stage = 1)
// The coefficients one plane of a tile reads -- an, ap, dl of every x- and
// y-edge touching the tile and of each node's up z-edge, and C, n_ie, tau_n,
// tau_p of each node -- are copied global -> shared with cp.async (8 bytes
// per copy, coalesced across the warp, zero-filled where the edge or node
// does not exist) one plane AHEAD: while plane k computes, plane k+1's
// copies are in flight, so the compute phase reads shared memory instead of
// waiting on global loads.  The values are the same, so the arithmetic and
// its result are bit-identical to the unstaged kernel.
struct PlaneStage {
  double ax[3][TY][TX + 1];  // x-edge slot a of row r: edge (i0-1+a, j0+r) -> +x
  double ay[3][TY + 1][TX];  // y-edge slot b of column c: edge (i0+c, j0-1+b) -> +y
  double az[3][TY][TX];      // own node's edge -> +z
  double nd[4][TY][TX];      // own node's C, n_ie, tau_n, tau_p
};
constexpr int kStageBytes = 2 * (int)sizeof(PlaneStage);

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid,
                                          const double* dummy) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d),
               "l"(valid ? src : dummy), "r"(n)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_one() {
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

// CTAs per SM the coupled assembly is compiled for (register budget):
// 4 in 2D (64 registers, no spills), 3 in 3D (80 registers; the z-march
// carries two edges and two node states in registers, and at 64 registers
// the spills cost more than the fourth CTA gains)
template <int DIM, bool STAGED>
__global__ void __launch_bounds__(kTileThreads, DIM == 2 ? 4 : (STAGED ? 2 : 3))
k_sg_assemble(const tcad_pack_t pk, const double* __restrict__ psi,
              const double* __restrict__ nn, const double* __restrict__ pp,
              double* __restrict__ F, double* __restrict__ J, int mode,
              const int32_t* __restrict__ tiles) {
  static_assert(DIM == 3 || !STAGED, "plane staging is the 3D z-march's");
  constexpr int NE = DIM == 2 ? TCAD_NE2 : TCAD_NE3;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  PlaneStage* const stage = reinterpret_cast<PlaneStage*>(s_dyn);
  __shared__ double s_psi[TY + 2][TX + 2], s_n[TY + 2][TX + 2], s_p[TY + 2][TX + 2];
  __shared__ uint8_t s_flag[TY + 2][TX + 2];
  __shared__ Edge s_ex[TY][TX + 1];  // x-edge slot a: nodes (i0-1+a, i0+a)
  __shared__ Edge s_ey[TY + 1][TX];  // y-edge slot b: nodes (j0-1+b, j0+b)

  const int64_t t = tiles ? (int64_t)tiles[blockIdx.x] : (int64_t)blockIdx.x;
  const int inst = pk.tile[4 * t + 0], i0 = pk.tile[4 * t + 1];
  const int j0 = pk.tile[4 * t + 2], k0 = pk.tile[4 * t + 3];
  const Inst g = load_inst(pk, inst);
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int i = i0 + tx, j = j0 + ty;
  const bool own = (i < g.nx) && (j < g.ny);
  const int64_t ax0 = pk.axis_off[3 * inst], ay0 = pk.axis_off[3 * inst + 1];
  const int64_t az0 = pk.axis_off[3 * inst + 2];
  const int64_t sxy = (int64_t)g.nx * g.ny;
  const int64_t NN = pk.n_nodes;
  const double* par = pk.par + TCAD_NPAR * inst;
  const int kend = DIM == 3 ? min(k0 + pk.tile_z, g.nz) : 1;

  // z-march registers (3D): own node values of the current / next plane
  NodeVals cur{0.0, 0.0, 0.0}, nxt{0.0, 0.0, 0.0};
  Edge eD, eU;
  zero_edge(eD);
  zero_edge(eU);
  if (own) {
    const int64_t q = g.off + (int64_t)k0 * sxy + (int64_t)j * g.nx + i;
    cur = NodeVals{psi[q], nn[q], pp[q]};
  }
  if (DIM == 3 && own && k0 > 0) {  // down-edge into the first plane
    const int64_t q = g.off + (int64_t)k0 * sxy + (int64_t)j * g.nx + i;
    const int64_t ql = q - sxy;
    sg_edge(psi[ql], cur.psi, nn[ql], cur.n, pp[ql], cur.p, pk.an[2][ql], pk.ap[2][ql],
            pk.dl[2][ql], pk.h[2][az0 + k0 - 1], eD);
  }

  // this thread's share of plane kz's staging copies into buffer st: its own
  // node's x-, y- and z-edge coefficients and node data, and (threads 0..7 /
  // 8..39) the tile's west x-edge / south y-edge halo
  auto issue = [&](int kz, PlaneStage* sb) {
    const int64_t pl = g.off + (int64_t)kz * sxy;
    const double* const dmy = pk.C;
    const bool xv = (i + 1 < g.nx) && (j < g.ny);
    const bool yv = (j + 1 < g.ny) && (i < g.nx);
    const bool zv = own && (kz + 1 < g.nz);
    const int64_t q = pl + (int64_t)j * g.nx + i;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double* const* arr = c == 0 ? pk.an : (c == 1 ? pk.ap : pk.dl);
      cp_async8(&sb->ax[c][ty][tx + 1], arr[0] + q, xv, dmy);
      cp_async8(&sb->ay[c][ty + 1][tx], arr[1] + q, yv, dmy);
      cp_async8(&sb->az[c][ty][tx], arr[2] + q, zv, dmy);
    }
    cp_async8(&sb->nd[0][ty][tx], pk.C + q, own, dmy);
    cp_async8(&sb->nd[1][ty][tx], pk.nie + q, own, dmy);
    cp_async8(&sb->nd[2][ty][tx], pk.tau_n + q, own, dmy);
    cp_async8(&sb->nd[3][ty][tx], pk.tau_p + q, own, dmy);
    if (tid < TY) {                        // west halo: edge (i0-1, j0+tid) -> +x
      const int r = tid, jj = j0 + r;
      const bool v = i0 >= 1 && i0 < g.nx && jj < g.ny;
      const int64_t qh = pl + (int64_t)jj * g.nx + (i0 - 1);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double* const* arr = c == 0 ? pk.an : (c == 1 ? pk.ap : pk.dl);
        cp_async8(&sb->ax[c][r][0], arr[0] + qh, v, dmy);
      }
    } else if (tid < TY + TX) {            // south halo: edge (i0+col, j0-1) -> +y
      const int col = tid - TY, ii = i0 + col;
      const bool v = j0 >= 1 && j0 < g.ny && ii < g.nx;
      const int64_t qh = pl + (int64_t)(j0 - 1) * g.nx + ii;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double* const* arr = c == 0 ? pk.an : (c == 1 ? pk.ap : pk.dl);
        cp_async8(&sb->ay[c][0][col], arr[1] + qh, v, dmy);
      }
    }
    cp_async_commit();
  };
  if constexpr (STAGED) issue(k0, &stage[0]);

  for (int kz = k0; kz < kend; ++kz) {
    const int64_t plane = g.off + (int64_t)kz * sxy;
    PlaneStage* const stg = STAGED ? &stage[(kz - k0) & 1] : nullptr;
    if constexpr (STAGED) {
      // the buffer it fills was last read before the previous plane's final
      // barrier; an empty group keeps the wait count uniform at the last plane
      if (kz + 1 < kend) issue(kz + 1, &stage[(kz + 1 - k0) & 1]);
      else cp_async_commit();
    }
    // ---- stage the plane (tile + 1-node halo, no corners) in shared memory
    s_psi[ty + 1][tx + 1] = cur.psi;
    s_n[ty + 1][tx + 1] = cur.n;
    s_p[ty + 1][tx + 1] = cur.p;
    s_flag[ty + 1][tx + 1] = own ? pk.bcflag[plane + (int64_t)j * g.nx + i] : 0;
    if (tid < 2 * TY + 2 * TX) {
      int r, c, hi, hj;
      if (tid < 2 * TY) {  // x halo: columns 0 and TX+1
        r = 1 + (tid >> 1);
        c = (tid & 1) ? TX + 1 : 0;
      } else {             // y halo: rows 0 and TY+1
        const int u = tid - 2 * TY;
        c = 1 + (u >> 1);
        r = (u & 1) ? TY + 1 : 0;
      }
      hi = i0 - 1 + c;
      hj = j0 - 1 + r;
      double a = 0.0, b = 0.0, d = 0.0;
      uint8_t f = 0;
      if (hi >= 0 && hi < g.nx && hj >= 0 && hj < g.ny) {
        const int64_t q = plane + (int64_t)hj * g.nx + hi;
        a = psi[q]; b = nn[q]; d = pp[q]; f = pk.bcflag[q];
      }
      s_psi[r][c] = a; s_n[r][c] = b; s_p[r][c] = d; s_flag[r][c] = f;
    }
    if (DIM == 3 && own && kz + 1 < g.nz) {
      const int64_t q = plane + sxy + (int64_t)j * g.nx + i;
      nxt = NodeVals{psi[q], nn[q], pp[q]};
    }
    if constexpr (STAGED) cp_async_wait_one();   // this plane's copies (own thread)
    __syncthreads();

    // ---- evaluate every edge touching the tile once
    auto xedge = [&](int row, int a) {
      const int ilo = i0 - 1 + a, jj = j0 + row;
      Edge e;
      if (ilo >= 0 && ilo + 1 < g.nx && jj < g.ny) {
        const int64_t q = plane + (int64_t)jj * g.nx + ilo;
        double an, ap, dl;
        if constexpr (STAGED) {
          an = stg->ax[0][row][a]; ap = stg->ax[1][row][a]; dl = stg->ax[2][row][a];
        } else {
          an = pk.an[0][q]; ap = pk.ap[0][q]; dl = pk.dl[0][q];
        }
        sg_edge(s_psi[row + 1][a], s_psi[row + 1][a + 1], s_n[row + 1][a],
                s_n[row + 1][a + 1], s_p[row + 1][a], s_p[row + 1][a + 1], an, ap, dl,
                pk.h[0][ax0 + ilo], e);
      } else {
        zero_edge(e);
      }
      s_ex[row][a] = e;
    };
    auto yedge = [&](int col, int b) {
      const int jlo = j0 - 1 + b, ii = i0 + col;
      Edge e;
      if (jlo >= 0 && jlo + 1 < g.ny && ii < g.nx) {
        const int64_t q = plane + (int64_t)jlo * g.nx + ii;
        double an, ap, dl;
        if constexpr (STAGED) {
          an = stg->ay[0][b][col]; ap = stg->ay[1][b][col]; dl = stg->ay[2][b][col];
        } else {
          an = pk.an[1][q]; ap = pk.ap[1][q]; dl = pk.dl[1][q];
        }
        sg_edge(s_psi[b][col + 1], s_psi[b + 1][col + 1], s_n[b][col + 1],
                s_n[b + 1][col + 1], s_p[b][col + 1], s_p[b + 1][col + 1], an, ap, dl,
                pk.h[1][ay0 + jlo], e);
      } else {
        zero_edge(e);
      }
      s_ey[b][col] = e;
    };
    xedge(ty, tx + 1);  // own E edge
    yedge(tx, ty + 1);  // own N edge
    if (tid < TY) xedge(tid, 0);                        // tile's west halo edges
    else if (tid < TY + TX) yedge(tid - TY, 0);         // tile's south halo edges
    if (DIM == 3) {
      if (own && kz + 1 < g.nz) {
        const int64_t q = plane + (int64_t)j * g.nx + i;
        double an, ap, dl;
        if constexpr (STAGED) {
          an = stg->az[0][ty][tx]; ap = stg->az[1][ty][tx]; dl = stg->az[2][ty][tx];
        } else {
          an = pk.an[2][q]; ap = pk.ap[2][q]; dl = pk.dl[2][q];
        }
        sg_edge(cur.psi, nxt.psi, cur.n, nxt.n, cur.p, nxt.p, an, ap, dl,
                pk.h[2][az0 + kz], eU);
      } else {
        zero_edge(eU);
      }
    }
    __syncthreads();

    // ---- assemble the own node's row block.  Each neighbour block is
    // streamed to HBM as soon as it is known (no per-node entry array in
    // registers, so several tiles stay resident per SM).
    if (own) {
      const int64_t k = plane + (int64_t)j * g.nx + i;
      const uint8_t flag = s_flag[ty + 1][tx + 1];
      double* __restrict__ Jk = J + k;
      auto st = [&](int e, double v) { Jk[(int64_t)e * NN] = v; };
      if ((flag & TCAD_BC_CONTACT) && mode != TCAD_MODE_UNSTAMPED) {
        F[k] = cur.psi - pk.bc_psi0[k];
        F[NN + k] = cur.n - pk.bc_n0[k];
        F[2 * NN + k] = cur.p - pk.bc_p0[k];
#pragma unroll
        for (int e = 0; e < NE; ++e) st(e, (e == 0 || e == 4 || e == 8) ? 1.0 : 0.0);
      } else {
        const double dvx = pk.dv[0][ax0 + i], dvy = pk.dv[1][ay0 + j];
        const double dvz = DIM == 3 ? pk.dv[2][az0 + kz] : 1.0;
        const double fx = DIM == 2 ? dvy : dvy * dvz;   // x-edge face
        const double fy = DIM == 2 ? dvx : dvx * dvz;   // y-edge face
        const double fz = dvx * dvy;                    // z-edge face
        const double dV = DIM == 2 ? dvy * dvx : (dvz * dvy) * dvx;
        const bool vW = i >= 1, vE = i + 1 < g.nx, vS = j >= 1, vN = j + 1 < g.ny;
        const bool vD = DIM == 3 && kz >= 1, vU = DIM == 3 && kz + 1 < g.nz;
        const Edge& W = s_ex[ty][tx];
        const Edge& E = s_ex[ty][tx + 1];
        const Edge& S = s_ey[ty][tx];
        const Edge& N = s_ey[ty + 1][tx];
        const double hW = vW ? pk.h[0][ax0 + i - 1] : 1.0, hE = vE ? pk.h[0][ax0 + i] : 1.0;
        const double hS = vS ? pk.h[1][ay0 + j - 1] : 1.0, hN = vN ? pk.h[1][ay0 + j] : 1.0;
        const double hD = vD ? pk.h[2][az0 + kz - 1] : 1.0, hU = vU ? pk.h[2][az0 + kz] : 1.0;
        // divergences: div[lo] += f; div[hi] -= f  (device2d.py:1512-1525)
        double f0, f1, f2;
        {
          double dx0 = 0.0, dx1 = 0.0, dx2 = 0.0, dy0 = 0.0, dy1 = 0.0, dy2 = 0.0;
          if (vE) { dx0 = dx0 + E.f; dx1 = dx1 + E.Jn; dx2 = dx2 + E.Jp; }
          if (vW) { dx0 = dx0 - W.f; dx1 = dx1 - W.Jn; dx2 = dx2 - W.Jp; }
          if (vN) { dy0 = dy0 + N.f; dy1 = dy1 + N.Jn; dy2 = dy2 + N.Jp; }
          if (vS) { dy0 = dy0 - S.f; dy1 = dy1 - S.Jn; dy2 = dy2 - S.Jp; }
          f0 = fx * dx0 + fy * dy0;
          f1 = fx * dx1 + fy * dy1;
          f2 = fx * dx2 + fy * dy2;
          if (DIM == 3) {
            double dz0 = 0.0, dz1 = 0.0, dz2 = 0.0;
            if (vU) { dz0 = dz0 + eU.f; dz1 = dz1 + eU.Jn; dz2 = dz2 + eU.Jp; }
            if (vD) { dz0 = dz0 - eD.f; dz1 = dz1 - eD.Jn; dz2 = dz2 - eD.Jp; }
            f0 = f0 + fz * dz0; f1 = f1 + fz * dz1; f2 = f2 + fz * dz2;
          }
        }
        double Rs, dRsn, dRsp;
        double Ck, niek, tnk, tpk;
        if constexpr (STAGED) {
          Ck = stg->nd[0][ty][tx]; niek = stg->nd[1][ty][tx];
          tnk = stg->nd[2][ty][tx]; tpk = stg->nd[3][ty][tx];
        } else {
          Ck = pk.C[k]; niek = pk.nie[k]; tnk = pk.tau_n[k]; tpk = pk.tau_p[k];
        }
        recomb(cur.n, cur.p, niek, tnk, tpk, par, Rs, dRsn, dRsp);
        double F0 = f0 - dV * (cur.n - cur.p - Ck);
        double F1 = f1 - Rs * dV;
        double F2 = f2 + Rs * dV;
        // diagonal block, summed in the reference's stamp order per axis
        // (low-role edge first, then high-role edge)
        double d00 = 0.0, d10 = 0.0, d11 = 0.0, d20 = 0.0, d22 = 0.0;
        auto lo_role = [&](const Edge& e, double face, double h) {  // node = low end
          d00 = d00 + (-(face / h));
          d10 = d10 + (-(face * e.npsi));
          d11 = d11 + face * e.nlo;
          d20 = d20 + (-(face * e.ppsi));
          d22 = d22 + face * e.plo;
        };
        auto hi_role = [&](const Edge& e, double face, double h) {  // node = high end
          d00 = d00 + (-(face / h));
          d10 = d10 + (-(face * e.npsi));
          d11 = d11 + (-face) * e.nhi;
          d20 = d20 + (-(face * e.ppsi));
          d22 = d22 + (-face) * e.phi;
        };
        if (vE) lo_role(E, fx, hE);
        if (vW) hi_role(W, fx, hW);
        if (vN) lo_role(N, fy, hN);
        if (vS) hi_role(S, fy, hS);
        if (DIM == 3) {
          if (vU) lo_role(eU, fz, hU);
          if (vD) hi_role(eD, fz, hD);
        }
        d11 = d11 + (-dRsn) * dV;
        d22 = d22 + dRsp * dV;
        if (flag & TCAD_BC_GATE) {  // oxide Robin term (device2d.py:1624-1637)
          const double gk = pk.gate_k[k];
          F0 = F0 + gk * (pk.gate_v[k] - (cur.psi - pk.gate_b[k]));
          d00 = d00 + (-gk);
        }
        st(0, d00); st(1, -dV); st(2, dV);
        st(3, d10); st(4, d11); st(5, (-dRsp) * dV);
        st(6, d20); st(7, dRsn * dV); st(8, d22);
        // off-diagonal blocks, W,E,S,N,D,U; in ELIMINATE mode a contact
        // neighbour's known update is folded into F and its block emptied
        const bool elim = mode == TCAD_MODE_ELIMINATE;
        auto emit = [&](int d, bool valid, bool lo_end, const Edge& e, double face, double h,
                        uint8_t nflag, int64_t m) {
          double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0;
          if (valid) {
            a0 = face / h;
            a1 = face * e.npsi;
            a3 = face * e.ppsi;
            if (lo_end) { a2 = face * e.nhi; a4 = face * e.phi; }          // nbr = high end
            else { a2 = (-face) * e.nlo; a4 = (-face) * e.plo; }           // nbr = low end
            if (elim && (nflag & TCAD_BC_CONTACT)) {
              const double g0 = psi[m] - pk.bc_psi0[m];
              const double g1 = nn[m] - pk.bc_n0[m];
              const double g2 = pp[m] - pk.bc_p0[m];
              F0 = F0 - a0 * g0;
              F1 = F1 - (a1 * g0 + a2 * g1);
              F2 = F2 - (a3 * g0 + a4 * g2);
              a0 = a1 = a2 = a3 = a4 = 0.0;
            }
          }
          st(nb(d, 0), a0); st(nb(d, 1), a1); st(nb(d, 2), a2); st(nb(d, 3), a3);
          st(nb(d, 4), a4);
        };
        emit(0, vW, false, W, fx, hW, s_flag[ty + 1][tx], k - 1);
        emit(1, vE, true, E, fx, hE, s_flag[ty + 1][tx + 2], k + 1);
        emit(2, vS, false, S, fy, hS, s_flag[ty][tx + 1], k - g.nx);
        emit(3, vN, true, N, fy, hN, s_flag[ty + 2][tx + 1], k + g.nx);
        if (DIM == 3) {
          emit(4, vD, false, eD, fz, hD, vD ? pk.bcflag[k - sxy] : 0, k - sxy);
          emit(5, vU, true, eU, fz, hU, vU ? pk.bcflag[k + sxy] : 0, k + sxy);
        }
        F[k] = F0;
        F[NN + k] = F1;
        F[2 * NN + k] = F2;
      }
    }
    __syncthreads();
    if (DIM == 3) {
      cur = nxt;
      eD = eU;
    }
  }
}

// ---------------------------------------------------------------------------
// raw continuity residual F_n + F_p at listed nodes (terminal currents)
template <int DIM>
__global__ void k_contact_current(const tcad_pack_t pk, const double* __restrict__ psi,
                                  const double* __restrict__ nn,
                                  const double* __restrict__ pp,
                                  const int64_t* __restrict__ nodes, int64_t count,
                                  double* __restrict__ out) {
  // out[t] = raw F_n, out[count + t] = raw F_p of node nodes[t]
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const int64_t k = nodes[t];
  // locate the instance by a binary search on node_off
  int lo = 0, hi = pk.n_inst;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pk.node_off[mid] <= k) lo = mid; else hi = mid;
  }
  const Inst g = load_inst(pk, lo);
  const int64_t loc = k - g.off;
  const int64_t sxy = (int64_t)g.nx * g.ny;
  const int i = (int)(loc % g.nx), j = (int)((loc / g.nx) % g.ny);
  const int kz = DIM == 3 ? (int)(loc / sxy) : 0;
  const int64_t ax0 = pk.axis_off[3 * lo], ay0 = pk.axis_off[3 * lo + 1];
  const int64_t az0 = pk.axis_off[3 * lo + 2];
  const double* par = pk.par + TCAD_NPAR * lo;
  const double dvx = pk.dv[0][ax0 + i], dvy = pk.dv[1][ay0 + j];
  const double dvz = DIM == 3 ? pk.dv[2][az0 + kz] : 1.0;
  const double face[3] = {DIM == 2 ? dvy : dvy * dvz, DIM == 2 ? dvx : dvx * dvz, dvx * dvy};
  const double dV = DIM == 2 ? dvy * dvx : (dvz * dvy) * dvx;
  const int coord[3] = {i, j, kz};
  const int extent[3] = {g.nx, g.ny, g.nz};
  const int64_t stride[3] = {1, g.nx, sxy};
  const int64_t aoff[3] = {ax0, ay0, az0};
  double tn = 0.0, tp = 0.0;
  for (int a = 0; a < DIM; ++a) {
    double dn = 0.0, dp = 0.0;
    if (coord[a] + 1 < extent[a]) {  // edge to the high neighbour (node = low end)
      const int64_t m = k + stride[a];
      Edge e;
      sg_edge(psi[k], psi[m], nn[k], nn[m], pp[k], pp[m], pk.an[a][k], pk.ap[a][k],
              pk.dl[a][k], pk.h[a][aoff[a] + coord[a]], e);
      dn = dn + e.Jn; dp = dp + e.Jp;
    }
    if (coord[a] >= 1) {             // edge from the low neighbour (node = high end)
      const int64_t m = k - stride[a];
      Edge e;
      sg_edge(psi[m], psi[k], nn[m], nn[k], pp[m], pp[k], pk.an[a][m], pk.ap[a][m],
              pk.dl[a][m], pk.h[a][aoff[a] + coord[a] - 1], e);
      dn = dn - e.Jn; dp = dp - e.Jp;
    }
    tn = a == 0 ? face[a] * dn : tn + face[a] * dn;
    tp = a == 0 ? face[a] * dp : tp + face[a] * dp;
  }
  double Rs, dRsn, dRsp;
  recomb(nn[k], pp[k], pk.nie[k], pk.tau_n[k], pk.tau_p[k], par, Rs, dRsn, dRsp);
  out[t] = tn - Rs * dV;
  out[count + t] = tp + Rs * dV;
}

// fixed-order sum of vals[0..count) by one block
__global__ void k_sum_list(const double* __restrict__ vals, int64_t count,
                           double* __restrict__ out) {
  __shared__ double sm[32];
  double s = 0.0;
  for (int64_t q = threadIdx.x; q < count; q += blockDim.x) s += vals[q] + vals[count + q];
  const double r = block_sum<256>(s, sm);
  if (threadIdx.x == 0) out[0] = r;
}

template <int DIM>
__global__ void k_edge_currents(const tcad_pack_t pk, int axis,
                                const double* __restrict__ psi,
                                const double* __restrict__ nn,
                                const double* __restrict__ pp, double* __restrict__ Jn,
                                double* __restrict__ Jp) {
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  const Inst g = load_inst(pk, fb.inst);
  const int64_t sxy = (int64_t)g.nx * g.ny;
  const int64_t stride = axis == 0 ? 1 : (axis == 1 ? g.nx : sxy);
  const int extent = axis == 0 ? g.nx : (axis == 1 ? g.ny : g.nz);
  const int64_t aoff = pk.axis_off[3 * fb.inst + axis];
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += blockDim.x) {
    const int64_t loc = k - fb.ioff;
    const int c = axis == 0 ? (int)(loc % g.nx)
                            : (axis == 1 ? (int)((loc / g.nx) % g.ny) : (int)(loc / sxy));
    double a = 0.0, b = 0.0;
    if (c + 1 < extent) {
      const int64_t m = k + stride;
      Edge e;
      sg_edge(psi[k], psi[m], nn[k], nn[m], pp[k], pp[m], pk.an[axis][k], pk.ap[axis][k],
              pk.dl[axis][k], pk.h[axis][aoff + c], e);
      a = e.Jn; b = e.Jp;
    }
    Jn[k] = a;
    Jp[k] = b;
  }
}

// ---------------------------------------------------------------------------
// equilibrium Poisson (slaved Boltzmann densities), node-centric
template <int DIM>
__global__ void __launch_bounds__(kFlatThreads)
k_poisson_assemble(const tcad_pack_t pk, const double* __restrict__ psi,
                   double* __restrict__ F, double* __restrict__ J, int mode) {
  constexpr int NP = 1 + 2 * DIM;
  const FlatBlock fb = flat_block(pk, blockIdx.x);
  const Inst g = load_inst(pk, fb.inst);
  const int64_t sxy = (int64_t)g.nx * g.ny;
  const int64_t ax0 = pk.axis_off[3 * fb.inst], ay0 = pk.axis_off[3 * fb.inst + 1];
  const int64_t az0 = pk.axis_off[3 * fb.inst + 2];
  const int64_t NN = pk.n_nodes;
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += blockDim.x) {
    const int64_t loc = k - fb.ioff;
    const int i = (int)(loc % g.nx), j = (int)((loc / g.nx) % g.ny);
    const int kz = DIM == 3 ? (int)(loc / sxy) : 0;
    const uint8_t flag = pk.bcflag[k];
    double Fv;
    double Jv[NP];
#pragma unroll
    for (int e = 0; e < NP; ++e) Jv[e] = 0.0;
    const double ps = psi[k];
    if (flag & TCAD_BC_CONTACT) {
      Fv = ps - pk.bc_psi0_eq[k];
      Jv[0] = 1.0;
    } else {
      const double ns = pk.nie_s[k] * exp(clip700(ps));
      const double ps_ = pk.nie_s[k] * exp(clip700(-ps));
      const double dnp = ns + ps_;
      const double dvx = pk.dv[0][ax0 + i], dvy = pk.dv[1][ay0 + j];
      const double dvz = DIM == 3 ? pk.dv[2][az0 + kz] : 1.0;
      const double face[3] = {DIM == 2 ? dvy : dvy * dvz, DIM == 2 ? dvx : dvx * dvz,
                              dvx * dvy};
      const double dV = DIM == 2 ? dvy * dvx : (dvz * dvy) * dvx;
      const int coord[3] = {i, j, kz};
      const int extent[3] = {g.nx, g.ny, g.nz};
      const int64_t stride[3] = {1, g.nx, sxy};
      const int64_t aoff[3] = {ax0, ay0, az0};
      double Ft = 0.0, dg = 0.0;
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        double dv = 0.0;
        const bool hiv = coord[a] + 1 < extent[a], lov = coord[a] >= 1;
        if (hiv) {
          const double h = pk.h[a][aoff[a] + coord[a]];
          dv = dv + (psi[k + stride[a]] - ps) / h;
          const double w = face[a] / h;
          dg = dg + (-w);
          Jv[2 + 2 * a] = w;
        }
        if (lov) {
          const double h = pk.h[a][aoff[a] + coord[a] - 1];
          dv = dv - (ps - psi[k - stride[a]]) / h;
          const double w = face[a] / h;
          dg = dg + (-w);
          Jv[1 + 2 * a] = w;
        }
        Ft = a == 0 ? face[a] * dv : Ft + face[a] * dv;
      }
      Fv = Ft - dV * (ns - ps_ - pk.C[k]);
      dg = dg + (-dV) * dnp;
      if (flag & TCAD_BC_GATE) {
        const double gk = pk.gate_k[k];
        Fv = Fv + gk * (pk.gate_veq[k] - (ps - pk.gate_b[k]));
        dg = dg + (-gk);
      }
      Jv[0] = dg;
      if (mode == TCAD_MODE_ELIMINATE) {
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          if (coord[a] >= 1) {
            const int64_t m = k - stride[a];
            if (pk.bcflag[m] & TCAD_BC_CONTACT) {
              Fv = Fv - Jv[1 + 2 * a] * (psi[m] - pk.bc_psi0_eq[m]);
              Jv[1 + 2 * a] = 0.0;
            }
          }
          if (coord[a] + 1 < extent[a]) {
            const int64_t m = k + stride[a];
            if (pk.bcflag[m] & TCAD_BC_CONTACT) {
              Fv = Fv - Jv[2 + 2 * a] * (psi[m] - pk.bc_psi0_eq[m]);
              Jv[2 + 2 * a] = 0.0;
            }
          }
        }
      }
    }
    F[k] = Fv;
#pragma unroll
    for (int e = 0; e < NP; ++e) J[(int64_t)e * NN + k] = Jv[e];
  }
}

// ---------------------------------------------------------------------------
// Theta-scheme storage term of one time step (pytcad/transient2d.py:104-135):
// at every non-contact node, on the assembled continuity rows,
//   F_n <- theta F_n + (1 - theta) fn_old - dV/dt (n - n_old)
//   F_p <- theta F_p + (1 - theta) fp_old + dV/dt (p - p_old)
// the n and p rows of J (diagonal-block rows 1 and 2, neighbour entries
// m = 1..4) scaled by theta, then J[n,n] += -dV/dt, J[p,p] += dV/dt.  The
// Poisson row and the contact rows are left as assembled.  Same operation
// order as the reference (this unit rounds step by step, -fmad=false).
template <int DIM>
__global__ void __launch_bounds__(kFlatThreads)
k_storage(const tcad_pack_t pk, const double* __restrict__ nn, const double* __restrict__ pp,
          const double* __restrict__ n_old, const double* __restrict__ p_old,
          const double* __restrict__ fn_old, const double* __restrict__ fp_old, double dt,
          double theta, double* __restrict__ F, double* __restrict__ J,
          const int32_t* __restrict__ blk) {
  const FlatBlock fb = flat_block(pk, blk ? (int64_t)blk[blockIdx.x] : (int64_t)blockIdx.x);
  const Inst g = load_inst(pk, fb.inst);
  const int64_t sxy = (int64_t)g.nx * g.ny;
  const int64_t ax0 = pk.axis_off[3 * fb.inst], ay0 = pk.axis_off[3 * fb.inst + 1];
  const int64_t az0 = pk.axis_off[3 * fb.inst + 2];
  const int64_t NN = pk.n_nodes;
  constexpr int NE = DIM == 2 ? TCAD_NE2 : TCAD_NE3;
  for (int64_t k = fb.begin + threadIdx.x; k < fb.end; k += kFlatThreads) {
    if (pk.bcflag[k] & TCAD_BC_CONTACT) continue;
    const int64_t loc = k - fb.ioff;
    const int i = (int)(loc % g.nx), j = (int)((loc / g.nx) % g.ny);
    const int kz = DIM == 3 ? (int)(loc / sxy) : 0;
    const double dvx = pk.dv[0][ax0 + i], dvy = pk.dv[1][ay0 + j];
    const double dvz = DIM == 3 ? pk.dv[2][az0 + kz] : 1.0;
    const double dV = DIM == 2 ? dvy * dvx : (dvz * dvy) * dvx;
    double f1 = F[NN + k], f2 = F[2 * NN + k];
    if (theta != 1.0) {
      f1 = theta * f1 + (1.0 - theta) * fn_old[k];
      f2 = theta * f2 + (1.0 - theta) * fp_old[k];
#pragma unroll
      for (int e = 3; e < 9; ++e) J[(int64_t)e * NN + k] = theta * J[(int64_t)e * NN + k];
#pragma unroll
      for (int e = 9; e < NE; ++e)
        if ((e - 9) % 5 != 0) J[(int64_t)e * NN + k] = theta * J[(int64_t)e * NN + k];
    }
    const double c = dV / dt;
    F[NN + k] = f1 - c * (nn[k] - n_old[k]);
    F[2 * NN + k] = f2 + c * (pp[k] - p_old[k]);
    J[(int64_t)4 * NN + k] = J[(int64_t)4 * NN + k] + (-c);
    J[(int64_t)8 * NN + k] = J[(int64_t)8 * NN + k] + c;
  }
}

// ---------------------------------------------------------------------------
// Elementwise evaluation of the SG device functions, compiled exactly as the
// assembly uses them (same unit, same -fmad=false rounding): the hook the
// elementwise parity tests read through.
__global__ void k_eval_bernoulli(const double* __restrict__ x, int64_t count,
                                 double* __restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  double Bp, Bm, dBp, dBm;
  bern4(x[t], Bp, Bm, dBp, dBm);
  out[t] = Bp;
  out[count + t] = Bm;
  out[2 * count + t] = dBp;
  out[3 * count + t] = dBm;
}

__global__ void k_eval_recombination(const double* __restrict__ n, const double* __restrict__ p,
                                     const double* __restrict__ nie,
                                     const double* __restrict__ taun,
                                     const double* __restrict__ taup, int64_t count,
                                     const double* __restrict__ par, double* __restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  double Rs, dRsn, dRsp;
  recomb(n[t], p[t], nie[t], taun[t], taup[t], par, Rs, dRsn, dRsp);
  out[t] = Rs;
  out[count + t] = dRsn;
  out[2 * count + t] = dRsp;
}

int storage_terms(const tcad_pack_t* pk, const double* n, const double* p,
                  const double* n_old, const double* p_old, const double* fn_old,
                  const double* fp_old, double dt, double theta, double* F, double* J,
                  const int32_t* blk, int64_t n_list, cudaStream_t s) {
  if (!pack_ok(pk) || !(dt > 0.0) || !n_old || !p_old) return TCAD_ERR_ARG;
  if (theta != 1.0 && (!fn_old || !fp_old)) return TCAD_ERR_ARG;
  const unsigned nb = (unsigned)(blk ? n_list : pk->n_flat);
  if (nb == 0) return TCAD_OK;
  if (pk->dim == 2)
    k_storage<2><<<nb, kFlatThreads, 0, s>>>(*pk, n, p, n_old, p_old, fn_old, fp_old, dt, theta,
                                             F, J, blk);
  else
    k_storage<3><<<nb, kFlatThreads, 0, s>>>(*pk, n, p, n_old, p_old, fn_old, fp_old, dt, theta,
                                             F, J, blk);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

int sg_assemble_tiles(const tcad_pack_t* pk, const double* psi, const double* n,
                      const double* p, double* F, double* J, int mode, const int32_t* tiles,
                      int64_t n_list, cudaStream_t s) {
  if (!pack_ok(pk) || pk->n_tiles <= 0) return TCAD_ERR_ARG;
  const unsigned nt = (unsigned)(tiles ? n_list : pk->n_tiles);
  if (nt == 0) return TCAD_OK;
  if (pk->dim == 2) {
    k_sg_assemble<2, false><<<nt, kTileThreads, 0, s>>>(*pk, psi, n, p, F, J, mode, tiles);
  } else if (pk->asm_stage) {
    TCAD_CUDA_CHECK(cudaFuncSetAttribute(k_sg_assemble<3, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kStageBytes));
    k_sg_assemble<3, true><<<nt, kTileThreads, kStageBytes, s>>>(*pk, psi, n, p, F, J, mode,
                                                                tiles);
  } else {
    k_sg_assemble<3, false><<<nt, kTileThreads, 0, s>>>(*pk, psi, n, p, F, J, mode, tiles);
  }
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

}  // namespace tcad

using namespace tcad;

extern "C" int tcad_sg_assemble(const tcad_pack_t* pk, const double* psi, const double* n,
                                const double* p, double* F, double* J, int mode,
                                void* stream) {
  if (mode != TCAD_MODE_RAW && mode != TCAD_MODE_ELIMINATE && mode != TCAD_MODE_UNSTAMPED)
    return TCAD_ERR_ARG;
  return sg_assemble_tiles(pk, psi, n, p, F, J, mode, nullptr, 0, (cudaStream_t)stream);
}

extern "C" int tcad_contact_current(const tcad_pack_t* pk, const double* psi,
                                    const double* n, const double* p,
                                    const int64_t* nodes, int64_t count, double* partial,
                                    int64_t partial_len, double* out_sum, void* stream) {
  if (!pack_ok(pk) || count < 0 || partial_len < 2 * count) return TCAD_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (count > 0) {
    const unsigned nb_ = (unsigned)((count + 255) / 256);
    if (pk->dim == 2)
      k_contact_current<2><<<nb_, 256, 0, s>>>(*pk, psi, n, p, nodes, count, partial);
    else
      k_contact_current<3><<<nb_, 256, 0, s>>>(*pk, psi, n, p, nodes, count, partial);
    note_launch();
    TCAD_LAUNCH_CHECK();
  }
  k_sum_list<<<1, 256, 0, s>>>(partial, count, out_sum);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

extern "C" int tcad_edge_currents(const tcad_pack_t* pk, int axis, const double* psi,
                                  const double* n, const double* p, double* Jn,
                                  double* Jp, void* stream) {
  if (!pack_ok(pk) || axis < 0 || axis >= pk->dim) return TCAD_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned nb_ = (unsigned)pk->n_flat;
  if (pk->dim == 2)
    k_edge_currents<2><<<nb_, kFlatThreads, 0, s>>>(*pk, axis, psi, n, p, Jn, Jp);
  else
    k_edge_currents<3><<<nb_, kFlatThreads, 0, s>>>(*pk, axis, psi, n, p, Jn, Jp);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

extern "C" int tcad_poisson_assemble(const tcad_pack_t* pk, const double* psi, double* F,
                                     double* J, int mode, void* stream) {
  if (!pack_ok(pk)) return TCAD_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned nb_ = (unsigned)pk->n_flat;
  if (pk->dim == 2)
    k_poisson_assemble<2><<<nb_, kFlatThreads, 0, s>>>(*pk, psi, F, J, mode);
  else
    k_poisson_assemble<3><<<nb_, kFlatThreads, 0, s>>>(*pk, psi, F, J, mode);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

extern "C" int tcad_eval_bernoulli(const double* x, int64_t count, double* out, void* stream) {
  if (count < 0 || (count > 0 && (!x || !out))) return TCAD_ERR_ARG;
  if (count == 0) return TCAD_OK;
  k_eval_bernoulli<<<(unsigned)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(x, count,
                                                                                     out);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}

extern "C" int tcad_eval_recombination(const double* n, const double* p, const double* nie,
                                       const double* tau_n, const double* tau_p, int64_t count,
                                       const double* par, double* out, void* stream) {
  if (count < 0 || !par || (count > 0 && (!n || !p || !nie || !tau_n || !tau_p || !out)))
    return TCAD_ERR_ARG;
  if (count == 0) return TCAD_OK;
  k_eval_recombination<<<(unsigned)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      n, p, nie, tau_n, tau_p, count, par, out);
  note_launch();
  TCAD_LAUNCH_CHECK();
  return TCAD_OK;
}
