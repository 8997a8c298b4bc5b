/*
 * tcad_b200 -- C ABI of the sm_100a drift-diffusion solve path.
 *
 * Every entry point takes plain device pointers and sizes, launches on the
 * given CUDA stream and returns a status code (TCAD_OK or a TCAD_ERR_*
 * value); nothing throws across this boundary.  A host binding maps the
 * codes onto the reference's error classes the way the reference's own
 * binding does (core/bindings/module.cpp:100-127): TCAD_ERR_ARG -> ValueError,
 * TCAD_ERR_SINGULAR / _NONFINITE / _NOCONV / _BREAKDOWN -> LinearSolveError
 * (pytcad/linsolve.py:344), TCAD_ERR_CUDA -> RuntimeError.
 *
 * Data model ("pack"): one or more devices (instances) of one dimension share
 * the node arrays.  Node arrays are structure-of-arrays of length n_nodes,
 * node k of instance i sitting at node_off[i] + k (instance i spans
 * Nx*Ny*Nz nodes; instances are listed in increasing node_off and may leave
 * gaps, as in a serving arena whose resident devices keep their places) with
 * k = (kz*Ny + j)*Nx + i_x (x fastest), the reference's flat order
 * (pytcad/mesh2d.py:1-7, pytcad/mesh3d.py:1-10).  Edge coefficients live at
 * the edge's low ("owner") node.  Vectors of the coupled system are
 * component-major: [psi(n_nodes) | n(n_nodes) | p(n_nodes)].
 *
 * Coupled Jacobian ("node-block" layout), TCAD_NE2 = 29 (2D) or
 * TCAD_NE3 = 39 (3D) doubles per node, entry-major (J[e*n_nodes + k]):
 *   e = 0..8            diagonal 3x3 block, row-major (row, col) over (psi,n,p)
 *   e = 9 + 5*d + m     neighbour d = W,E,S,N,D,U (-x,+x,-y,+y,-z,+z);
 *                       m = (psi<-psi), (n<-psi), (n<-n), (p<-psi), (p<-p)
 * which is exactly the structural pattern of the reference's COO stamps
 * (pytcad/device2d.py:1534-1621, core/src/device3d/kernels.cpp:40-168).
 * Equilibrium Poisson Jacobian: 1 + 2*dim doubles per node (diag, then the
 * neighbours in the same W,E,S,N,D,U order).
 */
#ifndef TCAD_B200_H
#define TCAD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TCAD_OK 0
#define TCAD_ERR_ARG 1
#define TCAD_ERR_SINGULAR 2
#define TCAD_ERR_NONFINITE 3
#define TCAD_ERR_NOCONV 4
#define TCAD_ERR_CUDA 5
#define TCAD_ERR_BREAKDOWN 6

#define TCAD_NE2 29
#define TCAD_NE3 39
#define TCAD_FLAT_NODES 512  /* default nodes per flat (vector-kernel) block */
#define TCAD_TILE_X 32       /* stencil tile: 32 x 8 nodes (x, y) */
#define TCAD_TILE_Y 8
#define TCAD_TILE_Z 16       /* largest z depth of a 3D stencil tile (tile_z <= this) */

/* per-instance scalar parameters: par[i*TCAD_NPAR + TCAD_P_*] */
#define TCAD_NPAR 8
#define TCAD_P_NS 0    /* reference concentration Ns [cm^-3] */
#define TCAD_P_R0 1    /* recombination scale D0 Ns / LD^2 */
#define TCAD_P_CN 2    /* Auger Cn [cm^6/s] */
#define TCAD_P_CP 3    /* Auger Cp [cm^6/s] */
#define TCAD_P_SRH 4   /* 1.0: recombination on (Models.srh) */
#define TCAD_P_AUGER 5 /* 1.0: Auger on (Models.auger) */

/* assembly modes */
#define TCAD_MODE_RAW 0        /* reference _residual_jacobian rows, BC rows stamped */
#define TCAD_MODE_ELIMINATE 1  /* + symmetric Dirichlet elimination (pytcad/dirichlet.py:270) */
#define TCAD_MODE_UNSTAMPED 2  /* contact rows left as assembled continuity/Poisson rows: the
                                  raw current rows the AC sensitivities sum
                                  (current_rows_for, pytcad/device2d.py:1751-1758) */

/* tcad_newton_opts_t.precision: FP32 operator copy, FP64 Krylov vectors */
#define TCAD_PRECISION_J32 33

/* bcflag bits */
#define TCAD_BC_CONTACT 1
#define TCAD_BC_GATE 2

typedef struct tcad_pack {
  int32_t dim;           /* 2 or 3 */
  int32_t n_inst;        /* packed instances */
  int64_t n_nodes;       /* length of every node array (>= the last instance's end) */
  int64_t n_flat;        /* flat blocks (flat_nodes nodes, never straddling instances) */
  int64_t n_tiles;       /* stencil tiles */
  int32_t tile_z;        /* z planes one 3D tile marches (1..TCAD_TILE_Z; the tiles'
                            k0 are multiples of it); 1 in 2D */
  int32_t flat_nodes;    /* nodes per flat block (>= 1; each instance starts a block) */
  int32_t asm_stage;     /* 3D coupled assembly: 0 loads each plane's edge and node
                            coefficients where it uses them; 1 stages the next plane's
                            into shared memory with asynchronous copies while the
                            current plane computes (same arithmetic, bit-identical) */
  int32_t reserved;      /* 0 */
  /* per-instance tables (device memory) */
  const int32_t* shape;    /* [3*n_inst] Nx, Ny, Nz (Nz = 1 in 2D) */
  const int64_t* node_off; /* [n_inst+1] first node of each instance, increasing;
                              node_off[n_inst] = n_nodes */
  const int64_t* flat_off; /* [n_inst+1] first flat block of each instance */
  const int32_t* flat_inst;/* [n_flat] instance of each flat block */
  const int64_t* axis_off; /* [3*n_inst] start of the instance's x/y/z entries in h[]/dv[] */
  const int32_t* tile;     /* [4*n_tiles] inst, i0, j0, k0 */
  const double* par;       /* [TCAD_NPAR*n_inst] */
  /* packed axis geometry, scaled by LD; h has the same count as dv (last unused) */
  const double* h[3];
  const double* dv[3];
  /* node data (device memory, n_nodes each) */
  const double* C;       /* net doping / Ns */
  const double* nie;     /* effective intrinsic density [cm^-3] */
  const double* nie_s;   /* nie / Ns */
  const double* tau_n;   /* SRH lifetimes [s] */
  const double* tau_p;
  const double* an[3];   /* electron edge coefficient D_edge/h at the edge's low node */
  const double* ap[3];   /* hole edge coefficient */
  const double* dl[3];   /* ln(nie_s[high]/nie_s[low]) */
  const uint8_t* bcflag; /* TCAD_BC_* bits */
  const double* bc_psi0; /* contact targets at the current bias (read where CONTACT) */
  const double* bc_n0;
  const double* bc_p0;
  const double* bc_psi0_eq; /* contact psi target of the zero-bias equilibrium */
  const double* gate_k;  /* kappa*w summed over the node's gates (read where GATE) */
  const double* gate_v;  /* Vg/VT - Vfb/VT */
  const double* gate_veq;/* 0 - Vfb/VT (equilibrium: gate at zero bias) */
  const double* gate_b;  /* local neutral-bulk potential psi_b */
} tcad_pack_t;

/* ABI guard: sizeof(tcad_pack_t) as compiled into the library. */
size_t tcad_pack_sizeof(void);
/* "tcad_b200 <version> sm_100a" */
const char* tcad_version(void);
/* Number of kernels this library has launched since it was loaded. */
uint64_t tcad_launch_count(void);

/* ---- assembly ------------------------------------------------------------
 * Coupled SG residual/Jacobian at (psi, n, p) [scaled, n_nodes each].
 * Replaces Device2D._residual_jacobian (pytcad/device2d.py:1402-1920) and
 * Device3D._residual_jacobian with its compiled stamps (pytcad/device3d.py:
 * 1485-1978, core/src/device3d/kernels.cpp:40-168).  F is [3][n_nodes],
 * J is [NE][n_nodes].  RAW: contact rows become (x - x0) with unit blocks;
 * ELIMINATE: in addition the contact columns are folded into F, so that
 * -F is the eliminated right-hand side of pytcad/dirichlet.py:270-300. */
int tcad_sg_assemble(const tcad_pack_t* pk, const double* psi, const double* n,
                     const double* p, double* F, double* J, int mode, void* stream);

/* Raw continuity residual F_n + F_p at a node list (before the contact rows
 * are stamped) -- the terminal-current kernel of Device2D/3D.terminal_current
 * (pytcad/device2d.py:2194-2227, pytcad/device3d.py:2274-2306).  Writes the
 * deterministic sum over the list to out_sum[0]. */
int tcad_contact_current(const tcad_pack_t* pk, const double* psi, const double* n,
                         const double* p, const int64_t* nodes, int64_t count,
                         double* partial, int64_t partial_len, double* out_sum,
                         void* stream);
/* (partial must hold 2*count doubles: F_n of the listed nodes, then F_p.) */

/* Edge current densities Jn, Jp of one axis at their low nodes (scaled;
 * Device2D/3D.Jn_x.. attributes, pytcad/device2d.py:2188-2190). */
int tcad_edge_currents(const tcad_pack_t* pk, int axis, const double* psi,
                       const double* n, const double* p, double* Jn, double* Jp,
                       void* stream);

/* Equilibrium Poisson residual/Jacobian with slaved Boltzmann densities,
 * Device2D._residual_jacobian_poisson (pytcad/device2d.py:844-942) and
 * Device3D's (pytcad/device3d.py:952-1020, core/src/device3d/poisson_eq.cpp:
 * 5-129).  F [n_nodes], J [(1+2*dim)][n_nodes]. */
int tcad_poisson_assemble(const tcad_pack_t* pk, const double* psi, double* F,
                          double* J, int mode, void* stream);

/* Elementwise SG device functions, compiled in the assembly's unit with the
 * assembly's rounding, for elementwise parity checks.
 * tcad_eval_bernoulli: out[4*count] = B(x), B(-x), B'(x), B'(-x) blocks of
 * count each -- pytcad/kernels.py:88-109 bernoulli / dbernoulli.
 * tcad_eval_recombination: out[3*count] = Rs, dRs/dn, dRs/dp blocks with
 * the per-instance parameters par[TCAD_NPAR] (Ns, R0, Cn, Cp, SRH, AUGER) --
 * pytcad/materials.py:474-518 recombination, scaled as
 * pytcad/device2d.py:1482-1508 (Ns = R0 = 1 gives the physical rates). */
int tcad_eval_bernoulli(const double* x, int64_t count, double* out, void* stream);
int tcad_eval_recombination(const double* n, const double* p, const double* nie,
                            const double* tau_n, const double* tau_p, int64_t count,
                            const double* par, double* out, void* stream);

/* ---- boundary conditions -------------------------------------------------
 * Contact targets at the current bias (contacts.ohmic_values,
 * pytcad/contacts.py:21-38, with psi0 = V/VT + ln(n0/nie)): for each listed
 * contact node t, contact id cid[t] with vv[cid] = V/VT:
 *   bc_psi0[node] = vv[cid[t]] + L[t],  bc_n0[node] = n0[t],  bc_p0[node] = p0[t]. */
int tcad_set_contacts(const tcad_pack_t* pk, const int64_t* nodes, int64_t count,
                      const int32_t* cid, const double* vv, const double* L,
                      const double* n0, const double* p0, double* bc_psi0,
                      double* bc_n0, double* bc_p0, void* stream);

/* Warm start at a new bias (pytcad/device2d.py:1949-1953): psi, n, p of the
 * listed contact nodes take their targets. */
int tcad_stamp_contacts(const tcad_pack_t* pk, const int64_t* nodes, int64_t count,
                        double* psi, double* n, double* p, void* stream);

/* Secant predictor for a bias sweep (no counterpart in the reference, which
 * warm-starts every point from the previous converged state,
 * pytcad/device2d.py:1949-1953; the converged state does not depend on the
 * start).  Per instance, ratio[inst] (device memory) = the new bias step over
 * the previous one when the two are parallel: psi moves linearly, n and p
 * geometrically (factor held to [0.1, 10]); ratio 0 leaves the state.  The
 * state before the call is saved into *_prev (all [n_nodes]). */
int tcad_state_extrapolate(const tcad_pack_t* pk, double* psi, double* n, double* p,
                           double* psi_prev, double* n_prev, double* p_prev,
                           const double* ratio, void* stream);

/* ---- linear algebra on the node-block layout ---------------------------
 * Workspace size in bytes for tcad_block_krylov / tcad_newton_solve.
 * method 2 includes the red-black Schur extension (two colour copies of the
 * Jacobian and five slot vectors), which tcad_block_krylov method 2 needs
 * and tcad_newton_opts_t.red_black uses; a tcad_newton_solve workspace
 * sized without it (method 0) solves the whole system.  restart is unused. */
size_t tcad_block_workspace_bytes(const tcad_pack_t* pk, int method, int restart);

/* Launch shape of the node-block-Jacobi BiCGStab (an implementation switch;
 * the reference has no counterpart: pytcad/linsolve.py:725-985 is one
 * scipy call).  on = 1 (the default): a single-instance pack whose flat
 * blocks all fit on the GPU at once is solved in ONE cooperative launch --
 * one CTA per flat block, bounded grid barriers between the steps, the same
 * arithmetic in the same order as the launch-per-step kernels, so the
 * result is bit-identical; on = 0: one launch per step always.  Process-
 * wide; returns the previous setting. */
int tcad_set_krylov_fused(int on);

/* Test hook of the fused solve's failure path (no counterpart in the
 * reference).  hold = 1: every later fused launch waits at its first grid
 * barrier for one arrival that never comes, so the barrier's bounded wait
 * (1 s of device time) runs out, the kernel returns, and the host solves
 * again with one launch per step.  Process-wide; returns the previous
 * setting.  tcad_krylov_fused_gave_up counts the fused launches whose
 * barrier gave up, hook or not. */
int tcad_set_krylov_fused_test(int hold);
uint64_t tcad_krylov_fused_gave_up(void);

/* Node-block-Jacobi set-up (pytcad/linsolve.py:363-427): inverts every
 * diagonal 3x3 block of J in place and replaces F by the block-scaled
 * right-hand side b^ = D^-1 (-F).  status[inst] gets TCAD_ERR_SINGULAR for a
 * block with |det| < 1e-300 or a non-finite entry. */
int tcad_block_jacobi_setup(const tcad_pack_t* pk, double* J, double* F,
                            int32_t* status, void* stream);

/* The same set-up in relative unknowns (u_psi, u_n, u_p) = (dpsi, dn/s_n,
 * dp/s_p) with s_n = max(n, dens_floor), s_p = max(p, dens_floor) at the
 * node: J and F are prepared for A^ = S^-1 D^-1 A S, S = diag(1, s_n, s_p),
 * and b^ = S^-1 D^-1 (-F).  The Krylov solve of tcad_newton_solve with
 * density_scaling = 1 runs on this operator; the update the reference's
 * Newton measures (pytcad/device2d.py:2079-2100) is relative in n and p. */
int tcad_block_jacobi_setup_rel(const tcad_pack_t* pk, double* J, double* F,
                                int32_t* status, const double* n, const double* p,
                                double dens_floor, void* stream);

/* Block ILU(0) of the block-scaled 2D operator A^ (J prepared by either
 * set-up above), the stronger preconditioner the reference reaches for on
 * hard 2D systems (pytcad/linsolve.py:430-525 builds an ILU-based one on
 * the CPU).  For the 5-point block stencil ILU(0) keeps the off-diagonal
 * blocks and replaces the diagonal ones: Q [9][n_nodes] receives their
 * inverses (tcad_block_ilu_bytes).  status[inst] gets TCAD_ERR_SINGULAR for
 * a singular block.  One CTA per instance sweeps its anti-diagonals. */
size_t tcad_block_ilu_bytes(const tcad_pack_t* pk);
int tcad_block_ilu_setup(const tcad_pack_t* pk, const double* J, double* Q,
                         int32_t* status, void* stream);
/* out = M^-1 r for the ILU(0) factor Q (r and out distinct, [3][n_nodes]). */
int tcad_block_ilu_apply(const tcad_pack_t* pk, const double* J, const double* Q,
                         const double* r, double* out, void* stream);

/* y = A^ x with A^ = I + D^-1 (off-diagonal blocks), J prepared by
 * tcad_block_jacobi_setup; x, y are [3][n_nodes]. */
int tcad_block_spmv(const tcad_pack_t* pk, const double* J, const double* x,
                    double* y, void* stream);

/* Krylov solve of A^ x = b^ for every instance of the pack, x starting at
 * zero, per-instance convergence ||b^ - A^ x|| <= rtol ||b^||.  method 0:
 * BiCGStab on A^; 2: BiCGStab on the red-black Schur complement of A^ (the
 * red nodes, (i + j + k) even, eliminated exactly; the same stopping test,
 * the full x returned; see tcad_newton_opts_t.red_black).  Any other method
 * is TCAD_ERR_ARG (GMRES runs on the CSR form, tcad_csr_krylov).
 * restart is unused.  iters/status/relres are per-instance host arrays.
 * Replaces the bicgstab + block-Jacobi branch of linsolve.solve_linear
 * (pytcad/linsolve.py:941-985). */
int tcad_block_krylov(const tcad_pack_t* pk, const double* J, const double* b,
                      double* x, int method, double rtol, int maxiter, int restart,
                      void* work, size_t work_bytes, int32_t* iters,
                      int32_t* status, double* relres, void* stream);

/* ---- general CSR (linsolve.solve_linear drop-in) -------------------------
 * Solve A x = b for one n x n CSR matrix (int32 indices, device memory),
 * x holding the initial guess.  method 0: BiCGStab (maxiter iterations),
 * 1: GMRES(restart) (maxiter restart cycles), both right-preconditioned by
 * node-block-Jacobi when block_size (3, or 6: the real-equivalent form of a
 * complex 3 x 3 node block) divides n (point Jacobi otherwise or when a
 * block is singular; *precond_out = 6, 3, 1 or 0), stopping at
 * ||b - A x|| <= max(atol, rtol ||b||) (pytcad/linsolve.py:941-985).
 * *resid_out = true ||b - A x|| / ||b||.  Returns TCAD_ERR_NOCONV when the
 * tolerance was not met (x then holds the last iterate). */
size_t tcad_csr_workspace_bytes(int64_t n, int method, int restart);
int tcad_csr_krylov(int64_t n, const int32_t* indptr, const int32_t* indices,
                    const double* data, const double* b, double* x, int method,
                    int block_size, double rtol, double atol, int maxiter, int restart,
                    void* work, size_t work_bytes, int32_t* iters_out, double* resid_out,
                    int32_t* precond_out, void* stream);

/* ---- node-block BiCGStab that allocates nothing ---------------------------
 * No counterpart in the reference.  The same solve as tcad_block_krylov
 * (method 0), for callers that cannot allocate device memory on demand: a
 * serving process whose HBM is already carved up by its own pool, a foreign-
 * language host (cgo / JNI / N-API) with no device allocator, or a latency-
 * critical loop that must not pay cudaMalloc's device-wide synchronisation.
 * The Krylov scratch is a file-scope device array of TCAD_STATIC_SCRATCH_BYTES
 * (5 MiB) that every GPU loading this library holds until exit; the entry
 * point calls no cudaMalloc / cudaFree and no host heap.  Limits:
 * n_nodes <= TCAD_STATIC_MAX_NODES (32768) and n_inst <= TCAD_STATIC_MAX_INST
 * (32); larger packs get TCAD_ERR_ARG.  The first call on each device looks up
 * the array's device address (cudaGetSymbolAddress) with that device current;
 * make it before any stream capture.  The looked-up address belongs to the
 * device's context: after cudaDeviceReset, reload the library before calling
 * this entry point again.  Calls share the array: each call clears what must
 * start at zero, and calls whose work overlaps on the GPU race. */
#define TCAD_STATIC_MAX_NODES 32768
#define TCAD_STATIC_MAX_INST 32
#define TCAD_STATIC_SCRATCH_BYTES (5u << 20)
int tcad_block_krylov_noalloc(const tcad_pack_t* pk, const double* J, const double* b,
                              double* x, double rtol, int maxiter, int32_t* iters,
                              int32_t* status, double* relres, void* stream);

/* ---- Newton --------------------------------------------------------------
 * Damped update of the coupled Newton loop (pytcad/device2d.py:2079-2160):
 * clip dpsi to +-max_dpsi, n/p to [0.1x, 10x], err = max(|dpsi|,
 * |dn|/max(n,floor), |dp|/max(p,floor)) per instance into err[inst]. */
int tcad_newton_update(const tcad_pack_t* pk, double* psi, double* n, double* p,
                       const double* du, double max_dpsi, double dens_floor,
                       const uint8_t* active, double* partial, double* err,
                       void* stream);

/* Options of one Newton solve (the NewtonOptions of pytcad/device.py:539-627). */
typedef struct tcad_newton_opts {
  int32_t max_iter;      /* 100 */
  int32_t method;        /* 0 BiCGStab, 1 GMRES */
  int32_t krylov_maxiter;
  int32_t restart;
  double tol_update;     /* 1e-8 */
  double max_dpsi;       /* 5 */
  double rtol;           /* Krylov relative tolerance (1e-10) */
  double dens_floor;     /* 1e-10 */
  int32_t verbose;
  int32_t polish;        /* extra Newton steps after the update test passes */
  double eta_max;        /* forcing: loosest Krylov tolerance of an early step */
  int32_t forcing;       /* 0: every step at rtol; 1: eta_k = clamp(0.1 err_{k-1}, eta_min,
                            eta_max) */
  int32_t precision;     /* 64: FP64 Krylov; 32: FP32 Krylov on an FP32 copy of the scaled
                            operator inside FP64 iterative refinement (residual, Newton,
                            convergence test stay FP64); TCAD_PRECISION_J32 (33): FP64
                            Krylov on an FP32 copy of the scaled operator in the steps
                            before the update test passes, FP64 operator in the
                            polishing steps (node-block Jacobi solves; ILU(0) solves
                            keep FP64) */
  int32_t density_scaling; /* 1: Krylov unknowns are (dpsi, dn/s_n, dp/s_p), s = max(n|p,
                              scale_floor) -- the quantities of the Newton update test */
  int32_t precond;       /* 0: node-block Jacobi; 1: + block ILU(0) right preconditioner on
                            2D packs; 2: automatic -- ILU(0) for the instances of a 2D
                            batch (n_inst > 1) and for any 2D instance whose
                            node-block-Jacobi solve fails (solved again with it).
                            FP64 Krylov only; 3D packs use node-block Jacobi */
  double eta_min;        /* forcing 1: tightest Krylov tolerance of a step (>= rtol) */
  double scale_floor;    /* density_scaling: floor of s (dens_floor when <= 0) */
  double polish_eta;     /* forcing 1: Krylov tolerance of the polishing steps (<= 0: the
                            forcing rule's) */
  double polish_scale_floor; /* density_scaling: floor of s in the polishing steps (<= 0:
                                scale_floor); a floor far below the densities lets the
                                polish resolve sub-floor minority densities */
  /* One time step of the theta scheme (pytcad/transient2d.py:104-135,
   * transient3d.py): dt > 0 adds, at every non-contact node, the storage
   * term to the continuity rows after each assembly --
   *   F_n <- theta F_n + (1 - theta) fn_old - dV/dt (n - n_old)
   *   F_p <- theta F_p + (1 - theta) fp_old + dV/dt (p - p_old)
   * with the n and p rows of J scaled by theta and their diagonal entries
   * moved by -dV/dt and +dV/dt.  dt is in the device's scaled time
   * (seconds * R0 / Ns); the arrays are [n_nodes], device memory; fn_old and
   * fp_old (raw continuity residuals at the previous time) are read only
   * when theta != 1.  dt = 0: a steady solve. */
  double dt;
  double theta;
  const double* n_old;
  const double* p_old;
  const double* fn_old;
  const double* fp_old;
  /* 1: the FP64 node-block-Jacobi solves run BiCGStab on the red-black Schur
   * complement of the block-scaled system (the face-neighbour stencil has
   * no coupling inside a colour of (i + j + k) & 1, so the red unknowns are
   * eliminated exactly: half the unknowns, the same matrix bytes per
   * product, about half the iterations); the stopping test stays the full
   * system's ||b - A x|| <= eta ||b||.  A single-instance pack whose slot
   * blocks fit on the GPU at once is solved in one cooperative launch (the
   * same arithmetic).  ILU(0) solves, FP32 operators and a workspace sized
   * without the red-black extension (tcad_block_workspace_bytes method 0)
   * keep the full system.  tcad_equilibrium_solve: its PCG runs on the
   * red-black Schur complement of the scalar Poisson system (every
   * workspace holds that extension).  0: the full systems always. */
  int32_t red_black;
  int32_t reserved_opts;  /* 0 */
} tcad_newton_opts_t;

/* Per-instance result of a Newton solve (host memory). */
typedef struct tcad_newton_result {
  int32_t iters;         /* Newton iterations taken */
  int32_t converged;     /* 1 when err < tol_update with a converged linear solve */
  int32_t krylov_iters;  /* total Krylov iterations */
  int32_t status;        /* last linear-solve status */
  double err;            /* last update norm */
  double relres;         /* last scaled linear residual */
  int32_t fp64_from;     /* precision 32: Newton iteration from which this instance
                            solved in FP64 after an FP32-solved step was rejected
                            (-1: never; always -1 for precision 64) */
  int32_t polish_iters;  /* of iters, the polishing steps taken after the update test
                            passed (the reference's own Newton count stops before them) */
} tcad_newton_result_t;

/* Full coupled Newton solve at the contact targets stored in the pack
 * (Device2D/3D.solve_bias inner loop, pytcad/device2d.py:2020-2160,
 * pytcad/device3d.py:2091-2239) for every instance whose active[inst] is
 * non-zero.  psi/n/p are updated in place.  J, F are assembly buffers
 * ([NE][n], [3][n]); du is [3][n]; work is tcad_block_workspace_bytes. */
int tcad_newton_solve(const tcad_pack_t* pk, double* psi, double* n, double* p,
                      double* F, double* J, double* du, const tcad_newton_opts_t* opts,
                      uint8_t* active, void* work, size_t work_bytes,
                      tcad_newton_result_t* result, void* stream);

/* Equilibrium Poisson Newton solve (Device2D/3D.solve_equilibrium,
 * pytcad/device2d.py:1308-1373, pytcad/device3d.py:1311-1454) from the psi
 * given; on return n, p hold the slaved densities. */
int tcad_equilibrium_solve(const tcad_pack_t* pk, double* psi, double* n, double* p,
                           double* F, double* J, double* d, const tcad_newton_opts_t* opts,
                           void* work, size_t work_bytes, tcad_newton_result_t* result,
                           void* stream);

#ifdef __cplusplus
}
#endif
#endif /* TCAD_B200_H */
