"""Models and NewtonOptions, the reference's option contract
(pytcad/device.py:373-535, 539-627), restricted to what the GPU path
implements.  A physics flag the path does not implement is refused loudly
instead of being ignored, the reference's own rule for unimplemented
compositions (e.g. pytcad/device2d.py:224-232)."""
from __future__ import annotations

from dataclasses import dataclass


@dataclass
class Models:
    doping_mobility: bool = True
    field_mobility: bool = False
    srh: bool = True
    tat: bool = False
    trap_et_rel: float = 0.5
    fd: bool = False
    incomplete_ion: bool = False
    impact: bool = False
    impact_nonlocal: bool = False
    impact_lambda_n: float = 6.5e-6   # ii_nonlocal.py:61
    impact_lambda_p: float = 6.5e-6
    btbt: bool = False
    btbt_nonlocal: bool = False
    dg: bool = False
    dg_gamma: float = 1.0
    auger: bool = True
    bgn: bool = True
    surface_mobility: bool = False
    driving_force: str = "field"
    band_offset: str = "nie"
    thermionic: bool = False
    S_n: float = 0.0
    S_p: float = 0.0
    energy_balance: bool = False

    _GPU_UNIMPLEMENTED = ("field_mobility", "tat", "fd", "incomplete_ion", "impact",
                          "impact_nonlocal", "btbt", "btbt_nonlocal", "dg",
                          "surface_mobility", "thermionic", "energy_balance")

    def __post_init__(self):
        if self.band_offset not in ("nie", "affinity"):
            raise ValueError(f"Models.band_offset={self.band_offset!r} is not recognised")
        if self.driving_force != "field":
            raise NotImplementedError(
                f"Models.driving_force={self.driving_force!r} is not implemented")

    def require_gpu_path(self):
        """Raise NotImplementedError for flags outside the GPU path."""
        on = [f for f in self._GPU_UNIMPLEMENTED if getattr(self, f)]
        if self.band_offset != "nie":
            on.append("band_offset='affinity'")
        if self.S_n != 0.0 or self.S_p != 0.0:
            on.append("S_n/S_p")
        if on:
            raise NotImplementedError(
                "tcad_b200 implements the plain drift-diffusion path (Boltzmann, "
                "full ionisation, SRH/Auger, doping mobility, BGN); refusing "
                f"Models({', '.join(on)}) rather than silently ignoring it")


@dataclass
class NewtonOptions:
    max_iter: int = 100
    tol_update: float = 1e-8
    tol_residual: float = 1e-10
    max_dpsi: float = 5.0
    verbose: bool = False
    linsolve: str = "auto"
    linsolve_rtol: float = 1e-10
    precond: str = "auto"
    block_size: int | None = 3
    direct_ordering: str | None = None
    # GPU-only: Krylov iteration budget per Newton step (the reference's
    # solve_linear caps at 500 and falls back to a CPU direct solve, which
    # the GPU path does not have)
    linsolve_maxiter: int = 4000
    # GPU-only: Newton steps taken after the update test passes.  The test
    # saturates at the 1e-10 density floor, so sub-floor minority densities
    # (and low-bias currents) are converged only to ~1e-5 when it first
    # passes; the first step (solved to polish_eta) brings them to round-off.
    # The second (solved to the forcing tolerance) lands on the FP64 fixed
    # point of the residual: at low-current points the terminal current is
    # a difference of contact fluxes ~1e11 times larger (a 20x6x5 p-i-n at
    # 0.4 V: 4.9e-15 A), so one ulp of the state still moves it by ~1e-4,
    # while at the fixed point -- the same one the reference's Newton
    # reaches, since the residual arithmetic is the reference's -- the
    # currents agree to 1e-16.
    polish: int = 2
    # GPU-only: Krylov tolerance of the first polishing step (the second
    # follows the forcing rule).  Measured over the fixture sweeps with the
    # floor-free polishing scale below: every current within 1.3e-8 of the
    # reference's in 14-24 % fewer Krylov iterations than 1e-10, except
    # currents that the last bits of the state decide (the 48x24x12 p-i-n at
    # 0.5 V, 1.2e-13 A: 1.2e-8 to 1.9e-6 off across the Krylov systems and
    # polishing tolerances, each state within rounding of the oracle's); on
    # the full system 1e-3 put the 201x101 diode's currents 4.5e-6 off.
    polish_eta: float = 1e-6
    # GPU-only: density floor of the relative Krylov unknowns in the
    # polishing steps (0: krylov_scale_floor).  The polishing steps run with
    # no floor to speak of, so minority densities below the 1e-10 floor of
    # the update test -- the ones low-bias currents are made of -- count in
    # their Krylov norm: with the floor, the 48x24x12 p-i-n's 0.5 V current
    # (1.2e-13 A, minority electrons in the p+ region at ~2e-10) was 1.9e-6
    # off the oracle; without, 1.2e-8.
    polish_scale_floor: float = 1e-30
    # GPU-only: inexact-Newton forcing.  "adaptive" solves step k to
    # eta_k = clamp(0.1 * update_{k-1}, linsolve_rtol, eta_max) (quadratic
    # convergence is kept; the converged state is the same); "fixed" solves
    # every step to linsolve_rtol like the reference's iterative branch.
    forcing: str = "adaptive"
    eta_max: float = 1e-3
    # tightest forcing term; None: eta_max for precision "fp64" (every step
    # to 1e-3: once Newton converges quadratically the step's size, not the
    # linear tolerance, decides the next update), linsolve_rtol for "mixed"
    eta_min: float | None = None
    # GPU-only: "fp64" solves the Newton systems in FP64; "fp32_operator"
    # runs the FP64 BiCGStab of the Newton steps before the update test on an
    # FP32 copy of the block-scaled Jacobian (half the operator's bytes; the
    # polishing steps keep FP64); "mixed" runs the
    # Krylov iterations in FP32 on an FP32 copy of the block-scaled Jacobian
    # inside FP64 iterative refinement -- residual, Newton update and the
    # convergence test stay FP64, so the converged state is the FP64 one.
    precision: str = "fp64"
    # GPU-only: Krylov unknowns.  "relative" solves for (dpsi, dn/max(n,1e-10),
    # dp/max(p,1e-10)) -- the quantities the Newton update test measures --
    # through a similarity transform of the block-scaled Jacobian; "absolute"
    # for (dpsi, dn, dp).
    krylov_unknowns: str = "relative"
    # GPU-only: floor of the density scale of the relative Krylov unknowns
    # (a similarity transform: it changes the conditioning, not the solution)
    krylov_scale_floor: float = 1e-10
    # GPU-only: start of a sweep point.  "secant" extrapolates the state
    # along the sweep when the new bias step is parallel to the previous one
    # (psi linearly, n and p in log space); "none" starts from the previous
    # converged state as the reference does.  The converged state is the
    # same discrete solution either way; a predicted start that fails to
    # converge is retried from the previous state.
    predictor: str = "secant"
    # GPU-only: the system the node-block-Jacobi BiCGStab iterates on.
    # "red_black" eliminates the red nodes ((i + j + k) even) exactly -- the
    # face-neighbour stencil couples no two nodes of one colour -- and
    # iterates on the Schur complement over the black nodes: half the
    # unknowns, the same matrix bytes per operator product, and on the
    # tri-gate Newton systems about half the iterations (the 983k-node
    # tri-gate sweep: 1,610 BiCGStab iterations per point against 3,634, 2.04
    # against 1.17 points/s); the stopping test is the full system's.
    # "full" iterates on the whole block-scaled system.  Either system runs
    # in one cooperative launch per solve on a single-instance pack small
    # enough to be resident at once (the 201x101 diode: 33.7 points/s
    # red-black, 21.3 whole system).
    krylov_system: str = "red_black"

    def __post_init__(self):
        if self.precond not in ("auto", "block_jacobi", "schur", "ilu"):
            raise ValueError(f"NewtonOptions.precond={self.precond!r} is not a known "
                             "preconditioner flavor")
        if self.block_size is not None and (
                not isinstance(self.block_size, int) or self.block_size <= 0):
            raise ValueError(f"NewtonOptions.block_size={self.block_size!r} must be "
                             "a positive int or None.")
        if self.linsolve not in ("auto", "direct", "gmres", "bicgstab", "gpu_direct",
                                 "petsc", "mumps"):
            raise ValueError(f"unknown linsolve {self.linsolve!r}")
        if self.predictor not in ("none", "secant"):
            raise ValueError(f"NewtonOptions.predictor={self.predictor!r}: 'none' or 'secant'")
        if self.krylov_system not in ("full", "red_black"):
            raise ValueError(f"NewtonOptions.krylov_system={self.krylov_system!r}: 'full' or "
                             "'red_black'")
        if self.precision not in ("fp64", "mixed", "fp32_operator"):
            raise ValueError(f"NewtonOptions.precision={self.precision!r}: 'fp64', 'mixed' "
                             "or 'fp32_operator'")
