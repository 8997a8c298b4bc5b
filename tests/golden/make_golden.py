"""Generate the golden fixtures in this directory from the reference itself.

Runs the UNMODIFIED reference (pytcad) in the build container, where it is
importable, and stores its outputs as small .npz files that travel with the
repository (the reference does not).  Device2D runs as-is; Device3D needs
five compiled ``pytcad._core`` stamps (device3d.py:261-293, 1670-1752) whose
shipped binary cannot load here, so a shim binds them to the reference's OWN
Python oracle functions (device3d.py:190, 335, 348, 366, 384) -- the same
functions the reference's parity tests hold its compiled kernels to
(tests/test_m47_s2_device3d_accel_parity.py,
tests/test_device3d_poisson_eq_accel_parity.py).

Usage:  python tests/golden/make_golden.py --ref <reference>/pytcad
        [--skip-c1]   (the 201x101 diode sweep takes about 1-2 minutes)
"""
import argparse
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# Converged-state fixtures are solved to tol_update = 1e-12 (a stock
# NewtonOptions value): at the stock 1e-8 the update test saturates at the
# 1e-10 density floor (pytcad/device2d.py:2096-2100), which leaves sub-floor
# minority densities -- and low-bias currents -- converged only to ~1e-5.
SWEEP_TOL = 1e-12


def _import_reference(ref):
    os.environ["PYTCAD_NATIVE_LINSOLVE"] = "0"
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    sys.path.insert(0, ref)
    import pytcad  # noqa: F401
    from pytcad import _accel
    from pytcad import device3d as d3

    def eq_stencil(Nz, Ny, Nx, psi, n, p, C, dnp, dV, et_x, et_y, et_z,
                   hx, hy, hz, dVx, dVy, dVz, gate_rows, gate_vals, contact_k):
        shp = (Nz, Ny, Nx)
        r = lambda a: np.asarray(a).reshape(shp)           # noqa: E731
        F, rows, cols, vals = d3._poisson_eq_stencil_py(
            r(psi), r(n), r(p), r(C), r(dnp), r(dV),
            np.asarray(et_x).reshape(Nz, Ny, Nx - 1),
            np.asarray(et_y).reshape(Nz, Ny - 1, Nx),
            np.asarray(et_z).reshape(Nz - 1, Ny, Nx),
            hx, hy, hz, dVx, dVy, dVz, gate_rows, gate_vals, contact_k)
        return F.ravel(), rows, cols, vals

    def base_diag(N, dV, has_ii, dcden, dcdp, dRs_dn, dRs_dp):
        return d3._base_diagonal_coo(np.arange(N), dV,
                                     dcden if has_ii else None,
                                     dcdp if has_ii else None, dRs_dn, dRs_dp)

    shim = types.SimpleNamespace(
        device3d_poisson_eq_stencil=eq_stencil,
        device3d_poisson_flux_row=d3._poisson_flux_row_coo,
        device3d_electron_continuity=d3._electron_continuity_coo,
        device3d_hole_continuity=d3._hole_continuity_coo,
        device3d_base_diagonal=base_diag)
    _accel.core = shim
    _accel.HAVE_ACCEL = True
    return pytcad


def _geom(n, L, focus, ratio):
    """Deterministic graded node set with exactly n nodes on [0, L]: cell
    sizes grow geometrically (ratio) away from the focus points."""
    t = np.linspace(0.0, 1.0, 4001)
    x = t * L
    d = np.min(np.abs(x[:, None] - np.asarray(focus)[None, :]), axis=1)
    s = 1.0 + (ratio - 1.0) * d / (L / n)
    w = 1.0 / s
    cum = np.concatenate(([0.0], np.cumsum(0.5 * (w[1:] + w[:-1]) * np.diff(x))))
    cum /= cum[-1]
    nodes = np.interp(np.linspace(0.0, 1.0, n), cum, x)
    nodes[0], nodes[-1] = 0.0, L
    return nodes


def _next_state_current(dev, volts, opts, contact):
    """Current after one more reference Newton step from the converged state
    (a second solve_bias call takes exactly one step).  At some low-bias
    points the reference's Newton settles into a period-2 round-off limit
    cycle between two states whose currents differ by up to ~1e-5 relative
    (sub-floor minority densities); this records the cycle's other state.
    The device state is restored afterwards."""
    keep = (dev.psi.copy(), dev.n.copy(), dev.p.copy())
    dev.solve_bias(volts, opts)
    I = dev.terminal_current(contact)
    dev.psi, dev.n, dev.p = keep
    return I


def _csr(J):
    J = J.tocsr()
    J.sort_indices()
    return dict(J_data=J.data, J_indices=J.indices.astype(np.int64),
                J_indptr=J.indptr.astype(np.int64))


def elem(pt, out):
    from pytcad.kernels import bernoulli, dbernoulli
    from pytcad.contacts import ohmic_values
    from pytcad.materials import SILICON, recombination
    mags = np.concatenate([np.logspace(-9, np.log10(800.0), 400),
                           [1e-4, 1e-4 * (1 - 1e-12), 1e-4 * (1 + 1e-12),
                            0.0, 700.0, 701.0, 36.7, 1e-300]])
    x = np.concatenate([mags, -mags])
    rng = np.random.default_rng(7)
    C = np.concatenate([rng.uniform(-1, 1, 64) * 10.0 ** rng.uniform(-6, 0, 64),
                        [0.0, 1.0, -1.0]])
    nie = 10.0 ** rng.uniform(-12, -3, C.size)
    n = 10.0 ** rng.uniform(2, 20, 64)
    p = 10.0 ** rng.uniform(2, 20, 64)
    nie_r = 10.0 ** rng.uniform(9, 10.5, 64)
    tn = 10.0 ** rng.uniform(-9, -5, 64)
    tp = 10.0 ** rng.uniform(-9, -5, 64)
    R1 = recombination(n, p, nie_r, tn, tp, SILICON, auger=True)
    R0 = recombination(n, p, nie_r, tn, tp, SILICON, auger=False)
    psi0, n0, p0 = ohmic_values(C, nie, 0.3, 0.025852)
    np.savez_compressed(out, x=x, B=bernoulli(x), dB=dbernoulli(x), C=C,
                        nie=nie, ohm_psi0=psi0, ohm_n0=n0, ohm_p0=p0,
                        rn=n, rp=p, rnie=nie_r, rtn=tn, rtp=tp,
                        R_aug=np.stack(R1), R_srh=np.stack(R0))


def _dump_dev(dev, dim, extra):
    d = dict(dim=dim, T=dev.T, x=dev.mesh.x, y=dev.mesh.y,
             doping=dev.doping.ravel(), Ntot=dev.Ntot.ravel(),
             Ns=dev.Ns, LD=dev.LD, J0=dev.J0, R0=dev.R0)
    if dim == 3:
        d["z"] = dev.mesh.z
    m = dev.models
    d["models"] = np.array([m.doping_mobility, m.srh, m.auger, m.bgn])
    names, kinds, idx, vals = [], [], [], []
    for name, bc in dev.bcs.items():
        i, j = np.broadcast_arrays(bc.i, bc.j)[:2]
        if dim == 2:
            k = bc.j * dev.Nx + bc.i
        else:
            k = bc.k * dev.Nx * dev.Ny + bc.j * dev.Nx + bc.i
        names.append(name)
        idx.append(np.asarray(k, dtype=np.int64))
        if hasattr(bc, "kappa"):
            kinds.append("gate")
            vals.append([bc.kappa, bc.Vfb, bc.Vg,
                         "xyz".index(getattr(bc, "normal_axis", "y"))])
        else:
            kinds.append("contact")
            vals.append([bc.V, 0.0, 0.0, 0.0])
    d["bc_names"] = np.array(names)
    d["bc_kinds"] = np.array(kinds)
    d["bc_vals"] = np.array(vals, dtype=float)
    d["bc_ptr"] = np.cumsum([0] + [a.size for a in idx]).astype(np.int64)
    d["bc_idx"] = np.concatenate(idx) if idx else np.zeros(0, np.int64)
    d.update(extra)
    return d


def asm2d(pt, out):
    """Small Device2D: graded diode with y-varying doping, all plain-path
    models on, two contacts and a top gate; assembly at equilibrium and at a
    perturbed biased state (the FD-test pattern of
    tests/test_validation_2d.py:104-147)."""
    from pytcad.device2d import Device2D
    from pytcad.mesh2d import Mesh2D
    from pytcad.device import Models, NewtonOptions
    x = _geom(17, 1.0e-4, [0.5e-4], 1.3)
    y = _geom(11, 0.4e-4, [0.0], 1.2)
    mesh = Mesh2D(x, y)
    X, Y = np.meshgrid(x, y)
    dop = np.where(X < 0.5e-4, -3e17, 2e18) * (1.0 + 0.3 * np.exp(-Y / 1e-5))
    dev = Device2D(mesh, dop, models=Models(doping_mobility=True, srh=True,
                                            auger=True, bgn=True))
    dev.add_contact("left", i=np.zeros(mesh.Ny, int), j=np.arange(mesh.Ny))
    dev.add_contact("right", i=np.full(mesh.Ny, mesh.Nx - 1), j=np.arange(mesh.Ny))
    ig = np.arange(5, 12)
    dev.add_gate("gate", i=ig, j=np.zeros_like(ig), tox_cm=3e-7, Vfb=-0.9, Vg=0.4)
    psi_g = dev._bulk_psi_guess()
    Fp0, Jp0 = dev._residual_jacobian_poisson(psi_g)
    rows_p0 = dev._dirichlet_rows_poisson.copy()
    opts = NewtonOptions(linsolve="direct")
    dev.solve_equilibrium(opts)
    psi_eq = dev.psi.copy()
    rng = np.random.default_rng(3)
    psi = dev.psi + 0.3 * rng.standard_normal(dev.psi.shape)
    n = dev.n * np.exp(0.5 * rng.standard_normal(dev.n.shape))
    p = dev.p * np.exp(0.5 * rng.standard_normal(dev.p.shape))
    volts = {"left": 0.0, "right": 0.25}
    F, J, Jn_x, Jn_y, Jp_x, Jp_y, F_n, F_p = dev._residual_jacobian(psi, n, p, volts)
    extra = dict(psi_guess=psi_g.ravel(), Fpois=Fp0.ravel(),
                 pois_fixed=rows_p0, psi_eq=psi_eq.ravel(),
                 st_psi=psi.ravel(), st_n=n.ravel(), st_p=p.ravel(),
                 V_right=0.25, F=F, F_n=F_n.ravel(), F_p=F_p.ravel(),
                 Jn_x=Jn_x.ravel(), Jn_y=Jn_y.ravel(), Jp_x=Jp_x.ravel(),
                 Jp_y=Jp_y.ravel(), fixed=dev._dirichlet_rows.copy())
    extra.update(_csr(J))
    c = _csr(Jp0)
    extra.update({"P" + k: v for k, v in c.items()})
    np.savez_compressed(out, **_dump_dev(dev, 2, extra))


def asm3d(pt, out):
    """Small Device3D with the tri-gate BC pattern of finfet3d.py:124-150
    (top gate normal y, side gates normal z), Models() defaults."""
    from pytcad.device3d import Device3D
    from pytcad.mesh3d import Mesh3D
    from pytcad.device import NewtonOptions
    x = _geom(11, 0.12e-4, [0.04e-4, 0.08e-4], 1.3)
    y = _geom(7, 0.04e-4, [0.0], 1.3)
    z = _geom(6, 0.02e-4, [0.0, 0.02e-4], 1.3)
    mesh = Mesh3D(x, y, z)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    sd = 1e20 * np.exp(-Y ** 2 / (2 * (0.01e-4) ** 2))
    dop = -1e18 + sd * ((X < 0.04e-4) | (X > 0.08e-4))
    dev = Device3D(mesh, dop)
    isrc = np.where(x < 0.04e-4)[0]
    idrn = np.where(x > 0.08e-4)[0]
    ig = np.where((x >= 0.04e-4) & (x <= 0.08e-4))[0]
    def slab(ii):
        I, J, K = np.meshgrid(ii, np.arange(mesh.Ny), np.arange(mesh.Nz), indexing="ij")
        return I.ravel(), J.ravel(), K.ravel()
    dev.add_contact("source", *slab(isrc))
    dev.add_contact("drain", *slab(idrn))
    bi, bk = np.meshgrid(np.arange(mesh.Nx), np.arange(mesh.Nz), indexing="ij")
    dev.add_contact("body", bi.ravel(), np.full(bi.size, mesh.Ny - 1), bk.ravel())
    ti, tk = np.meshgrid(ig, np.arange(mesh.Nz), indexing="ij")
    dev.add_gate("gate_top", ti.ravel(), np.zeros(ti.size, int), tk.ravel(),
                 tox_cm=1e-7, Vfb=-0.95, Vg=0.5, normal_axis="y")
    li, lj = np.meshgrid(ig, np.arange(1, mesh.Ny), indexing="ij")
    dev.add_gate("gate_left", li.ravel(), lj.ravel(), np.zeros(li.size, int),
                 tox_cm=1e-7, Vfb=-0.95, Vg=0.5, normal_axis="z")
    dev.add_gate("gate_right", li.ravel(), lj.ravel(),
                 np.full(li.size, mesh.Nz - 1), tox_cm=1e-7, Vfb=-0.95,
                 Vg=0.5, normal_axis="z")
    psi_g = dev._bulk_psi_guess()
    Fp0, Jp0 = dev._residual_jacobian_poisson(psi_g)
    rows_p0 = dev._dirichlet_rows_poisson.copy()
    dev.solve_equilibrium(NewtonOptions(linsolve="direct"))
    rng = np.random.default_rng(5)
    psi = dev.psi + 0.3 * rng.standard_normal(dev.psi.shape)
    n = dev.n * np.exp(0.5 * rng.standard_normal(dev.n.shape))
    p = dev.p * np.exp(0.5 * rng.standard_normal(dev.p.shape))
    volts = {"source": 0.0, "drain": 0.3, "body": 0.0}
    F, J, Jn_x, Jn_y, Jn_z, Jp_x, Jp_y, Jp_z, F_n, F_p = dev._residual_jacobian(
        psi, n, p, volts)
    extra = dict(psi_guess=psi_g.ravel(), Fpois=Fp0.ravel(),
                 pois_fixed=rows_p0, psi_eq=dev.psi.ravel(),
                 st_psi=psi.ravel(), st_n=n.ravel(), st_p=p.ravel(),
                 V_drain=0.3, F=F, F_n=F_n.ravel(), F_p=F_p.ravel(),
                 Jn_x=Jn_x.ravel(), Jn_z=Jn_z.ravel(),
                 fixed=np.sort(dev._dirichlet_rows))
    extra.update(_csr(J))
    c = _csr(Jp0)
    extra.update({"P" + k: v for k, v in c.items()})
    np.savez_compressed(out, **_dump_dev(dev, 3, extra))


def diode_c1(pt, out, nx=201, ny=101, vmax=0.70):
    """The CPU-runnable plain-method workload: silicon abrupt p-n diode, 2 um x
    1 um, x graded by a symmetric geometric series (ratio 1.05) toward the
    junction at 1 um, y uniform, N_A 1e17 | N_D 1e18, constant mobility,
    SRH with tau_n = tau_p = 1e-7 s, ohmic left/right, sweep 0..vmax."""
    from pytcad.device2d import Device2D
    from pytcad.mesh2d import Mesh2D
    from pytcad.device import Models, NewtonOptions
    from pytcad.materials import Semiconductor
    x = diode_x(nx)
    y = np.linspace(0.0, 1.0e-4, ny)
    mesh = Mesh2D(x, y)
    dop = np.where(np.meshgrid(x, y)[0] < 1.0e-4, -1e17, 1e18)
    mat = Semiconductor(tau_n0=1e-7, tau_p0=1e-7, tau_Nref=1e300)
    dev = Device2D(mesh, dop, material=mat,
                   models=Models(doping_mobility=False, srh=True, auger=False, bgn=False))
    dev.add_contact("anode", i=np.zeros(ny, int), j=np.arange(ny))
    dev.add_contact("cathode", i=np.full(ny, nx - 1), j=np.arange(ny))
    opts = NewtonOptions(linsolve="direct", tol_update=SWEEP_TOL)
    t0 = time.time()
    dev.solve_equilibrium(opts)
    psi_eq = dev.psi.copy()
    Vs = np.round(np.arange(0.0, vmax + 1e-9, 0.05), 10)
    I, keep = [], {}
    t_pts = []
    I_alt = []
    for V in Vs:
        t1 = time.time()
        dev.solve_bias({"anode": float(V)}, opts)
        t_pts.append(time.time() - t1)
        I.append(dev.terminal_current("anode"))
        I_alt.append(_next_state_current(dev, {"anode": float(V)}, opts, "anode"))
        if abs(V - 0.35) < 1e-9 or abs(V - Vs[-1]) < 1e-9:
            tag = "%03d" % int(round(V * 100))
            keep["psi_" + tag] = dev.psi.ravel().copy()
            keep["n_" + tag] = dev.n.ravel().copy()
            keep["p_" + tag] = dev.p.ravel().copy()
    print(f"  diode {nx}x{ny}: {time.time() - t0:.1f} s, per point "
          f"{np.mean(t_pts):.2f} s")
    extra = dict(V=Vs, I=np.array(I), I_alt=np.array(I_alt), psi_eq=psi_eq.ravel(),
                 tol_update=SWEEP_TOL,
                 sec_per_point=np.array(t_pts), mat_tau=1e-7, **keep)
    np.savez_compressed(out, **_dump_dev(dev, 2, extra))


def transient_small(pt, out, nx=41, ny=11):
    """pytcad.transient2d.solve_transient on the 41x11 diode of diode_small:
    from equilibrium, the anode stepped to 0.3 V at t = 0, 20 fixed steps of
    10 ps (growth 1), backward Euler and Crank-Nicolson (theta 0.5); the
    per-step terminal currents of both contacts and the final states."""
    from pytcad.device2d import Device2D
    from pytcad.mesh2d import Mesh2D
    from pytcad.device import Models, NewtonOptions
    from pytcad.materials import Semiconductor
    from pytcad.transient import StepWaveform
    from pytcad.transient2d import solve_transient
    x = diode_x(nx)
    y = np.linspace(0.0, 1.0e-4, ny)
    dop = np.where(np.meshgrid(x, y)[0] < 1.0e-4, -1e17, 1e18)
    mat = Semiconductor(tau_n0=1e-7, tau_p0=1e-7, tau_Nref=1e300)
    mdl = Models(doping_mobility=False, srh=True, auger=False, bgn=False)
    opts = NewtonOptions(linsolve="direct", tol_update=SWEEP_TOL)
    dt0, t_end = 1e-11, 2e-10
    extra = dict(dt0=dt0, t_end=t_end, v_step=0.3, tol_update=SWEEP_TOL, mat_tau=1e-7)
    dev = None
    for tag, theta in (("be", 1.0), ("cn", 0.5)):
        dev = Device2D(Mesh2D(x, y), dop, material=mat, models=mdl)
        dev.add_contact("anode", i=np.zeros(ny, int), j=np.arange(ny))
        dev.add_contact("cathode", i=np.full(ny, nx - 1), j=np.arange(ny))
        dev.solve_equilibrium(opts)
        r = solve_transient(dev, {"anode": StepWaveform(0.0, 0.3, 0.0)}, t_end, dt0,
                            theta=theta, opts=opts, growth=1.0)
        extra[tag + "_t"] = np.array(r.times)
        extra[tag + "_Ia"] = np.array(r.terminal_current["anode"])
        extra[tag + "_Ic"] = np.array(r.terminal_current["cathode"])
        extra[tag + "_psi"] = dev.psi.ravel().copy()
        extra[tag + "_n"] = dev.n.ravel().copy()
        extra[tag + "_p"] = dev.p.ravel().copy()
    np.savez_compressed(out, **_dump_dev(dev, 2, extra))


def transient_growth(pt, out, nx=41, ny=11):
    """pytcad.transient2d.solve_transient with its default adaptive step
    (growth 1.5 after every step that converges within max(3, max_iter/4)
    Newton steps, capped at 64 dt0): the 41x11 diode stepped to 0.3 V from
    dt0 = 1 ps to 0.2 ns, backward Euler.  Stores the time points, the step
    history and both contacts' currents."""
    from pytcad.device2d import Device2D
    from pytcad.mesh2d import Mesh2D
    from pytcad.device import Models, NewtonOptions
    from pytcad.materials import Semiconductor
    from pytcad.transient import StepWaveform
    from pytcad.transient2d import solve_transient
    x = diode_x(nx)
    y = np.linspace(0.0, 1.0e-4, ny)
    dop = np.where(np.meshgrid(x, y)[0] < 1.0e-4, -1e17, 1e18)
    mat = Semiconductor(tau_n0=1e-7, tau_p0=1e-7, tau_Nref=1e300)
    mdl = Models(doping_mobility=False, srh=True, auger=False, bgn=False)
    opts = NewtonOptions(linsolve="direct", tol_update=SWEEP_TOL)
    dt0, t_end = 1e-12, 2e-10
    dev = Device2D(Mesh2D(x, y), dop, material=mat, models=mdl)
    dev.add_contact("anode", i=np.zeros(ny, int), j=np.arange(ny))
    dev.add_contact("cathode", i=np.full(ny, nx - 1), j=np.arange(ny))
    dev.solve_equilibrium(opts)
    r = solve_transient(dev, {"anode": StepWaveform(0.0, 0.3, 0.0)}, t_end, dt0,
                        theta=1.0, opts=opts)
    extra = dict(dt0=dt0, t_end=t_end, v_step=0.3, tol_update=SWEEP_TOL, mat_tau=1e-7,
                 t=np.array(r.times), dt_hist=np.array(r.dt_hist),
                 Ia=np.array(r.terminal_current["anode"]),
                 Ic=np.array(r.terminal_current["cathode"]), psi=dev.psi.ravel().copy())
    np.savez_compressed(out, **_dump_dev(dev, 2, extra))


def transient3d_small(pt, out, nx=21, ny=5, nz=4):
    """pytcad.transient3d.solve_transient on a small 3D diode (x graded as the
    2D diode's, 1 um x 0.4 um x 0.3 um, N_A 1e17 | N_D 1e18, constant
    lifetimes): the anode stepped to 0.3 V at t = 0, 40 fixed steps of
    0.5 ps (at 10 ps the reference's own Newton fails and halves the step),
    backward Euler and Crank-Nicolson."""
    from pytcad.device3d import Device3D
    from pytcad.mesh3d import Mesh3D
    from pytcad.device import Models, NewtonOptions
    from pytcad.materials import Semiconductor
    from pytcad.transient import StepWaveform
    from pytcad.transient3d import solve_transient
    x = diode_x(nx)
    y = np.linspace(0.0, 0.4e-4, ny)
    z = np.linspace(0.0, 0.3e-4, nz)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    dop = np.where(X < 1.0e-4, -1e17, 1e18)
    mat = Semiconductor(tau_n0=1e-7, tau_p0=1e-7, tau_Nref=1e300)
    mdl = Models(doping_mobility=False, srh=True, auger=False, bgn=False)
    opts = NewtonOptions(linsolve="direct", tol_update=SWEEP_TOL)
    dt0, t_end = 5e-13, 2e-11
    extra = dict(dt0=dt0, t_end=t_end, v_step=0.3, tol_update=SWEEP_TOL, mat_tau=1e-7)
    dev = None
    J, K = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")
    for tag, theta in (("be", 1.0), ("cn", 0.5)):
        dev = Device3D(Mesh3D(x, y, z), dop, material=mat, models=mdl)
        dev.add_contact("anode", np.zeros(J.size, int), J.ravel(), K.ravel())
        dev.add_contact("cathode", np.full(J.size, nx - 1), J.ravel(), K.ravel())
        dev.solve_equilibrium(opts)
        r = solve_transient(dev, {"anode": StepWaveform(0.0, 0.3, 0.0)}, t_end, dt0,
                            theta=theta, opts=opts, growth=1.0)
        assert len(r.times) == 41, "the reference's Newton cut a step"
        extra[tag + "_t"] = np.array(r.times)
        extra[tag + "_Ia"] = np.array(r.terminal_current["anode"])
        extra[tag + "_Ic"] = np.array(r.terminal_current["cathode"])
        extra[tag + "_psi"] = dev.psi.ravel().copy()
    np.savez_compressed(out, **_dump_dev(dev, 3, extra))


def diode_x(nx, L=2.0e-4, xj=1.0e-4, ratio=1.05):
    """nx nodes on [0, L], cell widths a symmetric geometric series growing by
    `ratio` away from xj on both sides (nx odd puts a node at xj)."""
    half = (nx - 1) // 2
    w = ratio ** np.arange(half)
    w = w / w.sum() * xj
    right = np.concatenate(([0.0], np.cumsum(w)))
    x = np.concatenate([xj - right[::-1], xj + right[1:]])
    x[0], x[-1] = 0.0, L
    return x


def trigate_small(pt, out):
    """Small tri-gate sweep (3D converged states): equilibrium, then Vd =
    0.05 V with the gates at 0.0 / 0.4 / 0.8 V, warm-started."""
    from pytcad.device3d import Device3D
    from pytcad.mesh3d import Mesh3D
    from pytcad.device import NewtonOptions
    x = _geom(24, 0.12e-4, [0.04e-4, 0.08e-4], 1.25)
    y = _geom(10, 0.04e-4, [0.0], 1.25)
    z = _geom(8, 0.02e-4, [0.0, 0.02e-4], 1.25)
    mesh = Mesh3D(x, y, z)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    sig = 0.01e-4
    src = np.exp(-np.maximum(X - 0.04e-4, 0.0) ** 2 / (2 * sig ** 2))
    drn = np.exp(-np.maximum(0.08e-4 - X, 0.0) ** 2 / (2 * sig ** 2))
    dop = -1e18 + 1e20 * (src + drn)
    dev = Device3D(mesh, dop, Ntotal=1e18 + 1e20 * (src + drn))
    isrc = np.where(x <= 0.02e-4)[0]
    idrn = np.where(x >= 0.10e-4)[0]
    ig = np.where((x > 0.04e-4) & (x < 0.08e-4))[0]
    def slab(ii):
        I, J, K = np.meshgrid(ii, np.arange(mesh.Ny), np.arange(mesh.Nz), indexing="ij")
        return I.ravel(), J.ravel(), K.ravel()
    dev.add_contact("source", *slab(isrc))
    dev.add_contact("drain", *slab(idrn))
    bi, bk = np.meshgrid(np.arange(mesh.Nx), np.arange(mesh.Nz), indexing="ij")
    dev.add_contact("body", bi.ravel(), np.full(bi.size, mesh.Ny - 1), bk.ravel())
    ti, tk = np.meshgrid(ig, np.arange(mesh.Nz), indexing="ij")
    dev.add_gate("gate_top", ti.ravel(), np.zeros(ti.size, int), tk.ravel(),
                 tox_cm=1e-7, Vfb=-1.0, normal_axis="y")
    li, lj = np.meshgrid(ig, np.arange(1, mesh.Ny), indexing="ij")
    dev.add_gate("gate_left", li.ravel(), lj.ravel(), np.zeros(li.size, int),
                 tox_cm=1e-7, Vfb=-1.0, normal_axis="z")
    dev.add_gate("gate_right", li.ravel(), lj.ravel(),
                 np.full(li.size, mesh.Nz - 1), tox_cm=1e-7, Vfb=-1.0,
                 normal_axis="z")
    opts = NewtonOptions(linsolve="direct", tol_update=SWEEP_TOL)
    t0 = time.time()
    dev.solve_equilibrium(opts)
    keep = dict(psi_eq=dev.psi.ravel().copy())
    Vg = [0.0, 0.4, 0.8]
    I, I_alt = [], []
    for v in Vg:
        volts = {"drain": 0.05, "gate_top": v, "gate_left": v, "gate_right": v}
        dev.solve_bias(volts, opts)
        I.append(dev.terminal_current("drain"))
        tag = "%02d" % int(round(v * 10))
        keep["psi_" + tag] = dev.psi.ravel().copy()
        keep["n_" + tag] = dev.n.ravel().copy()
        keep["p_" + tag] = dev.p.ravel().copy()
        I_alt.append(_next_state_current(dev, volts, opts, "drain"))
    print(f"  trigate small {mesh.N} nodes: {time.time() - t0:.1f} s")
    extra = dict(Vg=np.array(Vg), Vd=0.05, I=np.array(I), I_alt=np.array(I_alt),
                 tol_update=SWEEP_TOL, **keep)
    np.savez_compressed(out, **_dump_dev(dev, 3, extra))


def mosfet_small(pt, out):
    """A small 2D MOSFET (mosfet.py:57-87 builder) at a few gate biases."""
    from pytcad.mosfet import build_mosfet
    from pytcad.device import NewtonOptions
    dev = build_mosfet(Lg=0.1e-4, Lsd=0.1e-4, depth=0.2e-4, Na=1e17,
                       Nsd_peak=1e20, tox_cm=3e-7, nx=16, ny=10)
    opts = NewtonOptions(linsolve="direct", tol_update=SWEEP_TOL)
    dev.solve_equilibrium(opts)
    keep = dict(psi_eq=dev.psi.ravel().copy())
    I, I_alt = [], []
    Vg = [0.0, 0.6, 1.2]
    for v in Vg:
        dev.solve_bias({"drain": 0.5, "gate": v}, opts)
        I.append(dev.terminal_current("drain"))
        tag = "%02d" % int(round(v * 10))
        keep["psi_" + tag] = dev.psi.ravel().copy()
        keep["n_" + tag] = dev.n.ravel().copy()
        keep["p_" + tag] = dev.p.ravel().copy()
        I_alt.append(_next_state_current(dev, {"drain": 0.5, "gate": v}, opts, "drain"))
    extra = dict(Vg=np.array(Vg), Vd=0.5, I=np.array(I), I_alt=np.array(I_alt),
                 tol_update=SWEEP_TOL, **keep)
    np.savez_compressed(out, **_dump_dev(dev, 2, extra))


def ac_small(pt, out):
    """pytcad.ac2d.y_parameters of the small 2D MOSFET of mosfet_small, biased
    on (drain 0.5 V, gate 0.8 V): the full 4-port complex Y matrix (source,
    drain, body ohmic ports and the gate port, in device.bcs order) at
    1 Hz .. 100 GHz, plus the DC state it linearises about."""
    from pytcad.mosfet import build_mosfet
    from pytcad.device import NewtonOptions
    from pytcad.ac2d import y_parameters
    dev = build_mosfet(Lg=0.1e-4, Lsd=0.1e-4, depth=0.2e-4, Na=1e17,
                       Nsd_peak=1e20, tox_cm=3e-7, nx=16, ny=10)
    opts = NewtonOptions(linsolve="direct", tol_update=SWEEP_TOL)
    dev.solve_equilibrium(opts)
    bias = {"drain": 0.5, "gate": 0.8}
    dev.solve_bias(bias, opts)
    freqs = np.array([1.0, 1e6, 1e9, 1e10, 3e10, 1e11])
    r = y_parameters(dev, freqs)
    extra = dict(freqs=freqs, Y=r.Y, ports=np.array(r.port_names), Vd=0.5, Vg=0.8,
                 tol_update=SWEEP_TOL, psi_dc=dev.psi.ravel().copy(),
                 n_dc=dev.n.ravel().copy(), p_dc=dev.p.ravel().copy())
    np.savez_compressed(out, **_dump_dev(dev, 2, extra))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PYTCAD_REF"),
                    help="the reference's pytcad project directory (default: $PYTCAD_REF)")
    ap.add_argument("--skip-c1", action="store_true")
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    if not a.ref:
        ap.error("give --ref or set PYTCAD_REF to the reference's pytcad directory")
    pt = _import_reference(a.ref)
    jobs = [("elem", elem), ("asm2d", asm2d), ("asm3d", asm3d),
            ("mosfet_small", mosfet_small), ("trigate_small", trigate_small),
            ("diode_small", lambda pt, out: diode_c1(pt, out, nx=41, ny=11)),
            ("transient_small", transient_small),
            ("transient3d_small", transient3d_small),
            ("transient_growth", transient_growth),
            ("ac_small", ac_small),
            ("diode_c1", diode_c1)]
    for name, fn in jobs:
        if a.only and name not in a.only.split(","):
            continue
        if a.skip_c1 and name == "diode_c1":
            continue
        t0 = time.time()
        fn(pt, os.path.join(HERE, name + ".npz"))
        print(f"{name}: {time.time() - t0:.1f} s")


if __name__ == "__main__":
    main()
