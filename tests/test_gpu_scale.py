"""Oracle parity at the headline size: the coupled SG assembly of the full
160 x 96 x 64 tri-gate (983,040 nodes, 38M Jacobian entries; the bench's
default workload) on the GPU against the oracle's assembly of the same device
and state (oracle/dd_oracle.py, pinned bit-exact to the reference's assembly
by tests/test_oracle_golden.py).  Every tile, the measured tile depth and the
1,920 flat blocks of the full mesh are covered, which the small fixtures do
not reach.

Two states: the equilibrium the GPU solves, at zero bias; and a perturbed
state (smooth +-0.3 potential, +-50 % densities) at Vd = 0.7 V, Vg = 0.6 V.
Bar: the Jacobian within 1e-12 relative per row and entry by entry (except
the rare entries where the reference's B'(x) formula amplifies an ulp of
expm1, tests/fixtures.py TOL_ENTRY_CANCEL), the residual within 1e-12 per
row on its natural scale (|J| |x| + |F|)."""
import numpy as np
import pytest

import fixtures as fx

pytestmark = pytest.mark.gpu

TOL_ASM = 1e-12


def _rownorm_vec(F, J, x, Fref):
    scale = np.asarray(abs(J) @ np.abs(x)).ravel() + np.abs(Fref)
    scale = np.where(scale == 0, 1.0, scale)
    return float((np.abs(F - Fref) / scale).max())


def _states(dev):
    s = dev.setup
    psi = dev.psi.copy()
    n = s.nie_s * np.exp(psi)
    p = s.nie_s * np.exp(-psi)
    yield psi, n, p, {}
    zz, yy, xx = np.meshgrid(*(np.linspace(0.0, 1.0, m) for m in s.shape), indexing="ij")
    w = np.sin(7.0 * xx + 3.0 * yy) * np.cos(5.0 * zz + 1.0)
    yield (psi + 0.3 * w, n * (1.0 + 0.5 * w), p * (1.0 - 0.5 * w),
           {"drain": 0.7, "gate_top": 0.6, "gate_left": 0.6, "gate_right": 0.6})


def test_trigate_full_mesh_assembly():
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    dev = W.trigate3d(tb.Device3D)
    assert dev.N == 160 * 96 * 64
    dev.solve_equilibrium()
    assert dev.last_equilibrium["converged"]
    for psi, n, p, volts in _states(dev):
        dev._apply_voltages(volts)
        out = dev._residual_jacobian(psi, n, p, {k: v for k, v in volts.items()
                                                 if k in ("drain", "source", "body")})
        F, J, F_n, F_p = out[0], out[1], out[-2], out[-1]
        ora = fx.oracle_from_device(dev)
        Fo, Jo, Fno, Fpo = ora.residual_jacobian(psi, n, p, {k: v for k, v in volts.items()
                                                             if k in ora.contacts})
        assert np.array_equal(np.sort(dev._dirichlet_rows), np.sort(ora.fixed))
        e_elem, n_cmp, frac = fx.elem_err(J, Jo)
        assert n_cmp == np.count_nonzero(Jo.data)
        assert e_elem < fx.TOL_ENTRY_CANCEL and frac <= fx.TOL_ENTRY_FRACTION, (e_elem, frac)
        assert fx.rownorm_err(J, Jo) < TOL_ASM
        x = np.stack([psi.ravel(), n.ravel(), p.ravel()], axis=1).ravel()
        assert _rownorm_vec(F, Jo, x, Fo) < TOL_ASM
        # raw continuity residuals (the terminal-current source) per row on
        # the row's natural scale: at equilibrium they are round-off noise
        nat = np.asarray(abs(Jo) @ np.abs(x)).ravel()
        for c, mine, ref in ((1, F_n.ravel(), Fno.ravel()), (2, F_p.ravel(), Fpo.ravel())):
            scale = nat[c::3] + np.abs(ref)
            assert float((np.abs(mine - ref) / np.where(scale == 0, 1.0, scale)).max()) \
                < TOL_ASM, c
        del out, F, J, Fo, Jo


def _check_currents(I, ref, noise, floor_frac=1e-9):
    """Each current within 1e-6 of the reference (on floor_frac x the largest
    reference current), or within ten times its rounding-level spread
    (fixtures.current_noise) where that is larger."""
    I, ref = np.asarray(I, float), np.asarray(ref, float)
    floor = floor_frac * np.abs(ref).max()
    for a, (x, r, nz) in enumerate(zip(I, ref, noise)):
        assert abs(x - r) <= fx.current_tol(r, nz, floor=floor), (a, x, r, nz)


def _check_fields(VT, state, ref, what):
    e_psi, e_n, e_p = fx.field_errs(*state, *ref)
    assert e_psi * VT < 1e-9, (what, e_psi * VT)
    assert max(e_n, e_p) * VT < 1e-8, (what, e_n * VT, e_p * VT)


@pytest.mark.parametrize("batched", [False, True])
def test_trigate_downscaled_sweeps_match_oracle(batched):
    """The tri-gate Id-Vg workload at 40 x 24 x 16 (tests/golden/trigate_ds.npz,
    the oracle's exact-Newton sweeps, tests/golden/make_oracle_sweeps.py): both
    Vd branches from equilibrium, 21 points each, with the default (chosen)
    Newton options; alone, one device per branch, and batched, both branches
    in ONE 2-instance pack (the bench's headline form).  Drain, source and
    body currents within 1e-6 (on 1e-9 x the branch's largest terminal
    current), psi within 1e-9 V and the quasi-Fermi levels within 1e-8 V at
    the sampled nodes."""
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    from tcad_b200.batch import DeviceBatch
    g = fx.load("trigate_ds")
    shape = tuple(int(v) for v in g["shape"])
    idx = g["idx"]
    fpts = list(g["field_points"])
    opts = tb.NewtonOptions()
    lanes = [W.trigate3d(tb.Device3D, *shape) for _ in W.TRIGATE_VD]
    VT = lanes[0].VT
    cur = {c: np.zeros((2, len(W.TRIGATE_VG))) for c in ("drain", "source", "body")}
    if batched:
        b = DeviceBatch(lanes)
        b.solve_equilibrium(opts)
        for a in range(2):
            assert np.abs(b.state(a)[0].ravel()[idx] - g["psi_eq"]).max() * VT < 1e-9
        for q, vg in enumerate(W.TRIGATE_VG):
            res = b.solve_bias([W.trigate_bias(vd, vg) for vd in W.TRIGATE_VD], opts)
            assert all(r["converged"] for r in res), vg
            for c in cur:
                cur[c][:, q] = b.terminal_currents(c)
            if q in fpts:
                for a in range(2):
                    st = [t.ravel()[idx] for t in b.state(a)]
                    _check_fields(VT, st, g["fields"][a][fpts.index(q)], (a, vg))
    else:
        for a, (dev, vd) in enumerate(zip(lanes, W.TRIGATE_VD)):
            dev.solve_equilibrium(opts)
            assert np.abs(dev.psi.ravel()[idx] - g["psi_eq"]).max() * VT < 1e-9
            for q, vg in enumerate(W.TRIGATE_VG):
                dev.solve_bias(W.trigate_bias(vd, vg), opts)
                assert dev.last_converged, (vd, vg)
                for c in cur:
                    cur[c][a, q] = dev.terminal_current(c)
                if q in fpts:
                    st = [t.ravel()[idx] for t in (dev.psi, dev.n, dev.p)]
                    _check_fields(VT, st, g["fields"][a][fpts.index(q)], (vd, vg))
    for a in range(2):
        # each contact on its own scale, floored at 1e-9 x the branch's
        # largest terminal current: the body current (~1e-19 A, fourteen
        # decades under the drain's) is a residual sum of cancelling fluxes
        top = max(np.abs(g["I_" + c][a]).max() for c in cur)
        for c in cur:
            ref = g["I_" + c][a]
            scale = np.maximum(np.abs(ref), 1e-9 * top)
            err = float((np.abs(cur[c][a] - ref) / scale).max())
            assert err < 1e-6, (c, a, err)


def test_pin_downscaled_sweep_matches_oracle():
    """The p-i-n forward sweep (SRH + Auger, doping mobility, erfc junctions)
    at 48 x 24 x 12 against the oracle's exact-Newton sweep
    (tests/golden/pin_ds.npz): every point's anode current within 1e-6 (or
    ten times its rounding-level spread, fixtures.current_noise, where that
    is larger: the 0.5 V current, 1.2e-13 A, is such a point),
    psi within 1e-9 V and the quasi-Fermi levels within 1e-8 V at the
    sampled nodes, default Newton options."""
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    g = fx.load("pin_ds")
    dev = W.pin3d(tb.Device3D, *(int(v) for v in g["shape"]))
    idx = g["idx"]
    dev.solve_equilibrium()
    assert np.abs(dev.psi.ravel()[idx] - g["psi_eq"]).max() * dev.VT < 1e-9
    I, noise = [], []
    for k, V in enumerate(g["V"]):
        dev.solve_bias({"anode": float(V)})
        assert dev.last_converged, V
        I.append(dev.terminal_current("anode"))
        noise.append(fx.current_noise(dev, "anode"))
        st = [t.ravel()[idx] for t in (dev.psi, dev.n, dev.p)]
        _check_fields(dev.VT, st, g["fields"][k], V)
    _check_currents(I, g["I_anode"], noise)


def test_trigate_mid_points_match_oracle():
    """The tri-gate at 64 x 40 x 28 (71,680 nodes), the down-scaled size of
    the headline sweep (tests/golden/trigate_mid.npz, the oracle's exact
    Newton, tests/golden/make_oracle_sweeps.py): equilibrium psi within
    1e-9 V; then each Vd branch from equilibrium through its points with the
    default options: drain, source and body currents within 1e-6 (on 1e-9 x
    the largest terminal current, or ten times the rounding-level spread),
    psi within 1e-9 V and the quasi-Fermi levels within 1e-8 V at the
    sampled nodes."""
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    g = fx.load("trigate_mid")
    shape = tuple(int(v) for v in g["shape"])
    idx = g["idx"]
    top = max(np.abs(g["I_" + c]).max() for c in ("drain", "source", "body"))
    for vd in sorted(set(float(v) for v in g["vd"])):
        dev = W.trigate3d(tb.Device3D, *shape)
        dev.solve_equilibrium()
        assert np.abs(dev.psi.ravel()[idx] - g["psi_eq"]).max() * dev.VT < 1e-9
        for k in np.flatnonzero(np.asarray(g["vd"]) == vd):
            vg = float(g["vg"][k])
            dev.solve_bias(W.trigate_bias(vd, vg))
            assert dev.last_converged, (vd, vg)
            for c in ("drain", "source", "body"):
                I, ref = dev.terminal_current(c), float(g["I_" + c][k])
                tol = fx.current_tol(ref, fx.current_noise(dev, c), floor=1e-9 * top)
                assert abs(I - ref) <= tol, (vd, vg, c, I, ref)
            st = [t.ravel()[idx] for t in (dev.psi, dev.n, dev.p)]
            _check_fields(dev.VT, st, g["fields"][k], (vd, vg))
