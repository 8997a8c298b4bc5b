"""GPU parity: the sm_100a kernels against the reference's own outputs (golden
fixtures) and the oracle.  Tolerances (the drop-in contract): assembled
residual / Jacobian entries within 1e-12 relative (the Jacobian both
normwise per row and entry by entry; the residual per row, where the
converging terms cancel),
converged psi within 1e-9 V, terminal currents within 1e-6 relative."""
import numpy as np
import pytest

import fixtures as fx

pytestmark = pytest.mark.gpu

TOL_ASM = 1e-12
TOL_PSI_V = 1e-9
TOL_I = 1e-6


def _rownorm_vec(F, J, x, Fref):
    """|F - Fref| per row against the row's natural magnitude: the sum of the
    absolute terms that make it up, estimated as |J|*|x| + |Fref|."""
    scale = np.asarray(abs(J) @ np.abs(x)).ravel() + np.abs(Fref)
    scale = np.where(scale == 0, 1.0, scale)
    return float((np.abs(F - Fref) / scale).max())


@pytest.mark.parametrize("name", ["asm2d", "asm3d"])
def test_coupled_assembly(name):
    g = fx.load(name)
    dev = fx.gpu_device(g)
    volts = {"right": float(g["V_right"])} if "V_right" in g else \
        {"drain": float(g["V_drain"])}
    out = dev._residual_jacobian(g["st_psi"], g["st_n"], g["st_p"], volts)
    F, J = out[0], out[1]
    F_n, F_p = out[-2], out[-1]
    Jref = fx.csr(g)
    assert fx.rownorm_err(J, Jref) < TOL_ASM
    # and entry by entry, not only normwise per row
    e_elem, n_cmp, frac = fx.elem_err(J, Jref)
    assert n_cmp == np.count_nonzero(Jref.data)
    assert e_elem < fx.TOL_ENTRY_CANCEL and frac <= fx.TOL_ENTRY_FRACTION, (e_elem, frac)
    x = np.stack([g["st_psi"], g["st_n"], g["st_p"]], axis=1).ravel()
    assert _rownorm_vec(F, Jref, x, g["F"]) < TOL_ASM
    assert np.array_equal(np.sort(dev._dirichlet_rows), np.sort(g["fixed"]))
    # raw continuity residuals (terminal-current source)
    for mine, ref in ((F_n.ravel(), g["F_n"]), (F_p.ravel(), g["F_p"])):
        assert fx.vec_err(mine, ref, 1e-12 * np.abs(ref).max()) < 1e-10


@pytest.mark.parametrize("name", ["asm2d", "asm3d"])
def test_poisson_assembly(name):
    g = fx.load(name)
    dev = fx.gpu_device(g)
    F, J = dev._residual_jacobian_poisson(g["psi_guess"])
    Jref = fx.csr(g, "P")
    assert fx.rownorm_err(J, Jref) < TOL_ASM
    assert _rownorm_vec(F.ravel(), Jref, g["psi_guess"], g["Fpois"]) < TOL_ASM
    assert np.array_equal(np.sort(dev._dirichlet_rows_poisson), np.sort(g["pois_fixed"]))


@pytest.mark.parametrize("name", ["asm2d", "asm3d", "trigate_small", "mosfet_small"])
def test_equilibrium(name):
    g = fx.load(name)
    dev = fx.gpu_device(g).solve_equilibrium()
    assert dev.last_equilibrium["converged"]
    assert np.abs(dev.psi.ravel() - g["psi_eq"]).max() * dev.VT < TOL_PSI_V


def test_diode_small_sweep():
    g = fx.load("diode_small")
    dev = fx.gpu_device(g, material=dict(tau_n0=1e-7, tau_p0=1e-7, tau_Nref=1e300))
    dev.solve_equilibrium()
    I = []
    for V in g["V"]:
        dev.solve_bias({"anode": float(V)})
        assert dev.last_converged, V
        I.append(dev.terminal_current("anode"))
    assert fx.current_err(I, g) < TOL_I


def test_mosfet_small_sweep():
    g = fx.load("mosfet_small")
    dev = fx.gpu_device(g)
    dev.solve_equilibrium()
    I = []
    for v, Iref in zip(g["Vg"], g["I"]):
        dev.solve_bias({"drain": float(g["Vd"]), "gate": float(v)})
        assert dev.last_converged
        tag = "%02d" % int(round(v * 10))
        assert np.abs(dev.psi.ravel() - g["psi_" + tag]).max() * dev.VT < TOL_PSI_V
        I.append(dev.terminal_current("drain"))
    assert fx.current_err(I, g) < TOL_I


def test_trigate_small_sweep():
    g = fx.load("trigate_small")
    dev = fx.gpu_device(g)
    dev.solve_equilibrium()
    I = []
    for v, Iref in zip(g["Vg"], g["I"]):
        dev.solve_bias({"drain": float(g["Vd"]), "gate_top": float(v),
                        "gate_left": float(v), "gate_right": float(v)})
        assert dev.last_converged
        tag = "%02d" % int(round(v * 10))
        assert np.abs(dev.psi.ravel() - g["psi_" + tag]).max() * dev.VT < TOL_PSI_V
        I.append(dev.terminal_current("drain"))
    assert fx.current_err(I, g) < TOL_I


def test_smoke_entry():
    import __graft_entry__
    __graft_entry__.smoke()


def test_diode_c1_sweep():
    """The 201x101 plain-method diode: equilibrium and the 0..0.7 V sweep,
    every point converged, currents within 1e-6 of the reference's."""
    g = fx.load("diode_c1")
    dev = fx.gpu_device(g, material=dict(tau_n0=1e-7, tau_p0=1e-7, tau_Nref=1e300))
    dev.solve_equilibrium()
    assert np.abs(dev.psi.ravel() - g["psi_eq"]).max() * dev.VT < TOL_PSI_V
    I = []
    for V in g["V"]:
        dev.solve_bias({"anode": float(V)})
        assert dev.last_converged, V
        I.append(dev.terminal_current("anode"))
        tag = "%03d" % int(round(V * 100))
        if "psi_" + tag in g:
            assert np.abs(dev.psi.ravel() - g["psi_" + tag]).max() * dev.VT < TOL_PSI_V
            VT = dev.VT
            for c, sgn in (("n", -1.0), ("p", 1.0)):
                phi = dev.psi.ravel() + sgn * np.log(getattr(dev, c).ravel() / dev.nie_s.ravel())
                phr = g["psi_" + tag] + sgn * np.log(g[c + "_" + tag] / dev.nie_s.ravel())
                assert np.abs(phi - phr).max() * VT < 1e-8, c
    assert fx.current_err(I, g) < TOL_I


@pytest.mark.parametrize("name", ["mosfet_small", "trigate_small"])
def test_mixed_precision_sweep(name):
    """The mixed-precision Newton (FP32 Krylov on an FP32 copy of the
    block-scaled Jacobian inside FP64 iterative refinement) converges to the
    same FP64 discrete solution: psi within 1e-9 V, currents within 1e-6."""
    import tcad_b200 as tb
    g = fx.load(name)
    dev = fx.gpu_device(g)
    dev.solve_equilibrium()
    opts = tb.NewtonOptions(precision="mixed")
    gates = [b for b in dev.bcs if b.startswith("gate")]
    I = []
    for v in g["Vg"]:
        volts = {"drain": float(g["Vd"]), **{gt: float(v) for gt in gates}}
        dev.solve_bias(volts, opts)
        assert dev.last_converged
        tag = "%02d" % int(round(v * 10))
        assert np.abs(dev.psi.ravel() - g["psi_" + tag]).max() * dev.VT < TOL_PSI_V
        I.append(dev.terminal_current("drain"))
    assert fx.current_err(I, g) < TOL_I


def test_mixed_precision_diode_c1():
    """Mixed precision on the 201x101 diode: where an FP32-solved step would
    be rejected (density clip hit, breakdown) the instance falls back to FP64
    on the GPU; the sweep still converges to the reference's currents."""
    import tcad_b200 as tb
    g = fx.load("diode_c1")
    dev = fx.gpu_device(g, material=dict(tau_n0=1e-7, tau_p0=1e-7, tau_Nref=1e300))
    dev.solve_equilibrium()
    opts = tb.NewtonOptions(precision="mixed")
    I = []
    for V in g["V"]:
        dev.solve_bias({"anode": float(V)}, opts)
        assert dev.last_converged, V
        I.append(dev.terminal_current("anode"))
    assert fx.current_err(I, g) < TOL_I
