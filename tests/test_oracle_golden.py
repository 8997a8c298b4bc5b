"""Pin the oracle (CPU restatement) against the reference's own outputs.

The fixtures come from running the unmodified reference
(tests/golden/make_golden.py).  The oracle follows the reference's
operation order, so the assembly comparisons are at round-off level; the
converged-state comparisons use the drop-in tolerances (psi 1e-9 V,
currents 1e-6 relative)."""
import os

import numpy as np
import pytest

import fixtures as fx
from oracle import (bernoulli, dbernoulli, ohmic_values, recombination,
                    SILICON_PARAMS)


def test_elementwise_kernels():
    g = fx.load("elem")
    assert np.array_equal(bernoulli(g["x"]), g["B"])
    assert fx.vec_err(dbernoulli(g["x"]), g["dB"]) < 1e-15
    psi0, n0, p0 = ohmic_values(g["C"], g["nie"], 0.3, 0.025852)
    assert np.array_equal(psi0, g["ohm_psi0"])
    assert np.array_equal(n0, g["ohm_n0"]) and np.array_equal(p0, g["ohm_p0"])
    m = SILICON_PARAMS
    for auger, key in ((True, "R_aug"), (False, "R_srh")):
        R = recombination(g["rn"], g["rp"], g["rnie"], g["rtn"], g["rtp"],
                          m["Cn_auger"], m["Cp_auger"], auger=auger)
        assert np.array_equal(np.stack(R), g[key])


@pytest.mark.parametrize("name", ["asm2d", "asm3d"])
def test_assembly_matches_reference(name):
    g = fx.load(name)
    dev = fx.oracle_device(g)
    assert dev.Ns == g["Ns"] and dev.LD == g["LD"] and dev.J0 == g["J0"]
    # equilibrium Poisson at the bulk guess
    psi_g = dev.bulk_guess()
    assert np.array_equal(psi_g.ravel(), g["psi_guess"])
    Fp, Jp = dev.residual_jacobian_poisson(psi_g)
    assert fx.vec_err(Fp.ravel(), g["Fpois"], 1e-300) < 1e-13
    assert fx.rownorm_err(Jp, fx.csr(g, "P")) < 1e-14
    assert np.array_equal(np.sort(dev.fixed_poisson), np.sort(g["pois_fixed"]))
    # coupled system at a perturbed, biased state
    volts = {"right": float(g["V_right"])} if "V_right" in g else \
        {"drain": float(g["V_drain"])}
    F, J, F_n, F_p = dev.residual_jacobian(g["st_psi"], g["st_n"], g["st_p"], volts)
    ref_J = fx.csr(g)
    assert fx.rownorm_err(J, ref_J) < 1e-14
    assert np.array_equal(np.sort(dev.fixed), np.sort(g["fixed"]))
    # residual rows: scale by the row's Jacobian norm x state magnitude
    assert fx.vec_err(F, g["F"], 1e-30) < 1e-12
    assert fx.vec_err(F_n.ravel(), g["F_n"], 1e-30) < 1e-12
    assert fx.vec_err(F_p.ravel(), g["F_p"], 1e-30) < 1e-12


@pytest.mark.parametrize("name", ["asm2d", "asm3d"])
def test_equilibrium_matches_reference(name):
    g = fx.load(name)
    dev = fx.oracle_device(g).solve_equilibrium()
    assert np.abs(dev.psi.ravel() - g["psi_eq"]).max() * dev.VT < 1e-9


def _sweep(g, volts_of, tags, dev):
    I = []
    for v, tag in zip(g[volts_of[0]], tags):
        dev.solve_bias(volts_of[1](float(v)), tol=float(g["tol_update"]))
        assert dev.last_converged
        I.append(dev.terminal_current(volts_of[2]))
        if "psi_" + tag in g:
            assert np.abs(dev.psi.ravel() - g["psi_" + tag]).max() * dev.VT < 1e-9
    return np.array(I)


def test_diode_small_sweep():
    g = fx.load("diode_small")
    dev = fx.oracle_device(g, material=dict(tau_n0=1e-7, tau_p0=1e-7,
                                            tau_Nref=1e300))
    dev.solve_equilibrium()
    assert np.abs(dev.psi.ravel() - g["psi_eq"]).max() * dev.VT < 1e-9
    I = []
    for V in g["V"]:
        dev.solve_bias({"anode": float(V)}, tol=float(g["tol_update"]))
        assert dev.last_converged
        I.append(dev.terminal_current("anode"))
    assert fx.current_err(I, g) < 1e-6


def test_mosfet_small_sweep():
    g = fx.load("mosfet_small")
    dev = fx.oracle_device(g)
    dev.solve_equilibrium()
    assert np.abs(dev.psi.ravel() - g["psi_eq"]).max() * dev.VT < 1e-9
    tags = ["%02d" % int(round(v * 10)) for v in g["Vg"]]
    I = _sweep(g, ("Vg", lambda v: {"drain": float(g["Vd"]), "gate": v}, "drain"),
               tags, dev)
    assert fx.current_err(I, g) < 1e-6


def test_trigate_small_sweep():
    g = fx.load("trigate_small")
    dev = fx.oracle_device(g)
    dev.solve_equilibrium()
    assert np.abs(dev.psi.ravel() - g["psi_eq"]).max() * dev.VT < 1e-9
    tags = ["%02d" % int(round(v * 10)) for v in g["Vg"]]
    vb = lambda v: {"drain": float(g["Vd"]), "gate_top": v,  # noqa: E731
                    "gate_left": v, "gate_right": v}
    I = _sweep(g, ("Vg", vb, "drain"), tags, dev)
    assert fx.current_err(I, g) < 1e-6


@pytest.mark.skipif(not os.path.exists(os.path.join(fx.GOLDEN, "diode_c1.npz")),
                    reason="full diode fixture not generated")
def test_diode_c1_equilibrium():
    g = fx.load("diode_c1")
    dev = fx.oracle_device(g, material=dict(tau_n0=1e-7, tau_p0=1e-7,
                                            tau_Nref=1e300))
    dev.solve_equilibrium()
    assert np.abs(dev.psi.ravel() - g["psi_eq"]).max() * dev.VT < 1e-9


@pytest.mark.parametrize("name", ["transient_small", "transient3d_small"])
@pytest.mark.parametrize("tag,theta", [("be", 1.0), ("cn", 0.5)])
def test_transient_matches_reference(name, tag, theta):
    """The oracle's theta-scheme time stepping against the reference's own
    solve_transient run (transient2d.py / transient3d.py)."""
    g = fx.load(name)
    dev = fx.oracle_device(g, material=dict(tau_n0=1e-7, tau_p0=1e-7, tau_Nref=1e300))
    tol = float(g["tol_update"])
    dev.solve_equilibrium(tol=tol)
    v = float(g["v_step"])
    r = dev.solve_transient({"anode": (lambda t: v if t >= 0.0 else 0.0)},
                            float(g["t_end"]), float(g["dt0"]), theta=theta, tol=tol,
                            growth=1.0)
    assert np.array_equal(r["times"], g[tag + "_t"])
    for c, key in (("anode", "_Ia"), ("cathode", "_Ic")):
        I, Iref = r["currents"][c], g[tag + key]
        err = np.abs(I - Iref) / np.maximum(np.abs(Iref), 1e-7 * np.abs(Iref).max())
        assert err.max() < 1e-9, (c, float(err.max()), int(err.argmax()))
    assert np.abs(dev.psi.ravel() - g[tag + "_psi"]).max() * dev.VT < 1e-12
