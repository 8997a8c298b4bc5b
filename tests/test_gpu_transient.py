"""The theta-scheme time stepping (tcad_b200.transient, storage term in the
GPU Newton) against the reference's own solve_transient run
(pytcad/transient2d.py, fixture transient_small: the 41x11 diode stepped to
0.3 V, 20 fixed steps of 10 ps; pytcad/transient3d.py, fixture
transient3d_small: a 21x5x4 diode, 40 steps of 0.5 ps), backward Euler and
Crank-Nicolson, Newton to the fixture's update tolerance (1e-12).  Every
step's terminal currents
within 1e-6 of max(|I|, 1e-7 x the run's peak current): the step response
falls five decades (0.28 A/cm to 1.6 nA/cm), and in its tail the two
contacts' currents differ by ~1e-13 A/cm, where the sub-floor minority
densities of each solve decide the last digits -- measured, the tail agrees
to ~1e-5 relative (1e-14 A/cm), every other step to ~1e-16.  The final
state's psi within 1e-9 V."""
import numpy as np
import pytest

import fixtures as fx

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["transient_small", "transient3d_small"])
@pytest.mark.parametrize("tag,theta", [("be", 1.0), ("cn", 0.5)])
def test_transient_matches_reference(name, tag, theta):
    import tcad_b200 as tb
    from tcad_b200.transient import StepWaveform, solve_transient
    g = fx.load(name)
    opts = tb.NewtonOptions(tol_update=float(g["tol_update"]))   # the fixture's own setting
    dev = fx.gpu_device(g, material=dict(tau_n0=1e-7, tau_p0=1e-7, tau_Nref=1e300))
    dev.solve_equilibrium()
    r = solve_transient(dev, {"anode": StepWaveform(0.0, float(g["v_step"]), 0.0)},
                        float(g["t_end"]), float(g["dt0"]), theta=theta, opts=opts,
                        growth=1.0)
    assert r.times.shape == g[tag + "_t"].shape
    assert np.allclose(r.times, g[tag + "_t"], rtol=1e-12, atol=0.0)
    for contact, key in (("anode", "_Ia"), ("cathode", "_Ic")):
        I, Iref = r.terminal_current[contact], g[tag + key]
        floor = 1e-7 * np.abs(Iref).max()
        err = np.abs(I - Iref) / np.maximum(np.abs(Iref), floor)
        assert err.max() < 1e-6, (contact, float(err.max()), int(err.argmax()))
    assert np.abs(dev.psi.ravel() - g[tag + "_psi"]).max() * dev.VT < 1e-9
    assert dev.bcs["anode"].V == pytest.approx(float(g["v_step"]))


def test_transient_adaptive_step_matches_reference():
    """The reference's DEFAULT adaptive step (growth 1.5 after every step
    that converges within max(3, max_iter/4) Newton steps, capped at 64 dt0;
    fixture transient_growth: the 41x11 diode stepped to 0.3 V from dt0 =
    1 ps to 0.2 ns, backward Euler): the same time points and step history,
    and the currents within 1e-6 of max(|I|, 1e-7 x the peak)."""
    import tcad_b200 as tb
    from tcad_b200.transient import StepWaveform, solve_transient
    g = fx.load("transient_growth")
    opts = tb.NewtonOptions(tol_update=float(g["tol_update"]))
    dev = fx.gpu_device(g, material=dict(tau_n0=1e-7, tau_p0=1e-7, tau_Nref=1e300))
    dev.solve_equilibrium()
    r = solve_transient(dev, {"anode": StepWaveform(0.0, float(g["v_step"]), 0.0)},
                        float(g["t_end"]), float(g["dt0"]), theta=1.0, opts=opts)
    assert r.times.shape == g["t"].shape
    assert np.allclose(r.times, g["t"], rtol=1e-12, atol=0.0)
    assert np.allclose(r.dt_hist, g["dt_hist"], rtol=1e-12, atol=0.0)
    for contact, key in (("anode", "Ia"), ("cathode", "Ic")):
        I, Iref = r.terminal_current[contact], g[key]
        floor = 1e-7 * np.abs(Iref).max()
        err = np.abs(I - Iref) / np.maximum(np.abs(Iref), floor)
        assert err.max() < 1e-6, (contact, float(err.max()), int(err.argmax()))
    assert np.abs(dev.psi.ravel() - g["psi"]).max() * dev.VT < 1e-9
