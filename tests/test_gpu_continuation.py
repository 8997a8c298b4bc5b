"""adaptive_bias_sweep on the GPU devices: a failed solve's state is put back
bit for bit, and the swept points' currents match the same points solved in
order on a fresh device."""
import pytest

pytestmark = pytest.mark.gpu


def _diode():
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    return W.diode2d(tb.Device2D, 41, 11)


def test_restore_after_a_failed_solve_is_exact():
    import tcad_b200 as tb
    dev = _diode()
    dev.solve_equilibrium()
    st = dev.save_state()
    dev.solve_bias({"anode": 0.5}, tb.NewtonOptions(max_iter=1))
    assert not dev.last_converged
    dev.restore_state(st)
    for name in ("psi", "n", "p"):
        assert bool((getattr(dev.pack, name) == st[name]).all()), name


def test_adaptive_sweep_backs_off_and_matches_ordered_solves():
    import tcad_b200 as tb
    from tcad_b200.continuation import adaptive_bias_sweep
    opts = tb.NewtonOptions()
    dev = _diode()
    real = dev.solve_bias
    tries = []

    def first_attempt_fails(voltages, o=None):
        tries.append(voltages["anode"])
        if len(tries) == 1:   # a 1-iteration Newton leaves a non-converged iterate
            real(voltages, tb.NewtonOptions(max_iter=1))
            assert not dev.last_converged
            return dev
        return real(voltages, o)

    dev.solve_bias = first_attempt_fails
    rec = adaptive_bias_sweep(dev, "anode", 0.6, 0.3, opts)
    Vs = [r["V"] for r in rec]
    assert tries[0] == pytest.approx(0.3) and Vs[0] == pytest.approx(0.15)
    assert Vs[-1] == pytest.approx(0.6) and Vs == sorted(Vs)
    ref = _diode()
    ref.solve_equilibrium()
    for r in rec:
        ref.solve_bias({"anode": r["V"]}, opts)
        assert ref.last_converged
        I = ref.terminal_current("anode")
        assert abs(r["I"] - I) <= 1e-6 * abs(I), (r["V"], r["I"], I)


def test_arc_length_sweep_lies_on_the_oracle_branch():
    """Pseudo-arclength continuation (the bordered corrector on the GPU
    Jacobian) along the 41x11 diode's forward branch 0 -> 0.6 V: every
    traced state lies on the oracle's voltage-controlled solution at that V
    (exact Newton to 1e-12): psi within 1e-9 V and the quasi-Fermi levels
    within 1e-8 V at every node, and the current within 1e-6 relative (on
    1e-9 x the branch's largest) or within ten times its rounding-level
    spread (fixtures.current_noise), whichever is larger.  Below ~0.1 V the
    current of this device is a difference of contact fluxes so much larger
    that the last bits of the state set it: at 0.07 V the bias-controlled GPU
    Newton and the oracle reach states within 4e-15 (psi, relative n) and
    currents 7.7e-4 apart, and the oracle's own current sum at the GPU state
    gives the GPU's value.  The branch has no fold, so V increases
    monotonically, and the trace reaches v_end."""
    import numpy as np
    import fixtures as fx
    from tcad_b200.continuation import arc_length_sweep
    dev = _diode()
    dev.solve_equilibrium()
    recs = arc_length_sweep(dev, "anode", 0.0, 0.6, 0.05, keep_states=True)
    V = np.array([r["V"] for r in recs])
    assert V[-1] >= 0.6 and np.all(np.diff(V) > 0)
    assert len(recs) >= 6
    ora = fx.oracle_from_device(dev)
    ora.contacts["anode"][1] = 0.0
    ora.solve_equilibrium()
    Iref = []
    for r in recs:
        ora.solve_bias({"anode": r["V"]}, tol=1e-12)
        Iref.append(ora.terminal_current("anode"))
        e_psi, e_n, e_p = fx.field_errs(r["psi"], r["n"], r["p"], ora.psi, ora.n, ora.p)
        assert e_psi * dev.VT < 1e-9, (r["V"], e_psi * dev.VT)
        assert max(e_n, e_p) * dev.VT < 1e-8, (r["V"], e_n * dev.VT, e_p * dev.VT)
    floor = 1e-9 * np.abs(Iref).max()
    for r, I_ref in zip(recs, Iref):
        noise = fx.current_noise(dev, "anode", state=(r["psi"], r["n"], r["p"]))
        assert abs(r["I"] - I_ref) <= fx.current_tol(I_ref, noise, floor=floor), \
            (r["V"], r["I"], I_ref, noise)


def test_arc_length_sweep_stalls_loudly():
    """A corrector that cannot converge (one Newton step allowed) halves ds
    down to ds_min and raises ArcLengthStalled with the traced records."""
    import pytest as _pt
    from tcad_b200.continuation import ArcLengthStalled, arc_length_sweep
    dev = _diode()
    dev.solve_equilibrium()
    with _pt.raises(ArcLengthStalled) as ei:
        arc_length_sweep(dev, "anode", 0.0, 0.6, 0.2, corrector_tol=1e-30,
                         corrector_max_iter=1, ds_min=0.05)
    assert len(ei.value.last_records) == 2 and ei.value.last_V > 0.0
