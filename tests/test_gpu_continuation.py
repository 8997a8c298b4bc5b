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
