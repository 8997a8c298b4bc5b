"""The transient waveforms (pytcad/transient.py:45-106 restated)."""
import pytest

from tcad_b200.transient import (ConstantWaveform, PulseWaveform, RampWaveform,
                                 StepWaveform, as_waveform)


def test_waveform_values():
    s = StepWaveform(0.0, 0.3, 1e-9)
    assert (s.value(0.0), s.value(1e-9), s.value(2e-9)) == (0.0, 0.3, 0.3)
    r = RampWaveform(0.0, 1.0, 1.0, 3.0)
    assert (r.value(0.5), r.value(2.0), r.value(4.0)) == (0.0, 0.5, 1.0)
    p = PulseWaveform(0.1, 0.9, 1.0, 2.0)
    assert (p.value(0.9), p.value(1.0), p.value(2.9), p.value(3.0)) == (0.1, 0.9, 0.9, 0.1)
    assert ConstantWaveform(0.7).value(123.0) == 0.7
    assert as_waveform(0.2).value(5.0) == 0.2 and as_waveform(s) is s


def test_waveform_arguments_checked():
    with pytest.raises(ValueError):
        RampWaveform(0.0, 1.0, 2.0, 2.0)
    with pytest.raises(ValueError):
        PulseWaveform(0.0, 1.0, 0.0, 0.0)


def _reference_rule(dt, converged, n_iter, max_iter, growth, shrink, dt_max, dt_min):
    """pytcad/transient2d.py:268-290, written out as the reference has it."""
    if converged:
        if n_iter <= max(3, max_iter // 4):
            return min(dt * growth, dt_max)
        return dt
    dt = dt * shrink
    return None if dt < dt_min else dt


def test_step_rule_follows_the_reference():
    """Growth, hold, back-off and stall over a scripted run of Newton
    outcomes, including counts at the growth threshold and a cap at dt_max."""
    from tcad_b200.transient import next_step
    outcomes = [(True, 2), (True, 3), (True, 25), (True, 26), (False, 0), (True, 4),
                (False, 0), (False, 0), (True, 1), (True, 1), (True, 1), (True, 1),
                (True, 1), (True, 1), (True, 1), (True, 1), (True, 30), (False, 0)]
    for max_iter in (100, 8, 3):
        a = b = 1.0
        for conv, it in outcomes:
            a = next_step(a, conv, it, max_iter, 1.5, 0.5, 8.0, 0.2)
            b = _reference_rule(b, conv, it, max_iter, 1.5, 0.5, 8.0, 0.2)
            assert a == b, (max_iter, conv, it)
            if a is None:
                break
    # a shrink below dt_min is a stall
    assert next_step(0.3, False, 0, 100, 1.5, 0.5, 8.0, 0.2) is None


def test_step_rule_counts_newton_steps_not_polishing():
    """The GPU Newton reports its polishing steps (taken after the update
    test passed); the rule must see the reference's count, which stops at
    the update test: 25 steps + 2 polishing steps still grow at max_iter
    100 (threshold 25)."""
    from tcad_b200.transient import next_step
    res = {"iters": 27, "polish_iters": 2}
    dt = next_step(1.0, True, res["iters"] - res["polish_iters"], 100, 1.5, 0.5, 64.0, 0.01)
    assert dt == 1.5
