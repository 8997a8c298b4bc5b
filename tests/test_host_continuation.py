"""adaptive_bias_sweep's step logic (pytcad/continuation.py:61-130) against a
fake device that converges only within `reach` of its last converged bias
and leaves a diverged state behind when it fails."""
from types import SimpleNamespace as NS

import pytest

from tcad_b200.continuation import adaptive_bias_sweep


class FakeDevice:
    def __init__(self, reach, wall=None):
        self.bcs = {"anode": NS(kind="contact"), "gate": NS(kind="gate")}
        self._have_state = False
        self.state = None
        self.reach, self.wall = reach, wall
        self.tries = []

    def solve_equilibrium(self, opts=None):
        self._have_state = True
        self.state = 0.0

    def save_state(self):
        return self.state

    def restore_state(self, st):
        self.state = st

    def solve_bias(self, voltages, opts=None):
        V = voltages["anode"]
        self.tries.append(V)
        ok = (isinstance(self.state, float) and abs(V - self.state) <= self.reach + 1e-12
              and (self.wall is None or abs(V) <= self.wall))
        self.last_converged = ok
        self.state = V if ok else "diverged"

    def terminal_current(self, name):
        assert isinstance(self.state, float), "current read from a diverged state"
        return 2.0 * self.state


def test_backs_off_and_regrows_to_the_end():
    dev = FakeDevice(reach=0.1)
    rec = adaptive_bias_sweep(dev, "anode", 0.7, 0.2)
    Vs = [r["V"] for r in rec]
    assert Vs == sorted(Vs) and abs(Vs[-1] - 0.7) < 1e-12
    assert all(abs(r["I"] - 2.0 * r["V"]) < 1e-15 for r in rec)
    steps = [b - a for a, b in zip([0.0] + Vs, Vs)]
    assert max(steps) <= 0.1 + 1e-12                   # only reachable steps accepted
    assert len(dev.tries) > len(rec)                    # some attempts failed ...
    assert dev.tries[0] == pytest.approx(0.2)           # ... the first one, at step0
    assert dev.tries[1] == pytest.approx(0.1)           # halved, from the saved state


def test_negative_direction():
    dev = FakeDevice(reach=0.25)
    rec = adaptive_bias_sweep(dev, "anode", -0.6, 0.2)
    assert [r["V"] for r in rec][-1] == pytest.approx(-0.6)
    assert all(b < a for a, b in zip([0.0] + [r["V"] for r in rec], [r["V"] for r in rec]))


def test_stalls_with_an_error_below_min_step():
    dev = FakeDevice(reach=1.0, wall=0.3)
    with pytest.raises(RuntimeError, match="stalled at V=0.29"):
        adaptive_bias_sweep(dev, "anode", 0.7, 0.1)
    # left at the last converged point, within a few min_steps of the wall
    assert isinstance(dev.state, float) and 0.3 - 4 * 0.1 / 64 < dev.state <= 0.3


def test_gate_ramp_records_no_current_without_a_contact():
    dev = FakeDevice(reach=1.0)
    dev.solve_bias = (lambda f: (lambda v, o=None: f({"anode": v["gate"]}, o)))(dev.solve_bias)
    rec = adaptive_bias_sweep(dev, "gate", 0.4, 0.2)
    assert [r["I"] for r in rec] == [None, None]
