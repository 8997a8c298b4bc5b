"""The secant predictor moves only the start of a sweep point: with and
without it the converged states agree (psi within 1e-9 V), so do the
currents (1e-6, and against the reference's fixture), and on a finely
stepped sweep it takes fewer Newton iterations."""
import numpy as np
import pytest

import fixtures as fx

pytestmark = pytest.mark.gpu


def _run(dev, points, predictor):
    import tcad_b200 as tb
    dev.solve_equilibrium()
    opts = tb.NewtonOptions(predictor=predictor)
    I, psi, iters, ratios = [], [], 0, []
    for v in points:
        dev.solve_bias(v, opts)
        assert dev.last_converged
        I.append(dev.terminal_current("drain"))
        psi.append(dev.psi.copy())
        iters += dev.last_newton["iters"]
        ratios.append(dev.last_newton["predictor_ratio"])
    return np.array(I), psi, iters, ratios


def test_predictor_keeps_reference_parity():
    g = fx.load("mosfet_small")
    pts = [{"drain": float(g["Vd"]), "gate": float(v)} for v in g["Vg"]]
    I0, psi0, _, r0 = _run(fx.gpu_device(g), pts, "none")
    I1, psi1, _, r1 = _run(fx.gpu_device(g), pts, "secant")
    assert all(r == 0.0 for r in r0)
    assert r1[0] == 0.0 and abs(r1[2] - 1.0) < 1e-12     # equal 0.6 V gate steps
    VT = fx.gpu_device(g).VT
    for a, b in zip(psi0, psi1):
        assert np.abs(a - b).max() * VT < 1e-9
    assert fx.current_err(I1, g) < 1e-6


def test_predictor_saves_newton_steps_on_a_fine_sweep():
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    build = lambda: W.mosfet2d(tb.Device2D, nx=48, ny=24, Lg=60e-7)  # noqa: E731
    pts = W.ramp({"drain": 0.5}, 2) + [{"drain": 0.5, "gate": 0.1 * k} for k in range(11)]
    I0, psi0, it0, _ = _run(build(), pts, "none")
    I1, psi1, it1, r1 = _run(build(), pts, "secant")
    VT = build().VT
    for a, b in zip(psi0, psi1):
        assert np.abs(a - b).max() * VT < 1e-9
    assert np.all(np.abs(I1 - I0) <= 1e-6 * np.abs(I0))
    assert sum(1 for r in r1 if r != 0.0) >= 9
    assert it1 < it0
