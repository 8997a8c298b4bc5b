"""Bias ramp with step back-off over the Device2D/Device3D solve API.

The reference's adaptive_bias_sweep (pytcad/continuation.py:61-130, written
for its 1D device) ramps one terminal with a step that grows after each
converged point and is halved after a Newton failure, retrying from the last
CONFIRMED-converged state -- never from the failed iterate, which solve_bias
leaves behind -- and raises once the step falls below min_step.  This is the
same strategy for the 2D/3D devices: the state is saved and put back on the
GPU (save_state / restore_state), the sweep history of the secant predictor
included, and each accepted point records the terminal current.
"""
import warnings

import numpy as np


def adaptive_bias_sweep(device, name, v_end, step0, opts=None, *, v_start=0.0, bias=None,
                        measure=None, min_step=None, max_step=None, growth=1.5,
                        shrink=0.5, verbose=False):
    """Ramp the bias of contact or gate `name` from v_start to v_end, the
    other terminals held at `bias` ({name: V}).  After a converged point the
    step grows by `growth` up to max_step (default 8 x step0); after a
    failure it shrinks by `shrink` and the point is retried from the last
    converged state; below min_step (default step0 / 64) RuntimeError.

    Returns one {"V", "I"} record per accepted point in ramp order (v_start
    excluded), I the terminal current of contact `measure` (default `name`;
    None when `name` is a gate and no contact is given)."""
    measure = name if measure is None else measure
    if not device._have_state:
        device.solve_equilibrium(opts)
    direction = 1.0 if v_end >= v_start else -1.0
    step = abs(step0) * direction
    min_step = abs(min_step) if min_step is not None else abs(step0) / 64.0
    max_step = abs(max_step) if max_step is not None else abs(step0) * 8.0
    held = dict(bias or {})
    is_contact = device.bcs[measure].kind == "contact" if measure in device.bcs else False

    V = v_start
    records = []
    while abs(v_end - V) > 1e-12:
        if abs(step) > abs(v_end - V):
            step = v_end - V
        V_try = V + step
        saved = device.save_state()
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            device.solve_bias({**held, name: V_try}, opts)
        if device.last_converged:
            V = V_try
            I = device.terminal_current(measure) if is_contact else None
            records.append({"V": V, "I": I})
            if verbose:
                print(f"  [adaptive] V={V:+.4f}  I={I}  step={step:+.4f}")
            if abs(step) < max_step:
                step = float(np.sign(step)) * min(abs(step) * growth, max_step)
        else:
            device.restore_state(saved)
            step *= shrink
            if abs(step) < min_step:
                raise RuntimeError(
                    f"adaptive_bias_sweep stalled at V={V:.4f} approaching V={V_try:.4f}: "
                    f"step shrank below min_step={min_step:.2e} without Newton convergence")
            if verbose:
                print(f"  [adaptive] back-off at V_try={V_try:+.4f}, new step={step:+.4f}")
    return records
