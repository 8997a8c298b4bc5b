"""Time-dependent drift-diffusion on the GPU devices: the reference's
theta-scheme time stepping (pytcad/transient2d.py:186-330 and its 3D twin
pytcad/transient3d.py) over Device2D / Device3D.

Each step solves, by Newton on the GPU, the steady residual plus the storage
term of the non-contact continuity rows (tcad_newton_opts_t.dt; the kernel
is k_storage): theta F(new) + (1 - theta) F(old) -/+ dV (n|p - old)/dt = 0,
with the Poisson rows and the contact rows unchanged.  The step size adapts
as the reference's does: a step that converged in at most
max(3, max_iter // 4) Newton iterations grows dt by `growth` (up to dt_max),
a failed step is retried from the last accepted state with dt * `shrink`,
and below dt_min the run stops with RuntimeError.  Terminal currents are the
raw continuity residuals at the contact nodes, as in terminal_current.
"""
import numpy as np

from .options import NewtonOptions
from .pack import bias_vector


class Waveform:
    """A bias in volts as a function of time in seconds: .value(t)."""

    def value(self, t):
        raise NotImplementedError


class StepWaveform(Waveform):
    """v0 before t_step, v1 from t_step on (pytcad/transient.py:52-59)."""

    def __init__(self, v0, v1, t_step=0.0):
        self.v0, self.v1, self.t_step = float(v0), float(v1), float(t_step)

    def value(self, t):
        return self.v1 if t >= self.t_step else self.v0


class RampWaveform(Waveform):
    """v0 until t0, linear to v1 at t1, v1 after (pytcad/transient.py:62-76)."""

    def __init__(self, v0, v1, t0, t1):
        if t1 <= t0:
            raise ValueError("RampWaveform requires t1 > t0")
        self.v0, self.v1, self.t0, self.t1 = float(v0), float(v1), float(t0), float(t1)

    def value(self, t):
        if t <= self.t0:
            return self.v0
        if t >= self.t1:
            return self.v1
        return self.v0 + (t - self.t0) / (self.t1 - self.t0) * (self.v1 - self.v0)


class PulseWaveform(Waveform):
    """v_pulse on [t_start, t_start + width), v_base elsewhere
    (pytcad/transient.py:79-92)."""

    def __init__(self, v_base, v_pulse, t_start, width):
        if width <= 0.0:
            raise ValueError("PulseWaveform requires width > 0")
        self.v_base, self.v_pulse = float(v_base), float(v_pulse)
        self.t_start, self.width = float(t_start), float(width)

    def value(self, t):
        return self.v_pulse if self.t_start <= t < self.t_start + self.width else self.v_base


class ConstantWaveform(Waveform):
    def __init__(self, v):
        self.v = float(v)

    def value(self, t):
        return self.v


def as_waveform(v):
    return v if isinstance(v, Waveform) else ConstantWaveform(v)


class TransientResult:
    """times [s]; psi/n/p_hist: one host snapshot (the device's shape) per
    accepted step, row 0 the initial condition; terminal_current:
    {contact: [...]} in terminal_current's unit; dt_hist [s]."""

    def __init__(self, times, psi_hist, n_hist, p_hist, terminal_current, dt_hist):
        self.times = np.asarray(times)
        self.psi_hist, self.n_hist, self.p_hist = psi_hist, n_hist, p_hist
        self.terminal_current = {k: np.asarray(v) for k, v in terminal_current.items()}
        self.dt_hist = np.asarray(dt_hist)


def next_step(step_dt, converged, newton_iters, max_iter, growth, shrink, dt_max, dt_min):
    """The adaptive step rule of pytcad/transient2d.py:268-290: after an
    accepted step, grow by `growth` (capped at dt_max) when Newton took at
    most max(3, max_iter // 4) steps to pass its update test, else keep the
    step; after a rejected step, shrink by `shrink`.  Returns the next step,
    or None when a shrunk step falls below dt_min (the run has stalled)."""
    if converged:
        if newton_iters <= max(3, max_iter // 4):
            return min(step_dt * growth, dt_max)
        return step_dt
    nxt = step_dt * shrink
    return None if nxt < dt_min else nxt


def solve_transient(device, waveforms, t_end, dt0, theta=1.0, opts=None, dt_min=None,
                    dt_max=None, growth=1.5, shrink=0.5, output_times=None, verbose=False,
                    keep_history=True):
    """Time-step `device` from its current state to t_end [s].

    waveforms: {contact: Waveform | volts}; a contact not named keeps its
    bias (names that are not contacts are ignored, as in the reference).
    theta in (0, 1]: 1 backward Euler, 0.5 Crank-Nicolson.  dt0, dt_min
    (default dt0 / 1024), dt_max (default 64 dt0) in seconds; output_times
    are landed on exactly.  keep_history=False keeps only the currents."""
    import torch
    if not 0.0 < theta <= 1.0:
        raise ValueError("theta must be in (0, 1]")
    opts = opts or NewtonOptions()
    if not device._have_state:
        raise RuntimeError("solve_transient needs an initial condition: call "
                           "solve_equilibrium() or solve_bias() first")
    wf = {name: as_waveform(v) for name, v in waveforms.items()}
    contacts = [name for name, b in device.bcs.items() if b.kind == "contact"]

    def voltages_at(t):
        return {name: (wf[name].value(t) if name in wf else device.bcs[name].V)
                for name in contacts}

    t_scale = device.Ns / device.R0
    dt_s = dt0 / t_scale
    dt_min_s = (dt_min if dt_min is not None else dt0 / 1024.0) / t_scale
    dt_max_s = (dt_max if dt_max is not None else dt0 * 64.0) / t_scale
    pk = device.pack
    all_nodes = (torch.arange(pk.N, dtype=torch.int64, device=pk.device)
                 if theta != 1.0 else None)

    t = 0.0
    times, dt_hist = [t], []
    hist = ([device.psi.copy()], [device.n.copy()], [device.p.copy()]) if keep_history \
        else ([], [], [])
    currents = {name: [device.terminal_current(name)] for name in contacts}
    out_times = sorted(output_times) if output_times else None
    out_idx = 0

    while t < t_end - 1e-15:
        step_dt_s = dt_s
        t_new = t + step_dt_s * t_scale
        if out_times is not None and out_idx < len(out_times) and t_new > out_times[out_idx]:
            t_new = out_times[out_idx]
            step_dt_s = (t_new - t) / t_scale
        if t_new > t_end:
            t_new = t_end
            step_dt_s = (t_new - t) / t_scale

        old = device.save_state()
        fn_old = fp_old = None
        if theta != 1.0:
            fn_old, fp_old = pk.raw_continuity(all_nodes, pk.psi, pk.n, pk.p)
        device._apply_voltages(voltages_at(t_new))
        pk.set_bias()
        pk.stamp_contacts()
        res = pk.newton(opts, transient=dict(dt=step_dt_s, theta=theta, n_old=old["n"],
                                             p_old=old["p"], fn_old=fn_old,
                                             fp_old=fp_old))[0]
        device._host.clear()
        if res["converged"]:
            t = t_new
            times.append(t)
            dt_hist.append(step_dt_s * t_scale)
            if keep_history:
                hist[0].append(device.psi.copy())
                hist[1].append(device.n.copy())
                hist[2].append(device.p.copy())
            for name in contacts:
                currents[name].append(device.terminal_current(name))
            if verbose:
                print(f"  [transient] t={t:.3e}s  dt={step_dt_s * t_scale:.3e}s "
                      f"iters={res['iters']}")
            if out_times is not None and out_idx < len(out_times) and \
                    abs(t - out_times[out_idx]) < 1e-15 * max(1.0, t):
                out_idx += 1
            # the reference's step-growth rule counts the Newton steps up to
            # the update test (transient2d.py _newton_step returns it + 1),
            # not the polishing steps taken after it
            dt_s = next_step(step_dt_s, True, res["iters"] - res.get("polish_iters", 0),
                             opts.max_iter, growth, shrink, dt_max_s, dt_min_s)
        else:
            device.restore_state(old)
            dt_s = next_step(step_dt_s, False, 0, opts.max_iter, growth, shrink, dt_max_s,
                             dt_min_s)
            if dt_s is None:
                raise RuntimeError(
                    f"solve_transient stalled at t={t:.3e}s approaching t={t_new:.3e}s: dt "
                    f"shrank below dt_min={dt_min_s * t_scale:.3e}s without Newton convergence")

    device._apply_voltages(voltages_at(t))
    device._bias_prev, device._bias_cur = None, bias_vector(device.setup)
    device._host.clear()
    return TransientResult(times, *hist, currents, dt_hist)
