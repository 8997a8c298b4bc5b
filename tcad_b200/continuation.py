"""Continuation drivers over the Device2D/Device3D solve API: a bias ramp
with step back-off, and pseudo-arclength continuation on the GPU Jacobian.

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


class ArcLengthStalled(RuntimeError):
    """arc_length_sweep could not converge even at ds_min
    (pytcad/continuation.py:32-50).  ``last_V`` / ``last_records``: the last
    traced bias and the records before the stall."""

    def __init__(self, message, last_V, last_records):
        super().__init__(message)
        self.last_V = last_V
        self.last_records = last_records


def _block_solve(pk, rhs, x, rtol, maxiter):
    """x = A^-1 rhs for the block-scaled operator the pack's J holds after
    tcad_block_jacobi_setup (rhs already scaled); True when converged."""
    import ctypes
    from . import _lib
    it, st, rr = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_double(0.0)
    x.zero_()
    rc = pk.lib.tcad_block_krylov(pk.pref, _lib.ptr(pk.J), _lib.ptr(rhs), _lib.ptr(x), 0,
                                  rtol, maxiter, 0, _lib.ptr(pk.work), pk.work.numel(),
                                  ctypes.byref(it), ctypes.byref(st), ctypes.byref(rr),
                                  pk.sp())
    _lib.check(rc, "tcad_block_krylov")
    return st.value == _lib.TCAD_OK


class _Bordered:
    """The pseudo-arclength corrector of pytcad/continuation.py:124-216 on a
    Device2D/3D: Newton on the bordered system

        [ F(u, V)                                   ]
        [ t_u . (u - u_prev) + t_V (V - V_prev) - ds ] = 0,

    with F assembled on the GPU with its contact rows stamped (RAW mode),
    so dF/dV is -1/VT on the swept contact's potential rows.  Each step is
    solved by block elimination with two GPU Krylov solves of the block-
    scaled Jacobian in relative unknowns, J a = -F and J b = -dF/dV:
        dV = (-N_arc - t_u . a) / (t_V + t_u . b),   du = a + dV b;
    then the reference's damping: psi clipped to +-max_dpsi, n and p to
    [0.1, 10] x, Armijo backtracking on the 2-norm of the full bordered
    residual, and convergence on the undamped update (|dpsi|, |dn/n|,
    |dp/p|, |dV|) < tol.  The converged point is then finished by the
    bias-controlled Newton at its V (update test, then NewtonOptions.polish
    steps in relative Krylov unknowns), which takes the state to the FP64
    fixed point at that bias: near zero bias the current is a small
    difference of large contact fluxes, and the state at the 1e-8 update
    test of the bordered system leaves it ~3e-2 off."""

    def __init__(self, device, contact, opts, rtol=1e-10, maxiter=4000):
        import torch
        from . import _lib
        self.torch, self._lib = torch, _lib
        self.dev, self.contact, self.opts = device, contact, opts
        self.pk = device.pack
        N = device.N
        self.N = N
        self.cv = torch.zeros(3 * N, dtype=torch.float64, device=self.pk.device)
        nodes = torch.as_tensor(np.asarray(device.bcs[contact].nodes), device=self.pk.device)
        self.cv[nodes] = -1.0 / device.VT            # dF/dV on the contact's psi rows
        self.rtol, self.maxiter = rtol, maxiter
        self.floor = float(getattr(opts, "krylov_scale_floor", 1e-10))

    def state(self):
        pk = self.pk
        return self.torch.cat([pk.psi, pk.n, pk.p])

    def put(self, u):
        N = self.N
        self.pk.psi.copy_(u[:N])
        self.pk.n.copy_(u[N:2 * N])
        self.pk.p.copy_(u[2 * N:])
        self.dev._host.clear()

    def residual(self, u, V):
        """F(u, V) with the contact rows stamped (a copy, component-major)."""
        pk = self.pk
        self.put(u)
        self.dev._apply_voltages({self.contact: V})
        pk.set_bias()
        pk.assemble(self._lib.MODE_RAW)
        return pk.F.clone()

    def finish(self, u, V):
        """Newton at fixed bias V from the corrector's converged u (its update
        test passes at once; the polishing steps follow); the finished state."""
        pk = self.pk
        self.put(u)
        self.dev._apply_voltages({self.contact: V})
        pk.set_bias()
        pk.stamp_contacts()
        res = pk.newton(self.opts)[0]
        if not res["converged"]:
            self.put(u)
        self.dev._host.clear()
        return self.state()

    def correct(self, u_pred, V_pred, u_prev, V_prev, t_u, t_V, ds, tol, max_iter):
        torch, pk, N = self.torch, self.pk, self.N
        opts = self.opts
        u, V = u_pred.clone(), float(V_pred)
        a = torch.empty_like(u)
        b = torch.empty_like(u)
        st = torch.zeros(1, dtype=torch.int32, device=pk.device)
        for it in range(max_iter):
            F = self.residual(u, V)
            narc = float(torch.dot(t_u, u - u_prev)) + t_V * (V - V_prev) - ds
            base = 0.5 * (float(torch.dot(F, F)) + narc * narc)
            # relative Krylov unknowns (dpsi, dn / s_n, dp / s_p), s = max(density,
            # floor), as in the bias-controlled Newton: in absolute unknowns the
            # solves leave sub-floor minority densities unresolved, and a step
            # that does not move them passes the update test with them off
            rhs = F.clone()          # the set-up replaces it by S^-1 D^-1 (-F)
            rc = pk.lib.tcad_block_jacobi_setup_rel(
                pk.pref, self._lib.ptr(pk.J), self._lib.ptr(rhs), self._lib.ptr(st),
                self._lib.ptr(pk.n), self._lib.ptr(pk.p), self.floor, pk.sp())
            self._lib.check(rc, "tcad_block_jacobi_setup_rel")
            if int(st.item()) != 0:
                return u, V, False, it + 1
            # the contact rows' diagonal blocks are identities and their unknowns
            # potentials, so the scaled -dF/dV is -dF/dV itself
            if not (_block_solve(pk, rhs, a, self.rtol, self.maxiter)
                    and _block_solve(pk, -self.cv, b, self.rtol, self.maxiter)):
                return u, V, False, it + 1
            sn = torch.clamp(u[N:2 * N], min=self.floor)
            sp_ = torch.clamp(u[2 * N:], min=self.floor)
            for y in (a, b):
                y[N:2 * N] *= sn
                y[2 * N:] *= sp_
            den = t_V + float(torch.dot(t_u, b))
            if den == 0.0 or not np.isfinite(den):
                return u, V, False, it + 1
            dV = (-narc - float(torch.dot(t_u, a))) / den
            du = a + dV * b
            psi, n, p = u[:N], u[N:2 * N], u[2 * N:]
            dpsi = torch.clamp(du[:N], -opts.max_dpsi, opts.max_dpsi)
            dn, dp = du[N:2 * N], du[2 * N:]
            lam = 1.0
            for _ in range(40):
                u_t = torch.cat([psi + lam * dpsi,
                                 torch.minimum(torch.maximum(n + lam * dn, 0.1 * n), 10.0 * n),
                                 torch.minimum(torch.maximum(p + lam * dp, 0.1 * p), 10.0 * p)])
                V_t = V + lam * dV
                narc_t = float(torch.dot(t_u, u_t - u_prev)) + t_V * (V_t - V_prev) - ds
                Ft = self.residual(u_t, V_t)
                merit = 0.5 * (float(torch.dot(Ft, Ft)) + narc_t * narc_t)
                if np.isfinite(merit) and merit <= base * (1.0 - 1e-4 * lam):
                    break
                lam *= 0.5
            else:
                lam = 0.0
            n_new = torch.minimum(torch.maximum(n + lam * dn, 0.1 * n), 10.0 * n)
            p_new = torch.minimum(torch.maximum(p + lam * dp, 0.1 * p), 10.0 * p)
            rel_n = float((n_new / torch.clamp(n, min=1e-300) - 1.0).abs().max())
            rel_p = float((p_new / torch.clamp(p, min=1e-300) - 1.0).abs().max())
            # the undamped step decides convergence (a step backtracked to
            # nothing must not look converged)
            err = max(float(dpsi.abs().max()), rel_n, rel_p, abs(dV))
            u = torch.cat([psi + lam * dpsi, n_new, p_new])
            V = V + lam * dV
            if err < tol:
                return self.finish(u, V), V, True, it + 1
        return u, V, False, max_iter


def arc_length_sweep(device, contact, v_start, v_end, ds0, opts=None, *, bias=None,
                     ds_min=None, ds_max=None, max_steps=2000, corrector_tol=1e-8,
                     corrector_max_iter=30, seed_step=None, keep_states=False,
                     verbose=False):
    """Trace the (state, bias) solution branch of a Device2D/3D by arc length
    as contact `contact` goes from v_start toward v_end, the other terminals
    held at `bias` (pseudo-arclength continuation, Keller 1977:
    pytcad/continuation.py:267-454, there for its 1D device).  V is not
    monotone along the records where the I-V curve folds.

    The branch is seeded by two voltage-controlled solves (v_start and
    v_start + seed_step, the seed halved up to 6 times); the arc-length
    metric sees the potential unknowns and V only (the reference's choice:
    densities spanning tens of decades would dominate any norm).  ds grows
    by 1.5 (to ds_max, default 8 ds0) after a corrector that converged in at
    most max(3, corrector_max_iter // 4) steps and is halved after a failure;
    below ds_min (default ds0 / 64) ArcLengthStalled.  Returns records
    {"V", "I", "ds"} in traced order (the two seeds first, without "ds"), I
    the contact's terminal current; with keep_states also "psi", "n", "p"."""
    import torch
    from .options import NewtonOptions
    opts = opts or NewtonOptions()
    held = dict(bias or {})
    if device.bcs[contact].kind != "contact":
        raise ValueError(f"arc_length_sweep: '{contact}' is not a contact")
    if not device._have_state:
        device.solve_equilibrium(opts)
    direction = 1.0 if v_end >= v_start else -1.0
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        device.solve_bias({**held, contact: v_start}, opts)
    if not device.last_converged:
        raise RuntimeError(f"arc_length_sweep: could not seed the branch at V={v_start}")
    cor = _Bordered(device, contact, opts)
    u0, V0 = cor.state(), float(v_start)

    def record(V, ds=None):
        r = {"V": float(V), "I": device.terminal_current(contact)}
        if ds is not None:
            r["ds"] = float(ds)
        if keep_states:
            r.update(psi=device.psi.copy(), n=device.n.copy(), p=device.p.copy())
        return r

    records = [record(V0)]
    eps = abs(seed_step) if seed_step else min(abs(ds0) * 0.1, 0.5)
    for _ in range(6):
        V1 = V0 + direction * eps
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            device.solve_bias({**held, contact: V1}, opts)
        if device.last_converged:
            break
        cor.put(u0)
        eps *= 0.5
    else:
        raise RuntimeError(f"arc_length_sweep: could not seed the tangent near V={v_start}")
    u1 = cor.state()
    records.append(record(V1))
    N = device.N

    def tangent(ua, Va, ub, Vb):
        d = ub - ua
        d[N:] = 0.0                          # metric: potential unknowns and V only
        dv = Vb - Va
        nrm = float(torch.sqrt(torch.dot(d, d) + dv * dv))
        return (d / nrm, dv / nrm) if nrm > 1e-300 else (None, None)

    t_u, t_V = tangent(u0, V0, u1, V1)
    if t_u is None:
        raise RuntimeError("arc_length_sweep: degenerate initial tangent")
    u_prev, V_prev = u1, V1
    ds = abs(ds0)
    ds_min = abs(ds_min) if ds_min is not None else abs(ds0) / 64.0
    ds_max = abs(ds_max) if ds_max is not None else abs(ds0) * 8.0
    reached = False
    for step in range(max_steps):
        u_c, V_c, ok, its = cor.correct(u_prev + ds * t_u, V_prev + ds * t_V, u_prev, V_prev,
                                        t_u, t_V, ds, corrector_tol, corrector_max_iter)
        if not ok:
            cor.put(u_prev)
            ds *= 0.5
            if ds < ds_min:
                device._apply_voltages({contact: V_prev})
                raise ArcLengthStalled(
                    f"arc_length_sweep stalled near V={V_prev:.4f}: ds shrank below "
                    f"ds_min={ds_min:.2e} without corrector convergence", V_prev, records)
            continue
        nt_u, nt_V = tangent(u_prev, V_prev, u_c, V_c)
        if nt_u is not None:
            t_u, t_V = nt_u, nt_V
        records.append(record(V_c, ds))
        if verbose:
            print(f"  [arclen] step={step:4d}  V={V_c:+.4f}  I={records[-1]['I']:+.4e}  "
                  f"ds={ds:.4f}  iters={its}")
        u_prev, V_prev = u_c, V_c
        if its <= max(3, corrector_max_iter // 4):
            ds = min(ds * 1.5, ds_max)
        if (direction > 0 and V_c >= v_end) or (direction < 0 and V_c <= v_end):
            reached = True
            break
    device._bias_prev, device._bias_cur = None, None
    if not reached:
        warnings.warn(f"arc_length_sweep hit max_steps={max_steps} before reaching V={v_end} "
                      f"(last traced V={V_prev:.4f})")
    return records
