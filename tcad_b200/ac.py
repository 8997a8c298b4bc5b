"""Small-signal AC analysis on the GPU Jacobian: the N-port complex
admittance matrix Y(f) of a Device2D / Device3D at its converged DC point
(pytcad/ac2d.py:237-342 and pytcad/ac3d.py:187-277, ``y_parameters``).

At each frequency the linearised system is (J0 + j w_s C) du = b_port, with
J0 the DC Jacobian (contact rows stamped), C the box-integration storage
diagonal of the n and p rows at non-contact nodes (-dV, +dV;
pytcad/ac2d.py:110-128) and w_s = 2 pi f Ns / R0 the scaled angular
frequency.  An ohmic port is forced by a unit scaled voltage on its contact
nodes' potential rows; a gate port by -kappa w on its nodes' Poisson rows.
Y[i, k] is then, for an ohmic port i, S_i . du_k with S_i the sum of the raw
(unstamped) continuity rows of the contact's nodes -- the exact derivative
of terminal_current's own quantity (pytcad/ac2d.py:148-173); for a gate port
j w_s sum(kappa w (delta_ik - du_k[psi])).  Physical units: x J0 LD / VT
(2D, per unit width) or J0 LD^2 / VT (3D).

On the GPU: J0 and the raw current rows come from the assembly kernel
(TCAD_MODE_RAW / TCAD_MODE_UNSTAMPED), and each complex solve runs as its
real-equivalent system [[J0, -w C], [w C, J0]] with the real and imaginary
parts of a node interleaved, so each node is one 6 x 6 block: GPU GMRES with
6 x 6 node-block-Jacobi (``tcad_csr_krylov``).  The reference factorises the
complex matrix with SuperLU per frequency; the solution is the same to the
Krylov tolerance (rtol, default 1e-12 on the true residual).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import _lib


class YParamResult:
    """freqs [Hz]; Y complex N-port admittance, shape (len(freqs), P, P)
    [A/V per unit width in 2D, A/V in 3D]; port_names in device.bcs order
    (pytcad/ac2d.py:218-234)."""

    def __init__(self, freqs, Y, port_names):
        self.freqs = np.asarray(freqs, dtype=float)
        self.Y = np.asarray(Y, dtype=complex)
        P = len(port_names)
        if self.Y.shape != (self.freqs.size, P, P):
            raise ValueError(f"Y must have shape (len(freqs), {P}, {P}); got {self.Y.shape}")
        self.port_names = tuple(port_names)


def _storage_diag(device):
    """Diagonal of C (3N, interleaved 3k + c): -dV on the n rows, +dV on the
    p rows, 0 on the potential rows and on every contact node
    (pytcad/ac2d.py:86-128; S_n = S_p = 0 on this path)."""
    s = device.setup
    dv = [np.asarray(v, float) for v in s.dv]
    if device.dim == 2:
        dV = (dv[1][:, None] * dv[0][None, :]).ravel()
    else:
        dV = ((dv[2][:, None, None] * dv[1][None, :, None]) * dv[0][None, None, :]).ravel()
    keep = np.ones(device.N, dtype=bool)
    for b in device.bcs.values():
        if b.kind == "contact":
            keep[np.asarray(b.nodes)] = False
    c = np.zeros(3 * device.N)
    c[1::3] = np.where(keep, -dV, 0.0)
    c[2::3] = np.where(keep, dV, 0.0)
    return c


def _unstamped_jacobian(device):
    """The Jacobian with every contact row left as its assembled raw row
    (TCAD_MODE_UNSTAMPED), as scipy CSR over the interleaved numbering."""
    pk = device.pack
    pk.set_bias()
    rc = pk.lib.tcad_sg_assemble(pk.pref, _lib.ptr(pk.psi), _lib.ptr(pk.n), _lib.ptr(pk.p),
                                 _lib.ptr(pk.F), _lib.ptr(pk.J), _lib.MODE_UNSTAMPED, pk.sp())
    _lib.check(rc, "tcad_sg_assemble")
    return device._block_to_csr(pk.J.cpu().numpy(), 3)


def _real_equivalent(J, c, w):
    """[[J, -w C], [w C, J]] with node k's real parts at 6k..6k+2 and its
    imaginary parts at 6k+3..6k+5 (one 6 x 6 block per node)."""
    n3 = J.shape[0]
    Cw = sp.diags(w * c, format="csr")
    K = sp.bmat([[J, -Cw], [Cw, J]], format="csr")
    k = np.arange(n3 // 3)
    perm = np.empty(2 * n3, dtype=np.int64)      # perm[new] = old
    for q in range(3):
        perm[6 * k + q] = 3 * k + q
        perm[6 * k + 3 + q] = n3 + 3 * k + q
    K = K[perm][:, perm].tocsr()
    K.sort_indices()
    return K, perm


def _gpu_solve(K, rhs_list, rtol, maxiter, restart):
    """GMRES with 6 x 6 node-block-Jacobi on the GPU for each right-hand
    side; raises LinearSolveError when one does not converge."""
    from .linsolve import solve_linear
    out = []
    for rhs in rhs_list:
        x, info = solve_linear(K, rhs, method="gmres", rtol=rtol, maxiter=maxiter,
                               restart=restart, block_size=6)
        out.append(x)
    return out


def y_parameters(device, freqs, *, rtol=1e-12, maxiter=200, restart=200):
    """Full N-port complex Y(f) of the device at its CURRENT converged DC
    operating point (call solve_equilibrium() / solve_bias() first).  Every
    contact and gate is a port, in device.bcs order; Y[k, i, j] = dI_i/dV_j
    at freqs[k] with the other ports AC-grounded, I_i positive into terminal
    i (pytcad/ac2d.py:237-342, pytcad/ac3d.py:187-277)."""
    if not getattr(device, "_have_state", False):
        raise RuntimeError("y_parameters needs a converged DC operating point: call "
                           "solve_equilibrium() or solve_bias() first")
    freqs = np.atleast_1d(np.asarray(freqs, dtype=float))
    N = device.N
    psi0, n0, p0 = device.psi, device.n, device.p
    voltages = {name: b.V for name, b in device.bcs.items() if b.kind == "contact"}
    _, J0, *_ = device._residual_jacobian(psi0, n0, p0, voltages)
    Jraw = _unstamped_jacobian(device)
    c = _storage_diag(device)
    t0 = device.Ns / device.R0

    ports = list(device.bcs)
    P = len(ports)
    kinds, nodes, gw, S, forcing = [], [], [], [], []
    for name in ports:
        b = device.bcs[name]
        kk = np.asarray(b.nodes, dtype=np.int64)
        nodes.append(kk)
        f = np.zeros(3 * N)
        if b.kind == "contact":
            kinds.append("ohmic")
            f[3 * kk] = 1.0
            rows = np.concatenate([3 * kk + 1, 3 * kk + 2])
            S.append(np.asarray(Jraw[rows].sum(axis=0)).ravel())
            gw.append(None)
        else:
            kinds.append("gate")
            w = b.kappa * np.asarray(b.w, dtype=float)
            f[3 * kk] = -w
            gw.append(w)
            S.append(None)
        forcing.append(f)

    Y = np.empty((freqs.size, P, P), dtype=complex)
    for kf, fr in enumerate(freqs):
        ws = 2.0 * np.pi * fr * t0
        K, perm = _real_equivalent(J0, c, ws)
        rhs = [f_[perm % (3 * N)] * (perm < 3 * N) for f_ in forcing]
        sols = _gpu_solve(K, rhs, rtol, maxiter, restart)
        du = []
        for x in sols:
            z = np.empty(6 * N)
            z[perm] = x
            du.append(z[:3 * N] + 1j * z[3 * N:])
        for k in range(P):
            for i in range(P):
                if kinds[i] == "ohmic":
                    Y[kf, i, k] = S[i] @ du[k]
                else:
                    d_ik = 1.0 if i == k else 0.0
                    Y[kf, i, k] = 1j * ws * np.sum(gw[i] * (d_ik - du[k][3 * nodes[i]]))
    exp = 1 if device.dim == 2 else 2
    return YParamResult(freqs, Y * device.J0 * device.LD ** exp / device.VT, ports)


def cutoff_frequency(yres, port_in, port_out):
    """Current-gain cutoff f_T: where |h21| = |Y[out, in] / Y[in, in]|
    falls through 1, by log-log interpolation between the two computed
    frequencies around the first point below 1 (pytcad/ac2d.py:345-404).
    Ports by name or index.  None when there is no gain at the lowest
    frequency, or |h21| is still >= 1 at the highest (no extrapolation)."""
    def idx(p):
        return yres.port_names.index(p) if isinstance(p, str) else int(p)
    i_in, i_out = idx(port_in), idx(port_out)
    y_in = yres.Y[:, i_in, i_in]
    with np.errstate(divide="ignore", invalid="ignore"):
        mag = np.abs(np.where(np.abs(y_in) > 0, yres.Y[:, i_out, i_in] / y_in, np.inf))
    if not np.any(np.isfinite(mag)) or mag[0] < 1.0 or mag[-1] >= 1.0:
        return None
    i1 = int(np.where(mag < 1.0)[0][0])
    i0 = i1 - 1
    if i0 < 0:
        return None
    f = yres.freqs
    lm0, lm1 = np.log(mag[i0]), np.log(mag[i1])
    if lm0 == lm1:
        return float(f[i0])
    t = -lm0 / (lm1 - lm0)
    return float(np.exp(np.log(f[i0]) + t * (np.log(f[i1]) - np.log(f[i0]))))
