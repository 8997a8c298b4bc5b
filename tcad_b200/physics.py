"""Host-side device set-up: constants, the silicon parameter set, the material
laws evaluated once per device, contact values and tensor-product meshes.

This is the part of Device2D/Device3D.__init__ that runs once per device and
produces the coefficient arrays that then live in HBM.  It keeps the
reference's formulas and operation order (so the arrays handed to the
kernels are bit-identical to the reference's) -- file:line citations are to
the reference's ``pytcad/`` package.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass

import numpy as np

# constants.py:10-14, moscap.py:60, kernels.py:29
Q = 1.602176634e-19
KB = 1.380649e-23
KB_EV = 8.617333262e-5
EPS0 = 8.8541878128e-14
EPS_OX_R = 3.9
D0_REF = 1.0


def thermal_voltage(T):
    """constants.py:18-20."""
    return KB * T / Q


@dataclass
class Semiconductor:
    """Bulk parameter set (materials.py:18-119); defaults are silicon."""
    name: str = "Silicon"
    eps_r: float = 11.7
    chi: float = 4.05
    Eg0: float = 1.1700
    varshni_alpha: float = 4.730e-4
    varshni_beta: float = 636.0
    Nc300: float = 2.86e19
    Nv300: float = 3.10e19
    mu_n_min: float = 92.0
    mu_n_max: float = 1360.0
    mu_n_Nref: float = 1.3e17
    mu_n_alpha: float = 0.91
    mu_n_Texp: float = -2.33
    mu_p_min: float = 47.7
    mu_p_max: float = 495.0
    mu_p_Nref: float = 6.3e16
    mu_p_alpha: float = 0.76
    mu_p_Texp: float = -2.23
    tau_n0: float = 1.0e-5
    tau_p0: float = 3.0e-6
    tau_Nref: float = 5.0e16
    Cn_auger: float = 2.8e-31
    Cp_auger: float = 9.9e-32
    bgn_E0: float = 6.92e-3
    bgn_N0: float = 1.3e17

    def Eg(self, T):
        return self.Eg0 - self.varshni_alpha * T ** 2 / (T + self.varshni_beta)

    def Nc(self, T):
        return self.Nc300 * (T / 300.0) ** 1.5

    def Nv(self, T):
        return self.Nv300 * (T / 300.0) ** 1.5

    def ni(self, T):
        return np.sqrt(self.Nc(T) * self.Nv(T)) * np.exp(
            -self.Eg(T) / (2.0 * KB_EV * T))


SILICON = Semiconductor()


def mobility_caughey_thomas(N, mat, T, carrier):
    """materials.py:271-290."""
    N = np.maximum(np.asarray(N, dtype=float), 1.0)
    if carrier == "n":
        mu_max = mat.mu_n_max * (T / 300.0) ** mat.mu_n_Texp
        mu_min, Nref, a = mat.mu_n_min, mat.mu_n_Nref, mat.mu_n_alpha
    else:
        mu_max = mat.mu_p_max * (T / 300.0) ** mat.mu_p_Texp
        mu_min, Nref, a = mat.mu_p_min, mat.mu_p_Nref, mat.mu_p_alpha
    return mu_min + (mu_max - mu_min) / (1.0 + (N / Nref) ** a)


def nie_effective(N, mat, T, use_bgn=True):
    """Slotboom BGN-corrected intrinsic density, materials.py:425-465."""
    ni = mat.ni(T)
    if not use_bgn:
        return np.full_like(np.asarray(N, dtype=float), ni)
    N = np.maximum(np.asarray(N, dtype=float), 1.0)
    x = np.log(N / mat.bgn_N0)
    dEg = mat.bgn_E0 * (x + np.sqrt(x * x + 0.5) - np.sqrt(0.5))
    dEg = np.where(N > mat.bgn_N0, dEg, 0.0)
    return ni * np.exp(dEg / (2.0 * KB_EV * T))


def lifetime_scharfetter(N, tau0, Nref):
    """materials.py:468-471."""
    N = np.maximum(np.asarray(N, dtype=float), 1.0)
    return tau0 / (1.0 + N / Nref)


def ohmic_values(C, nie, V, VT):
    """Neutrality + mass action at a contact (contacts.py:21-38): returns
    (ln(n0/nie), n0, p0); the contact potential is V/VT + ln(n0/nie)."""
    C = np.asarray(C, dtype=float)
    nie = np.asarray(nie, dtype=float)
    root = np.sqrt(C * C + 4.0 * nie * nie)
    maj_n = 0.5 * (C + root)
    maj_p = 0.5 * (-C + root)
    ntype = C >= 0.0
    n0 = np.where(ntype, maj_n, nie * nie / np.maximum(maj_p, 1e-300))
    p0 = np.where(ntype, nie * nie / np.maximum(maj_n, 1e-300), maj_p)
    return np.log(n0 / nie), n0, p0


def control_volume_widths(h):
    """mesh2d.py:15-27."""
    h = np.asarray(h, dtype=float)
    dv = np.zeros(h.size + 1)
    dv[1:-1] = 0.5 * (h[:-1] + h[1:])
    dv[0] = 0.5 * h[0]
    dv[-1] = 0.5 * h[-1]
    return dv


def flatband_voltage(Nsub, tox_cm, gate="n+poly", Qf=0.0, T=300.0, material=SILICON):
    """MOS flat-band voltage (moscap.py:63-90)."""
    VT = thermal_voltage(T)
    Cox = (EPS_OX_R * EPS0) / tox_cm
    ni = material.ni(T)
    nie = float(nie_effective(abs(Nsub), material, T, True))
    Ns = max(abs(float(Nsub)), ni)
    psi_b = np.arcsinh((Nsub / Ns) / (2.0 * (nie / Ns)))
    chi, Eg = material.chi, material.Eg(T)
    if isinstance(gate, (int, float)):
        phi_m = float(gate)
    elif gate == "n+poly":
        phi_m = chi
    elif gate == "p+poly":
        phi_m = chi + Eg
    elif gate == "Al":
        phi_m = 4.10
    else:
        raise ValueError(f"unknown gate '{gate}'")
    phi_semi = chi + 0.5 * Eg - psi_b * VT
    return (phi_m - phi_semi) - Q * Qf / Cox


@dataclass
class Mesh2D:
    """Tensor-product 2D mesh (mesh2d.py:30-62); node k = j*Nx + i."""
    x: np.ndarray
    y: np.ndarray

    def __post_init__(self):
        self.x = np.asarray(self.x, dtype=float)
        self.y = np.asarray(self.y, dtype=float)
        self.Nx, self.Ny = self.x.size, self.y.size
        self.N = self.Nx * self.Ny
        self.hx, self.hy = np.diff(self.x), np.diff(self.y)
        self.dVx = control_volume_widths(self.hx)
        self.dVy = control_volume_widths(self.hy)
        self.dV = np.outer(self.dVy, self.dVx).ravel()

    def idx(self, i, j):
        return j * self.Nx + i


@dataclass
class Mesh3D:
    """Tensor-product 3D mesh (mesh3d.py:18-60); k = kk*Nx*Ny + j*Nx + i."""
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray

    def __post_init__(self):
        self.x = np.asarray(self.x, dtype=float)
        self.y = np.asarray(self.y, dtype=float)
        self.z = np.asarray(self.z, dtype=float)
        self.Nx, self.Ny, self.Nz = self.x.size, self.y.size, self.z.size
        self.N = self.Nx * self.Ny * self.Nz
        self.hx, self.hy, self.hz = np.diff(self.x), np.diff(self.y), np.diff(self.z)
        self.dVx = control_volume_widths(self.hx)
        self.dVy = control_volume_widths(self.hy)
        self.dVz = control_volume_widths(self.hz)
        self.dV = (self.dVz[:, None, None] * self.dVy[None, :, None]
                   * self.dVx[None, None, :]).ravel()

    def idx(self, i, j, k):
        return k * self.Nx * self.Ny + j * self.Nx + i


def graded_nodes(n, L, focus, ratio):
    """Exactly `n` nodes on [0, L], spacing growing linearly with the distance
    d to the nearest focus point, s(d) = h0 + (ratio - 1) d -- the target
    size of pytcad/mesh.py:30-116 (graded_mesh), i.e. a geometric series of
    cell sizes with the given ratio -- with h0 chosen so that the node count
    is exactly n.  Used by the workload builders, which need explicit node
    counts.

    The node density 1/s(d) is integrated in closed form: between the
    breakpoints (ends, focus points, midpoints between focus points) d is
    linear with slope +-1, so the cell count over a piece is
    |ln(s(d_b) / s(d_a))| / g, and the count-to-position map inverts with an
    exponential."""
    focus = np.unique(np.clip(np.atleast_1d(np.asarray(focus, dtype=float)), 0.0, L))
    if n < 2:
        raise ValueError("need at least 2 nodes")
    g = ratio - 1.0
    bp = np.unique(np.concatenate(([0.0, L], focus, 0.5 * (focus[1:] + focus[:-1]))))
    a, b = bp[:-1], bp[1:]
    dist = lambda x: np.min(np.abs(np.asarray(x)[:, None] - focus[None, :]), axis=1)  # noqa: E731
    da, db = dist(a), dist(b)
    up = db >= da                      # d grows along the piece

    def counts(h0):
        if g == 0.0:
            return (b - a) / h0
        return np.abs(np.log((h0 + g * db) / (h0 + g * da))) / g

    lo, hi = L * 1e-12, 2.0 * L
    for _ in range(300):               # bisection on h0 (log scale)
        h0 = np.sqrt(lo * hi)
        if counts(h0).sum() > n - 1:
            lo = h0
        else:
            hi = h0
        if hi / lo < 1.0 + 1e-15:
            break
    h0 = np.sqrt(lo * hi)
    c = counts(h0)
    c *= (n - 1) / c.sum()             # exact total, the bisection's residue spread
    C = np.concatenate(([0.0], np.cumsum(c)))
    t = np.arange(n, dtype=float)
    seg = np.clip(np.searchsorted(C, t, side="right") - 1, 0, a.size - 1)
    u = np.minimum(t - C[seg], c[seg])
    sa = h0 + g * da[seg]
    if g == 0.0:
        dd = u * h0
    else:
        dd = np.where(up[seg], (sa * np.expm1(g * u)) / g, (sa * -np.expm1(-g * u)) / g)
    x = np.minimum(a[seg] + dd, b[seg])
    x[0], x[-1] = 0.0, L
    return x
