"""ORACLE -- test infrastructure only (see ``oracle/__init__.py``).

A numpy/scipy restatement of PyTCAD's plain structured drift-diffusion path
(Boltzmann statistics, full ionisation, single material, SRH + optional
Auger, optional Caughey-Thomas mobility and Slotboom BGN, ohmic contacts,
oxide-gate Robin BCs).  The arithmetic follows the reference's operation
order so that the fixtures generated from the reference itself pin it to
round-off.  Written axis-generically: one code path serves the 2D 5-point
(Device2D) and the 3D 7-point (Device3D) stencils.

Reference files (paths relative to the reference's ``pytcad/``):
  constants.py:10-14, kernels.py:29,88-109, materials.py:18-121,271-290,
  442-518, mesh2d.py:15-27, contacts.py:21-38, dirichlet.py:270-300,
  linsolve.py:363-427,941-985, device2d.py:168-453,676-759,844-942,
  1308-1373,1402-2227, device3d.py:190-258,320-408,437-724,774-947,
  952-1020,1311-1454,1485-2306, moscap.py:60-90, transient2d.py:94-330,
  transient3d.py:108-380.
"""
from __future__ import annotations

import dataclasses
import warnings

import numpy as np
import scipy.sparse as sp
from scipy.sparse.linalg import LinearOperator, bicgstab, gmres, spsolve

# constants.py:10-14, moscap.py:60, kernels.py:29
Q = 1.602176634e-19
KB = 1.380649e-23
KB_EV = 8.617333262e-5
EPS0 = 8.8541878128e-14
EPS_OX_R = 3.9
D0_REF = 1.0

# materials.py:18-119 -- the silicon parameter table (Semiconductor defaults)
SILICON_PARAMS = dict(
    eps_r=11.7, chi=4.05, Eg0=1.1700, varshni_alpha=4.730e-4,
    varshni_beta=636.0, Nc300=2.86e19, Nv300=3.10e19,
    mu_n_min=92.0, mu_n_max=1360.0, mu_n_Nref=1.3e17, mu_n_alpha=0.91,
    mu_n_Texp=-2.33, mu_p_min=47.7, mu_p_max=495.0, mu_p_Nref=6.3e16,
    mu_p_alpha=0.76, mu_p_Texp=-2.23, tau_n0=1.0e-5, tau_p0=3.0e-6,
    tau_Nref=5.0e16, Cn_auger=2.8e-31, Cp_auger=9.9e-32, bgn_E0=6.92e-3,
    bgn_N0=1.3e17)


@dataclasses.dataclass
class OracleModels:
    """The subset of ``device.py:373-535`` Models flags on the plain path."""
    doping_mobility: bool = True
    srh: bool = True
    auger: bool = True
    bgn: bool = True


# ---------------------------------------------------------------------------
# material laws (materials.py)
# ---------------------------------------------------------------------------
def _eg(m, T):                       # materials.py:89-95 (Varshni)
    return m["Eg0"] - m["varshni_alpha"] * T ** 2 / (T + m["varshni_beta"])


def _ni(m, T):                       # materials.py:103-113
    nc = m["Nc300"] * (T / 300.0) ** 1.5
    nv = m["Nv300"] * (T / 300.0) ** 1.5
    return np.sqrt(nc * nv) * np.exp(-_eg(m, T) / (2.0 * KB_EV * T))


def _mobility(N, m, T, carrier):     # materials.py:271-290 (Caughey-Thomas)
    N = np.maximum(np.asarray(N, dtype=float), 1.0)
    c = "mu_" + carrier + "_"
    mu_max = m[c + "max"] * (T / 300.0) ** m[c + "Texp"]
    return m[c + "min"] + (mu_max - m[c + "min"]) / (
        1.0 + (N / m[c + "Nref"]) ** m[c + "alpha"])


def _nie(N, m, T, bgn):              # materials.py:425-465 (Slotboom BGN)
    ni = _ni(m, T)
    if not bgn:
        return np.full_like(np.asarray(N, dtype=float), ni)
    N = np.maximum(np.asarray(N, dtype=float), 1.0)
    x = np.log(N / m["bgn_N0"])
    dEg = m["bgn_E0"] * (x + np.sqrt(x * x + 0.5) - np.sqrt(0.5))
    dEg = np.where(N > m["bgn_N0"], dEg, 0.0)
    return ni * np.exp(dEg / (2.0 * KB_EV * T))


def _lifetime(N, tau0, Nref):        # materials.py:468-471 (Scharfetter)
    N = np.maximum(np.asarray(N, dtype=float), 1.0)
    return tau0 / (1.0 + N / Nref)


def recombination(n, p, nie, tau_n, tau_p, Cn, Cp, auger=True):
    """SRH (mid-gap) + Auger rate and exact dR/dn, dR/dp, physical units.
    materials.py:474-518 (Boltzmann branch, np_eq=None)."""
    excess = n * p - nie * nie
    den = tau_p * (n + nie) + tau_n * (p + nie)
    R = excess / den
    dRdn = (p * den - excess * tau_p) / den ** 2
    dRdp = (n * den - excess * tau_n) / den ** 2
    if auger:
        cc = Cn * n + Cp * p
        R = R + cc * excess
        dRdn = dRdn + Cn * excess + cc * p
        dRdp = dRdp + Cp * excess + cc * n
    return R, dRdn, dRdp


# ---------------------------------------------------------------------------
# kernels.py:88-109 -- Bernoulli function and derivative
# ---------------------------------------------------------------------------
def bernoulli(x):
    x = np.clip(np.asarray(x, dtype=float), -700.0, 700.0)
    tiny = np.abs(x) < 1e-4
    safe = np.where(tiny, 1.0, x)
    return np.where(tiny, 1.0 - x / 2.0 + x * x / 12.0, safe / np.expm1(safe))


def dbernoulli(x):
    x = np.clip(np.asarray(x, dtype=float), -700.0, 700.0)
    tiny = np.abs(x) < 1e-4
    safe = np.where(tiny, 1.0, x)
    b = np.where(tiny, 1.0, safe / np.expm1(safe))
    one_minus = -np.expm1(-safe)
    one_minus = np.where(np.abs(one_minus) < 1e-300, 1e-300, one_minus)
    return np.where(tiny, -0.5 + x / 6.0 - x ** 3 / 180.0,
                    b * (1.0 / safe - 1.0 / one_minus))


def ohmic_values(C, nie, V, VT):
    """Charge-neutral, mass-action contact values.  contacts.py:21-38."""
    C = np.asarray(C, dtype=float)
    nie = np.asarray(nie, dtype=float)
    root = np.sqrt(C * C + 4.0 * nie * nie)
    maj_n = 0.5 * (C + root)
    maj_p = 0.5 * (-C + root)
    ntype = C >= 0.0
    n0 = np.where(ntype, maj_n, nie * nie / np.maximum(maj_p, 1e-300))
    p0 = np.where(ntype, nie * nie / np.maximum(maj_n, 1e-300), maj_p)
    return V / VT + np.log(n0 / nie), n0, p0


def control_volume_widths(h):
    """Box widths: half-intervals summed per node.  mesh2d.py:15-27."""
    h = np.asarray(h, dtype=float)
    dv = np.zeros(h.size + 1)
    dv[1:-1] = 0.5 * (h[:-1] + h[1:])
    dv[0] = 0.5 * h[0]
    dv[-1] = 0.5 * h[-1]
    return dv


def eliminate_csr(J, rhs, fixed):
    """Symmetric Dirichlet elimination: fold the known updates of the fixed
    rows into the right-hand side and empty their columns.
    dirichlet.py:270-300 (+ the `_mask` helper at :85-88)."""
    n = J.shape[0]
    rhs = np.array(rhs, dtype=float, copy=True)
    mask = np.zeros(n, dtype=bool)
    mask[fixed] = True
    if not mask.any():
        return J.tocsr(), rhs
    g = np.zeros(n)
    g[mask] = rhs[mask]
    Jc = J.tocsr()
    rhs = rhs - Jc @ g
    rhs[mask] = g[mask]
    out = Jc @ sp.diags((~mask).astype(float), format="csr")
    out = out + sp.diags(mask.astype(float), format="csr")
    return out.tocsr(), rhs


def build_block_jacobi(A, bs):
    """Node-block-Jacobi inverse blocks; None when singular.
    linsolve.py:363-427."""
    n = A.shape[0]
    if n % bs:
        return None
    nb = n // bs
    Ac = A.tocsr()
    blocks = np.zeros((nb, bs, bs))
    base = np.arange(nb) * bs
    for r in range(bs):
        for c in range(bs):
            d = Ac.diagonal(c - r)
            blocks[:, r, c] = d[base + r] if c >= r else d[base + c]
    det = np.linalg.det(blocks)
    if not np.all(np.isfinite(det)) or np.any(np.abs(det) < 1e-300):
        return None
    return np.linalg.inv(blocks)


def solve_linear_iterative(A, b, method="bicgstab", rtol=1e-10, maxiter=500,
                           block_size=3, restart=None, x0=None):
    """scipy GMRES/BiCGStab, right node-block-Jacobi preconditioning and
    the true-residual acceptance test.  linsolve.py:941-985.
    Returns (x, iterations, converged, relative_residual)."""
    A = A.tocsr()
    inv = build_block_jacobi(A, block_size) if block_size else None
    M = None
    if inv is not None:
        nb = A.shape[0] // block_size

        def apply(v):
            return np.einsum("nij,nj->ni", inv,
                             v.reshape(nb, block_size)).ravel()
        M = LinearOperator(A.shape, apply)
    count = [0]

    def cb(_):
        count[0] += 1
    kw = dict(rtol=rtol, atol=0.0, maxiter=maxiter, M=M, x0=x0, callback=cb)
    if method == "gmres":
        kw["callback_type"] = "pr_norm"
        kw["restart"] = min(restart or 100, A.shape[0])
        x, code = gmres(A, b, **kw)
    else:
        x, code = bicgstab(A, b, **kw)
    res = float(np.linalg.norm(A @ x - b)) / max(float(np.linalg.norm(b)),
                                                1e-300)
    ok = code == 0 and bool(np.all(np.isfinite(x))) and res <= max(rtol, 1e-6)
    return x, count[0], ok, res


# ---------------------------------------------------------------------------
# the device
# ---------------------------------------------------------------------------
def _face(dv, dim, ax):
    """Control-volume face (2D: length, 3D: area) crossed by axis-`ax`
    edges, as an array broadcastable over the node grid.  2D x-edges use
    dVy, y-edges dVx (device2d.py:1563-1578); 3D x-edges dVy*dVz, y-edges
    dVx*dVz, z-edges dVx*dVy (device3d.py:1639-1641)."""
    if dim == 2:
        return dv[1][:, None] if ax == 0 else dv[0][None, :]
    if ax == 0:
        return dv[1][None, :, None] * dv[2][:, None, None]
    if ax == 1:
        return dv[0][None, None, :] * dv[2][:, None, None]
    return dv[0][None, None, :] * dv[1][None, :, None]


class OracleDevice:
    """Device2D / Device3D state and equations on a tensor-product mesh.

    ``coords`` = (x, y) or (x, y, z) in cm.  Node arrays are shaped
    (Ny, Nx) or (Nz, Ny, Nx); node k = j*Nx + i (+ kz*Nx*Ny), x fastest
    (mesh2d.py:1-7, mesh3d.py:1-10).  Axis index 0 = x, 1 = y, 2 = z.
    """

    def __init__(self, coords, doping, Ntotal=None, T=300.0, models=None,
                 material=None):
        self.dim = len(coords)
        self.coords = [np.asarray(c, dtype=float) for c in coords]
        self.Nax = [c.size for c in self.coords]            # Nx, Ny(, Nz)
        self.shape = tuple(reversed(self.Nax))
        self.N = int(np.prod(self.Nax))
        self.doping = np.asarray(doping, dtype=float).reshape(self.shape)
        self.Ntot = (np.abs(self.doping) if Ntotal is None else
                     np.asarray(Ntotal, dtype=float).reshape(self.shape))
        self.T = T
        self.mat = dict(SILICON_PARAMS if material is None else material)
        self.models = models or OracleModels()
        m = self.mat
        # device2d.py:319-347, device3d.py:576-606: scaling
        self.VT = KB * T / Q
        self.eps = m["eps_r"] * EPS0
        self.ni = _ni(m, T)
        self.Ns = max(float(np.abs(self.doping).max()), self.ni)
        self.LD = np.sqrt(self.eps * self.VT / (Q * self.Ns))
        self.J0 = Q * D0_REF * self.Ns / self.LD
        self.R0 = D0_REF * self.Ns / self.LD ** 2
        self.h = [np.diff(c / self.LD) for c in self.coords]
        self.dv = [control_volume_widths(h) for h in self.h]
        if self.dim == 2:
            self.dV = np.outer(self.dv[1], self.dv[0])
        else:
            self.dV = (self.dv[2][:, None, None] * self.dv[1][None, :, None]
                       * self.dv[0][None, None, :])
        self.C = self.doping / self.Ns
        # device2d.py:361-407: per-node coefficients (single material)
        nt = self.Ntot
        self.nie = _nie(nt, m, T, self.models.bgn)
        self.nie_s = self.nie / self.Ns
        if self.models.doping_mobility:
            mu_n = _mobility(nt, m, T, "n")
            mu_p = _mobility(nt, m, T, "p")
        else:
            mu_n = np.full(self.shape, m["mu_n_max"])
            mu_p = np.full(self.shape, m["mu_p_max"])
        self.tau_n = _lifetime(nt, m["tau_n0"], m["tau_Nref"])
        self.tau_p = _lifetime(nt, m["tau_p0"], m["tau_Nref"])
        # device2d.py:442-450, device3d.py:696-706: harmonic-mean edge D
        self.an, self.ap, self.dlnnie = [], [], []
        for ax in range(self.dim):
            lo, hi = self._lo(ax), self._hi(ax)
            dn = 2.0 * mu_n[lo] * mu_n[hi] / (mu_n[lo] + mu_n[hi]) * self.VT / D0_REF
            dp = 2.0 * mu_p[lo] * mu_p[hi] / (mu_p[lo] + mu_p[hi]) * self.VT / D0_REF
            hb = self._axis_bcast(self.h[ax], ax)
            self.an.append(dn / hb)
            self.ap.append(dp / hb)
            self.dlnnie.append(np.log(self.nie_s[hi] / self.nie_s[lo]))
        self.contacts = {}     # name -> [flat node idx, V]
        self.gates = {}        # name -> [flat node idx, kappa, Vfb, Vg, w]
        self.psi = self.n = self.p = None

    # -- index helpers -------------------------------------------------------
    def _arr_axis(self, ax):
        return self.dim - 1 - ax

    def _lo(self, ax):
        s = [slice(None)] * self.dim
        s[self._arr_axis(ax)] = slice(None, -1)
        return tuple(s)

    def _hi(self, ax):
        s = [slice(None)] * self.dim
        s[self._arr_axis(ax)] = slice(1, None)
        return tuple(s)

    def _axis_bcast(self, v, ax):
        shp = [1] * self.dim
        shp[self._arr_axis(ax)] = v.size
        return v.reshape(shp)

    def _edge_nodes(self, ax):
        """Flat (low, high) node pairs of every axis-`ax` edge, in C order of
        the edge grid (device2d.py:107-120, device3d.py:166-187)."""
        k = np.arange(self.N).reshape(self.shape)
        return k[self._lo(ax)].ravel(), k[self._hi(ax)].ravel()

    def flat(self, *ijk):
        i = np.atleast_1d(np.asarray(ijk[0], dtype=np.int64))
        out = i.copy()
        stride = 1
        for a in range(1, self.dim):
            stride *= self.Nax[a - 1]
            out = out + np.atleast_1d(np.asarray(ijk[a], dtype=np.int64)) * stride
        return out

    # -- boundary conditions ---------------------------------------------------
    def add_contact(self, name, *ijk, V=0.0):
        """device2d.py:672-674, device3d.py:748-750."""
        self.contacts[name] = [self.flat(*ijk), float(V)]

    def add_gate(self, name, *ijk, tox_cm, Vfb, Vg=0.0, normal_axis="y"):
        """Oxide Robin BC.  kappa = eps_ox LD / (eps t_ox); the face weight is
        dVx (2D, device2d.py:676-680,1624-1637) or the face area normal to
        `normal_axis` (3D, device3d.py:752-756, 939-947)."""
        kappa = EPS_OX_R * EPS0 * self.LD / (self.eps * tox_cm)
        idx = [np.atleast_1d(np.asarray(a, dtype=np.int64)) for a in ijk]
        dv = self.dv
        if self.dim == 2:
            w = dv[0][idx[0]]
        elif normal_axis == "z":
            w = dv[0][idx[0]] * dv[1][idx[1]]
        elif normal_axis == "y":
            w = dv[0][idx[0]] * dv[2][idx[2]]
        else:
            w = dv[1][idx[1]] * dv[2][idx[2]]
        self.gates[name] = [self.flat(*ijk), kappa, float(Vfb), float(Vg), w]

    def contact_values(self, name, V):
        k = self.contacts[name][0]
        return ohmic_values(self.C.ravel()[k], self.nie_s.ravel()[k], V,
                            self.VT)

    def bulk_guess(self):
        """device2d.py:744-759."""
        return np.arcsinh(self.C / (2.0 * self.nie_s))

    def _gate_rhs(self, name, psi_flat, equilibrium):
        k, kappa, Vfb, Vg, w = self.gates[name]
        Vg_s = 0.0 if equilibrium else Vg / self.VT
        psi_b = np.arcsinh(self.C.ravel()[k] / (2.0 * self.nie_s.ravel()[k]))
        return k, kappa * w * (Vg_s - Vfb / self.VT - (psi_flat[k] - psi_b)), -kappa * w

    # -- equilibrium Poisson (device2d.py:844-942, device3d.py:190-258,952-1020)
    def residual_jacobian_poisson(self, psi):
        psi = np.asarray(psi, dtype=float).reshape(self.shape)
        n = self.nie_s * np.exp(np.clip(psi, -700, 700))
        p = self.nie_s * np.exp(np.clip(-psi, -700, 700))
        dnp = n + p
        F = None
        rows, cols, vals = [], [], []
        for ax in range(self.dim):
            lo, hi = self._lo(ax), self._hi(ax)
            hb = self._axis_bcast(self.h[ax], ax)
            flux = (psi[hi] - psi[lo]) / hb
            div = np.zeros(self.shape)
            div[lo] += flux
            div[hi] -= flux
            face = _face(self.dv, self.dim, ax)
            term = face * div
            F = term if F is None else F + term
            kL, kR = self._edge_nodes(ax)
            w = np.broadcast_to(face / hb, flux.shape).ravel()
            rows += [kL, kR, kL, kR]
            cols += [kL, kR, kR, kL]
            vals += [-w, -w, w, w]
        F = F - self.dV * (n - p - self.C)
        kd = np.arange(self.N)
        rows.append(kd); cols.append(kd); vals.append((-self.dV * dnp).ravel())
        Ff = F.ravel()
        for name in self.gates:
            k, add, jv = self._gate_rhs(name, psi.ravel(), equilibrium=True)
            Ff[k] += add
            rows.append(k); cols.append(k); vals.append(jv)
        fixed = []
        for name, (k, _V) in self.contacts.items():
            psi0 = self.contact_values(name, 0.0)[0]
            Ff[k] = psi.ravel()[k] - psi0
            fixed.append(k)
        rows = np.concatenate(rows); cols = np.concatenate(cols)
        vals = np.concatenate(vals)
        if fixed:
            fixed = np.unique(np.concatenate(fixed))
            keep = ~np.isin(rows, fixed)
            rows = np.concatenate([rows[keep], fixed])
            cols = np.concatenate([cols[keep], fixed])
            vals = np.concatenate([vals[keep], np.ones(fixed.size)])
        else:
            fixed = np.zeros(0, dtype=np.int64)
        J = sp.csr_matrix((vals, (rows, cols)), shape=(self.N, self.N))
        self.fixed_poisson = fixed
        return Ff.reshape(self.shape), J

    def solve_equilibrium(self, max_iter=100, tol=1e-8, max_dpsi=5.0):
        """device2d.py:1308-1373 / device3d.py:1311-1454 (direct solve)."""
        psi = self.bulk_guess()
        self.eq_iters = 0
        for it in range(max_iter):
            F, J = self.residual_jacobian_poisson(psi)
            Jd, rhs = eliminate_csr(J, -F.ravel(), self.fixed_poisson)
            d = spsolve(Jd.tocsc(), rhs).reshape(self.shape)
            d = np.clip(d, -max_dpsi, max_dpsi)
            psi = psi + d
            self.eq_iters = it + 1
            if np.abs(d).max() < tol:
                break
        else:
            warnings.warn("oracle equilibrium did not converge")
        self.psi = psi
        self.n = self.nie_s * np.exp(np.clip(psi, -700, 700))
        self.p = self.nie_s * np.exp(np.clip(-psi, -700, 700))
        return self

    # -- coupled system (device2d.py:1402-1920, device3d.py:1485-1978) -------
    def residual_jacobian(self, psi, n, p, voltages=None):
        """Returns (F interleaved [3N], J csr, F_n, F_p) and sets
        ``self.fixed``; F_n/F_p are the raw continuity residuals used for
        terminal currents."""
        voltages = voltages or {}
        sh = self.shape
        psi = np.asarray(psi, dtype=float).reshape(sh)
        n = np.asarray(n, dtype=float).reshape(sh)
        p = np.asarray(p, dtype=float).reshape(sh)
        edges = []
        for ax in range(self.dim):
            lo, hi = self._lo(ax), self._hi(ax)
            dpsi = psi[hi] - psi[lo]
            de = dpsi + self.dlnnie[ax]          # electron SG argument
            dh = dpsi - self.dlnnie[ax]          # hole SG argument
            Bp, Bm = bernoulli(de), bernoulli(-de)
            dBp, dBm = dbernoulli(de), dbernoulli(-de)
            Bph, Bmh = bernoulli(dh), bernoulli(-dh)
            dBph, dBmh = dbernoulli(dh), dbernoulli(-dh)
            an, ap = self.an[ax], self.ap[ax]
            Jn = an * (n[hi] * Bp - n[lo] * Bm)
            Jp = -ap * (p[hi] * Bmh - p[lo] * Bph)
            Sn = n[hi] * dBp + n[lo] * dBm
            Sp = p[hi] * dBmh + p[lo] * dBph
            edges.append(dict(
                dpsi=dpsi, Jn=Jn, Jp=Jp,
                n_psi=an * Sn, n_lo=-an * Bm, n_hi=an * Bp,
                p_psi=ap * Sp, p_lo=ap * Bph, p_hi=-ap * Bmh))
        # recombination in physical units, scaled by R0 (device2d.py:1482-1508)
        m = self.mat
        R, dRdn, dRdp = recombination(n * self.Ns, p * self.Ns, self.nie,
                                      self.tau_n, self.tau_p, m["Cn_auger"],
                                      m["Cp_auger"], auger=self.models.auger)
        if not self.models.srh:
            R = np.zeros_like(R); dRdn = np.zeros_like(R); dRdp = np.zeros_like(R)
        Rs = R / self.R0
        dRs_dn = dRdn * self.Ns / self.R0
        dRs_dp = dRdp * self.Ns / self.R0

        def divergence(key):
            tot = None
            for ax in range(self.dim):
                lo, hi = self._lo(ax), self._hi(ax)
                f = edges[ax][key]
                if key == "dpsi":
                    f = f / self._axis_bcast(self.h[ax], ax)
                d = np.zeros(sh)
                d[lo] += f
                d[hi] -= f
                t = _face(self.dv, self.dim, ax) * d
                tot = t if tot is None else tot + t
            return tot
        F_psi = divergence("dpsi") - self.dV * (n - p - self.C)
        F_n = divergence("Jn") - Rs * self.dV
        F_p = divergence("Jp") + Rs * self.dV
        F = np.empty((self.N, 3))
        F[:, 0] = F_psi.ravel(); F[:, 1] = F_n.ravel(); F[:, 2] = F_p.ravel()
        F = F.ravel()

        rows, cols, vals = [], [], []

        def stamp(kL, kR, w, rc, cL, dL, cR, dR):
            # one edge's derivative into both endpoint rows (+ near, - far)
            w = np.asarray(w).ravel(); dL = np.asarray(dL).ravel()
            dR = np.asarray(dR).ravel()
            rows.extend([3 * kL + rc, 3 * kL + rc, 3 * kR + rc, 3 * kR + rc])
            cols.extend([3 * kL + cL, 3 * kR + cR, 3 * kL + cL, 3 * kR + cR])
            vals.extend([w * dL, w * dR, -w * dL, -w * dR])

        kk = [self._edge_nodes(ax) for ax in range(self.dim)]
        fshape = [edges[ax]["Jn"].shape for ax in range(self.dim)]
        faces = [np.broadcast_to(_face(self.dv, self.dim, ax), fshape[ax])
                 for ax in range(self.dim)]
        for ax in range(self.dim):          # Poisson row
            w = faces[ax] / self._axis_bcast(self.h[ax], ax)
            one = np.ones(fshape[ax])
            stamp(kk[ax][0], kk[ax][1], w, 0, 0, -one, 0, one)
        for ax in range(self.dim):          # electron continuity row
            e = edges[ax]
            stamp(kk[ax][0], kk[ax][1], faces[ax], 1, 0, -e["n_psi"], 0, e["n_psi"])
            stamp(kk[ax][0], kk[ax][1], faces[ax], 1, 1, e["n_lo"], 1, e["n_hi"])
        for ax in range(self.dim):          # hole continuity row
            e = edges[ax]
            stamp(kk[ax][0], kk[ax][1], faces[ax], 2, 0, -e["p_psi"], 0, e["p_psi"])
            stamp(kk[ax][0], kk[ax][1], faces[ax], 2, 2, e["p_lo"], 2, e["p_hi"])
        kd = np.arange(self.N)
        dVf = self.dV.ravel()
        for r, c, v in ((0, 1, -dVf), (0, 2, dVf),
                        (1, 1, -dRs_dn.ravel() * dVf),
                        (1, 2, -dRs_dp.ravel() * dVf),
                        (2, 2, dRs_dp.ravel() * dVf),
                        (2, 1, dRs_dn.ravel() * dVf)):
            rows.append(3 * kd + r); cols.append(3 * kd + c); vals.append(v)
        F3 = F.reshape(self.N, 3)
        psif = psi.ravel()
        for name in self.gates:
            k, add, jv = self._gate_rhs(name, psif, equilibrium=False)
            F3[k, 0] += add
            rows.append(3 * k); cols.append(3 * k); vals.append(jv)
        rows = np.concatenate(rows); cols = np.concatenate(cols)
        vals = np.concatenate(vals)
        fixed = []
        for name, (k, V0) in self.contacts.items():
            V = voltages.get(name, V0)
            psi0, n0, p0 = self.contact_values(name, V)
            F3[k, 0] = psif[k] - psi0
            F3[k, 1] = n.ravel()[k] - n0
            F3[k, 2] = p.ravel()[k] - p0
            fixed += [3 * k, 3 * k + 1, 3 * k + 2]
        if fixed:
            fixed = np.unique(np.concatenate(fixed))
            keep = ~np.isin(rows, fixed)
            rows = np.concatenate([rows[keep], fixed])
            cols = np.concatenate([cols[keep], fixed])
            vals = np.concatenate([vals[keep], np.ones(fixed.size)])
        else:
            fixed = np.zeros(0, dtype=np.int64)
        self.fixed = fixed
        J = sp.csr_matrix((vals, (rows, cols)), shape=(3 * self.N, 3 * self.N))
        return F3.ravel(), J, F_n, F_p

    def solve_bias(self, voltages=None, max_iter=100, tol=1e-8, max_dpsi=5.0,
                   linsolve="direct", rtol=1e-10):
        """device2d.py:1923-2191 / device3d.py:1981-2271, plain path.
        ``linsolve``: "direct" (SuperLU) or "bicgstab"/"gmres" with node
        block-Jacobi and the per-iteration direct fallback of
        device3d.py:2146-2168."""
        if self.psi is None:
            self.solve_equilibrium()
        for name, V in (voltages or {}).items():
            if name in self.contacts:
                self.contacts[name][1] = float(V)
            else:
                self.gates[name][3] = float(V)
        sh = self.shape
        psi, n, p = self.psi.copy(), self.n.copy(), self.p.copy()
        for name, (k, V) in self.contacts.items():
            psi0, n0, p0 = self.contact_values(name, V)
            psi.ravel()[k] = psi0; n.ravel()[k] = n0; p.ravel()[k] = p0
        cur = {name: V for name, (k, V) in self.contacts.items()}
        self.krylov_iters = []
        converged = False
        err = np.inf
        for it in range(max_iter):
            F, J, _, _ = self.residual_jacobian(psi, n, p, cur)
            Jd, rhs = eliminate_csr(J, -F, self.fixed)
            du = None
            if linsolve != "direct":
                x, its, ok, _ = solve_linear_iterative(
                    Jd, rhs, method=linsolve, rtol=rtol)
                self.krylov_iters.append(its)
                if ok:
                    du = x
            if du is None:
                du = spsolve(Jd.tocsc(), rhs)
            dpsi = np.clip(du[0::3].reshape(sh), -max_dpsi, max_dpsi)
            n_new = np.clip(n + du[1::3].reshape(sh), 0.1 * n, 10.0 * n)
            p_new = np.clip(p + du[2::3].reshape(sh), 0.1 * p, 10.0 * p)
            rel_n = (np.abs(n_new - n) / np.maximum(n, 1e-10)).max()
            rel_p = (np.abs(p_new - p) / np.maximum(p, 1e-10)).max()
            err = max(np.abs(dpsi).max(), rel_n, rel_p)
            psi = psi + dpsi
            n, p = n_new, p_new
            if err < tol:
                converged = True
                break
        if not converged:
            warnings.warn(f"oracle Newton did not converge; last update {err:.2e}")
        self.newton_iters = it + 1
        self.last_converged = converged
        self.psi, self.n, self.p = psi, n, p
        return self

    # -- transient: theta scheme (transient2d.py:94-330, transient3d.py:108-380)
    def _free_nodes(self):
        mask = np.zeros(self.N, dtype=bool)
        for k, _ in self.contacts.values():
            mask[np.asarray(k)] = True
        return np.arange(self.N)[~mask]

    def _step_residual_jacobian(self, psi, n, p, volts, n_old, p_old, Fn_old, Fp_old,
                                dt_s, theta, k_free):
        """transient2d.py:104-135: the storage term on the non-contact
        continuity rows, theta-weighted with the previous time's residual."""
        F_new, J_new, _, _ = self.residual_jacobian(psi, n, p, volts)
        F = F_new.copy()
        idx_n = 3 * k_free + 1
        idx_p = 3 * k_free + 2
        dVi = self.dV.ravel()[k_free]
        nf, pf = np.asarray(n).ravel()[k_free], np.asarray(p).ravel()[k_free]
        n0f, p0f = np.asarray(n_old).ravel()[k_free], np.asarray(p_old).ravel()[k_free]
        if theta != 1.0:
            F[idx_n] = theta * F[idx_n] + (1.0 - theta) * Fn_old.ravel()[k_free]
            F[idx_p] = theta * F[idx_p] + (1.0 - theta) * Fp_old.ravel()[k_free]
            row_scale = np.ones(F.shape[0])
            row_scale[idx_n] = theta
            row_scale[idx_p] = theta
            J = sp.diags(row_scale) @ J_new
        else:
            J = J_new
        F[idx_n] -= dVi / dt_s * (nf - n0f)
        F[idx_p] += dVi / dt_s * (pf - p0f)
        rows = np.concatenate([idx_n, idx_p])
        vals = np.concatenate([-dVi / dt_s, dVi / dt_s])
        J = J + sp.csr_matrix((vals, (rows, rows)), shape=J.shape)
        return F, J

    def _transient_newton(self, psi0, n0, p0, volts, Fn_old, Fp_old, dt_s, theta, k_free,
                          max_iter, tol, max_dpsi):
        """transient2d.py:138-183: Newton with exact (direct) steps and a
        backtracking line search on 0.5 |F|^2, densities clipped to
        [0.1, 10] x per step, stopped on the update test."""
        sh = self.shape
        psi, n, p = psi0.copy(), n0.copy(), p0.copy()
        args = (volts, n0, p0, Fn_old, Fp_old, dt_s, theta, k_free)
        for it in range(max_iter):
            F, J = self._step_residual_jacobian(psi, n, p, *args)
            du = spsolve(J.tocsc(), -F)
            dpsi = np.clip(du[0::3].reshape(sh), -max_dpsi, max_dpsi)
            dn = du[1::3].reshape(sh)
            dp = du[2::3].reshape(sh)
            base = 0.5 * float(np.dot(F, F))
            lam = 1.0
            for _ in range(40):
                psi_t = psi + lam * dpsi
                n_t = np.clip(n + lam * dn, 0.1 * n, 10.0 * n)
                p_t = np.clip(p + lam * dp, 0.1 * p, 10.0 * p)
                Ft, _ = self._step_residual_jacobian(psi_t, n_t, p_t, *args)
                merit = 0.5 * float(np.dot(Ft, Ft))
                if np.isfinite(merit) and merit <= base * (1.0 - 1e-4 * lam):
                    break
                lam *= 0.5
            else:
                lam = 0.0
            n_prev, p_prev = n, p
            psi = psi + lam * dpsi
            n = np.clip(n + lam * dn, 0.1 * n, 10.0 * n)
            p = np.clip(p + lam * dp, 0.1 * p, 10.0 * p)
            rel_n = (np.abs(n - n_prev) / np.maximum(n_prev, 1e-10)).max()
            rel_p = (np.abs(p - p_prev) / np.maximum(p_prev, 1e-10)).max()
            err = max(float(np.abs(dpsi).max()), float(rel_n), float(rel_p))
            if err < tol:
                return psi, n, p, True, it + 1
        return psi, n, p, False, max_iter

    def _current_at(self, psi, n, p, name):
        k, _ = self.contacts[name]
        cur = {nm: V for nm, (kk, V) in self.contacts.items()}
        *_, F_n, F_p = self.residual_jacobian(psi, n, p, cur)
        scale = self.J0 * self.LD if self.dim == 2 else self.J0 * self.LD ** 2
        return float((F_n.ravel()[k] + F_p.ravel()[k]).sum()) * scale

    def solve_transient(self, waveforms, t_end, dt0, theta=1.0, max_iter=100, tol=1e-8,
                        max_dpsi=5.0, dt_min=None, dt_max=None, growth=1.5, shrink=0.5):
        """transient2d.py:186-330 / transient3d.py:234-380 from the current
        state: waveforms {contact: object with .value(t), function of t, or
        volts}.  Returns
        {"times", "currents": {contact: [...]}} and leaves the final state."""
        def wv(w, t):   # a waveform object, a function of t, or a constant
            return w.value(t) if hasattr(w, "value") else (w(t) if callable(w) else float(w))
        names = list(self.contacts)

        def volts_at(t):
            return {nm: (wv(waveforms[nm], t) if nm in waveforms else self.contacts[nm][1])
                    for nm in names}

        k_free = self._free_nodes()
        t0 = self.Ns / self.R0
        dt_s = dt0 / t0
        dt_min_s = (dt_min if dt_min is not None else dt0 / 1024.0) / t0
        dt_max_s = (dt_max if dt_max is not None else dt0 * 64.0) / t0
        t = 0.0
        psi, n, p = self.psi.copy(), self.n.copy(), self.p.copy()
        times = [t]
        currents = {nm: [self._current_at(psi, n, p, nm)] for nm in names}
        while t < t_end - 1e-15:
            step_dt_s = dt_s
            t_new = t + step_dt_s * t0
            if t_new > t_end:
                t_new = t_end
                step_dt_s = (t_new - t) / t0
            volts = volts_at(t_new)
            Fn_old = Fp_old = None
            if theta != 1.0:
                *_, Fn_old, Fp_old = self.residual_jacobian(psi, n, p, volts_at(t))
            for nm, V in volts.items():
                self.contacts[nm][1] = float(V)
            psi_n, n_n, p_n, ok, iters = self._transient_newton(
                psi, n, p, volts, Fn_old, Fp_old, step_dt_s, theta, k_free, max_iter, tol,
                max_dpsi)
            if ok:
                t = t_new
                psi, n, p = psi_n, n_n, p_n
                times.append(t)
                for nm in names:
                    currents[nm].append(self._current_at(psi, n, p, nm))
                dt_s = min(step_dt_s * growth, dt_max_s) \
                    if iters <= max(3, max_iter // 4) else step_dt_s
            else:
                dt_s = step_dt_s * shrink
                if dt_s < dt_min_s:
                    raise RuntimeError(f"oracle transient stalled at t={t:.3e}s")
        self.psi, self.n, self.p = psi, n, p
        return {"times": np.array(times), "currents": {k: np.array(v) for k, v in currents.items()}}

    def terminal_current(self, name):
        """device2d.py:2194-2227 (A/cm) / device3d.py:2274-2306 (A)."""
        k, _ = self.contacts[name]
        cur = {nm: V for nm, (kk, V) in self.contacts.items()}
        *_, F_n, F_p = self.residual_jacobian(self.psi, self.n, self.p, cur)
        scale = self.J0 * self.LD if self.dim == 2 else self.J0 * self.LD ** 2
        return float((F_n.ravel()[k] + F_p.ravel()[k]).sum()) * scale
