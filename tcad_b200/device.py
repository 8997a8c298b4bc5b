"""Device2D / Device3D: the reference's device API on the GPU path.

Constructor, ``add_contact``, ``add_gate``, ``solve_equilibrium``,
``solve_bias``, ``terminal_current``, ``_residual_jacobian``,
``_residual_jacobian_poisson`` and the ``psi/n/p``, ``psi_V/n_cm3/p_cm3``,
``Jn_*/Jp_*``, ``last_converged`` attributes keep the signatures, units and
shapes of pytcad/device2d.py and pytcad/device3d.py.  The state lives in HBM
(``psi_gpu``...); the numpy attributes are copies made on access.

Differences that are by design: the Newton linear systems are solved by the
GPU's block-scaled BiCGStab whatever ``NewtonOptions.linsolve`` says (there is
no direct solver on this path), and the Krylov budget per Newton step is
``NewtonOptions.linsolve_maxiter``.  Converged states agree with the
reference to its own Newton tolerance, not bit for bit.
"""
from __future__ import annotations

import warnings

import numpy as np
import scipy.sparse as sp

from . import _lib
from .options import Models, NewtonOptions
from .pack import Contact, Gate, Pack, Setup, bias_vector, secant_ratio
from .physics import SILICON


class _Device:
    dim = None
    _current_len_exp = None   # J0*LD**exp converts the scaled current

    def __init__(self, mesh, doping, Ntotal=None, T=300.0, material=SILICON,
                 models=None, Ns_override=None):
        if isinstance(material, (list, tuple)):
            raise NotImplementedError("tcad_b200: per-node material lists are not on the "
                                      "GPU path")
        self.mesh = mesh
        coords = (mesh.x, mesh.y) if self.dim == 2 else (mesh.x, mesh.y, mesh.z)
        self.setup = Setup(coords, doping, Ntotal=Ntotal, T=T, material=material,
                           models=models or Models(), Ns_override=Ns_override)
        s = self.setup
        self.models = s.models
        self.mat = material
        self.T = T
        self.Nx, self.Ny = s.nax[0], s.nax[1]
        if self.dim == 3:
            self.Nz = s.nax[2]
        self.N = s.N
        for a in ("VT", "eps", "ni", "Ns", "LD", "J0", "R0", "C", "nie", "nie_s",
                  "tau_n", "tau_p", "doping", "Ntot"):
            setattr(self, a, getattr(s, a))
        self.bcs = s.bcs
        self._pack = None
        self._bias_prev = self._bias_cur = None   # biases of the prev / current state
        self._have_state = False
        self._host = {}
        self.last_converged = None
        self.last_auto_method = None
        self.last_auto_reason = None
        self.last_newton = None
        self.last_equilibrium = None

    # ---- pack / state --------------------------------------------------------
    @property
    def pack(self):
        if self._pack is None:
            self._pack = Pack([self.setup])
        return self._pack

    def _bcs_changed(self):
        if self._pack is not None:
            self._pack.refresh_bcs()

    def _to_dev(self, a):
        import torch
        a = np.ascontiguousarray(np.asarray(a, dtype=float).reshape(-1))
        if a.size != self.N:
            raise ValueError(f"state array has {a.size} entries, expected {self.N}")
        return torch.from_numpy(a).to(self.pack.device)

    def _get(self, name):
        if not self._have_state:
            return None
        if name not in self._host:
            t = getattr(self.pack, name)
            self._host[name] = t.cpu().numpy().reshape(self.setup.shape).copy()
        return self._host[name]

    def _set(self, name, value):
        self._bias_prev = self._bias_cur = None
        if value is None:
            self._have_state = False
            self._host.clear()
            return
        getattr(self.pack, name).copy_(self._to_dev(value))
        self._host.pop(name, None)
        self._have_state = True

    psi = property(lambda self: self._get("psi"), lambda self, v: self._set("psi", v))
    n = property(lambda self: self._get("n"), lambda self, v: self._set("n", v))
    p = property(lambda self: self._get("p"), lambda self, v: self._set("p", v))

    @property
    def psi_gpu(self):
        return self.pack.psi

    @property
    def n_gpu(self):
        return self.pack.n

    @property
    def p_gpu(self):
        return self.pack.p

    @property
    def psi_V(self):
        return self.psi * self.VT

    @property
    def n_cm3(self):
        return self.n * self.Ns

    @property
    def p_cm3(self):
        return self.p * self.Ns

    # ---- boundary conditions --------------------------------------------------
    def _add_contact(self, name, *ijk, V=0.0):
        self.bcs[name] = Contact(self.setup.flat(*ijk), V)
        self._bcs_changed()
        return self.bcs[name]

    def _add_gate(self, name, ijk, tox_cm, Vfb, Vg, normal_axis):
        s = self.setup
        idx = [np.atleast_1d(np.asarray(a, dtype=np.int64)) for a in ijk]
        w = s.gate_weight(idx, normal_axis)
        self.bcs[name] = Gate(s.flat(*ijk), s.gate_kappa(tox_cm), Vfb, Vg, w, normal_axis)
        self._bcs_changed()
        return self.bcs[name]

    def _apply_voltages(self, voltages):
        for name, V in (voltages or {}).items():
            b = self.bcs[name]
            if b.kind == "contact":
                b.V = float(V)
            else:
                b.Vg = float(V)

    # ---- solves -------------------------------------------------------------
    def solve_equilibrium(self, opts: NewtonOptions = None, psi_guess=None):
        """Poisson-only Newton with slaved densities on the GPU
        (pytcad/device2d.py:1308-1373, pytcad/device3d.py:1311-1454)."""
        opts = opts or NewtonOptions()
        pk = self.pack
        guess = self.setup.bulk_guess() if psi_guess is None else np.asarray(psi_guess)
        pk.psi.copy_(self._to_dev(guess))
        res = pk.equilibrium(opts)[0]
        self.last_equilibrium = res
        self._have_state = True
        self._host.clear()
        # the equilibrium state is the state at zero applied bias
        self._bias_prev, self._bias_cur = None, np.zeros(len(self.bcs))
        if not res["converged"]:
            warnings.warn(f"{self.dim}D equilibrium Poisson solve did not converge "
                          f"(last |d| {res['err']:.2e}, linear status "
                          f"{_lib.STATUS_NAMES.get(res['status'])}).")
        return self

    def solve_bias(self, voltages=None, opts: NewtonOptions = None):
        """Coupled Newton at applied bias, warm-started from the current state
        (pytcad/device2d.py:1923-2191, pytcad/device3d.py:1981-2271)."""
        opts = opts or NewtonOptions()
        if not self._have_state:
            self.solve_equilibrium(opts)
        self._apply_voltages(voltages)
        pk = self.pack
        pk.set_bias()
        new = bias_vector(self.setup)
        use_pred = getattr(opts, "predictor", "none") == "secant"
        ratio = secant_ratio(self._bias_prev, self._bias_cur, new) if use_pred else 0.0
        if use_pred:
            pk.predict([ratio])
        pk.stamp_contacts()
        self.last_auto_method = "bicgstab" if opts.linsolve == "auto" else None
        self.last_auto_reason = ("GPU path: node-block-scaled BiCGStab for every coupled "
                                 "Newton system" if opts.linsolve == "auto" else None)
        res = pk.newton(opts)[0]
        res["predictor_ratio"] = ratio
        if ratio != 0.0 and not res["converged"]:
            # the predicted start did not converge: solve again from the
            # previous converged state
            pk.restore_prev()
            pk.stamp_contacts()
            first = res
            res = pk.newton(opts)[0]
            res["iters"] += first["iters"]
            res["krylov_iters"] += first["krylov_iters"]
            res["predictor_ratio"] = 0.0
            res["predictor_retry"] = True
        if use_pred:
            self._bias_prev = self._bias_cur
        else:
            self._bias_prev = None
        self._bias_cur = new if res["converged"] else None
        self._host.clear()
        self.last_newton = res
        self.last_converged = bool(res["converged"])
        if not self.last_converged:
            warnings.warn(f"{self.dim}D Newton did not converge; last update "
                          f"{res['err']:.2e} (linear status "
                          f"{_lib.STATUS_NAMES.get(res['status'])}, relres "
                          f"{res['relres']:.1e})")
        return self

    def save_state(self):
        """A copy of the solution state (the GPU psi/n/p and the sweep history
        the predictor uses), for restore_state."""
        pk = self.pack
        return dict(psi=pk.psi.clone(), n=pk.n.clone(), p=pk.p.clone(),
                    have=self._have_state, prev=self._bias_prev, cur=self._bias_cur)

    def restore_state(self, st):
        """Put back a state taken by save_state (e.g. the last converged one
        after a failed solve, which leaves its diverged iterate behind)."""
        pk = self.pack
        pk.psi.copy_(st["psi"])
        pk.n.copy_(st["n"])
        pk.p.copy_(st["p"])
        self._have_state = st["have"]
        self._bias_prev, self._bias_cur = st["prev"], st["cur"]
        self._host.clear()

    def terminal_current(self, name):
        """Total current into a contact from the raw continuity residual at its
        nodes: A/cm (2D) or A (3D) (pytcad/device2d.py:2194-2227,
        pytcad/device3d.py:2274-2306)."""
        b = self.bcs[name]
        if b.kind != "contact":
            raise ValueError(f"terminal_current: '{name}' is not a Dirichlet contact")
        if not self._have_state:
            raise RuntimeError("terminal_current: solve the device first")
        I = float(self.pack.contact_current(0, name).item())
        return I * self.J0 * self.LD ** self._current_len_exp

    # ---- edge current densities (computed on access) -------------------------
    def _edge(self, axis, which):
        if not self._have_state:
            return None
        key = f"J{which}{axis}"
        if key not in self._host:
            Jn, Jp = self.pack.edge_currents(axis)
            s = self.setup
            for w, t in (("n", Jn), ("p", Jp)):
                a = t.cpu().numpy().reshape(s.shape)[s.lo(axis)] * self.J0
                self._host[f"J{w}{axis}"] = a.copy()
        return self._host[key]

    Jn_x = property(lambda self: self._edge(0, "n"))
    Jp_x = property(lambda self: self._edge(0, "p"))
    Jn_y = property(lambda self: self._edge(1, "n"))
    Jp_y = property(lambda self: self._edge(1, "p"))

    # ---- the reference's assembly entry points ----------------------------------
    def _block_to_csr(self, Jflat, nfield):
        """Node-block layout -> scipy CSR with the reference's interleaved
        (3k + c) numbering (pytcad/device2d.py:1529)."""
        s = self.setup
        N = self.N
        k = np.arange(N)
        rows, cols, vals = [], [], []
        J = Jflat.reshape(-1, N)
        if nfield == 1:       # equilibrium Poisson: diag, W,E,S,N,D,U
            rows.append(k); cols.append(k); vals.append(J[0])
            for d in range(2 * self.dim):
                m, ok = self._nbr(d)
                rows.append(k[ok]); cols.append(m[ok]); vals.append(J[1 + d][ok])
            return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows),
                                  np.concatenate(cols))), shape=(N, N))
        for r in range(3):
            for c in range(3):
                rows.append(3 * k + r); cols.append(3 * k + c); vals.append(J[3 * r + c])
        rc_pairs = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 2)]
        for d in range(2 * self.dim):
            m, ok = self._nbr(d)
            for q, (r, c) in enumerate(rc_pairs):
                rows.append(3 * k[ok] + r); cols.append(3 * m[ok] + c)
                vals.append(J[9 + 5 * d + q][ok])
        return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows),
                              np.concatenate(cols))), shape=(3 * N, 3 * N))

    def _nbr(self, d):
        s = self.setup
        coord = np.indices(s.shape).reshape(s.dim, -1)[::-1]   # x, y(, z) per node
        ax, sgn = d // 2, (-1 if d % 2 == 0 else 1)
        stride = int(np.prod(s.nax[:ax])) if ax else 1
        ok = (coord[ax] + sgn >= 0) & (coord[ax] + sgn < s.nax[ax])
        return np.arange(self.N) + sgn * stride, ok

    def _residual_jacobian_poisson(self, psi):
        """Equilibrium Poisson (F (shape), J csr); sets
        ``_dirichlet_rows_poisson`` (pytcad/device2d.py:844-942)."""
        import torch
        pk = self.pack
        F = torch.empty(self.N, dtype=torch.float64, device=pk.device)
        J = torch.empty((1 + 2 * self.dim) * self.N, dtype=torch.float64, device=pk.device)
        pk.assemble_poisson(_lib.MODE_RAW, psi=self._to_dev(psi), F=F, J=J)
        Jc = self._block_to_csr(J.cpu().numpy(), 1)
        self._dirichlet_rows_poisson = pk.c_nodes.cpu().numpy() - int(pk.node_off[0])
        return F.cpu().numpy().reshape(self.setup.shape), Jc

    def _residual_jacobian(self, psi, n, p, voltages, **unsupported):
        """Coupled SG residual/Jacobian on the GPU.  Returns the reference's
        tuple (F [3N interleaved], J csr, Jn_x, Jn_y[, Jn_z], Jp_x, Jp_y[, Jp_z],
        F_n, F_p) and sets ``_dirichlet_rows`` (pytcad/device2d.py:1402-1920,
        pytcad/device3d.py:1485-1978)."""
        if any(v is not None for v in unsupported.values()):
            raise NotImplementedError("tcad_b200: energy-balance / AC row capture "
                                      "arguments are not on the GPU path")
        pk = self.pack
        s = self.setup
        dpsi, dn, dp = self._to_dev(psi), self._to_dev(n), self._to_dev(p)
        pk.set_bias([dict(voltages or {})])
        pk.assemble(_lib.MODE_RAW, dpsi, dn, dp)
        F = pk.F.cpu().numpy().reshape(3, self.N)
        Fi = F.T.ravel().copy()                       # interleaved 3k + c
        J = self._block_to_csr(pk.J.cpu().numpy(), 3)
        # raw continuity residuals (contact rows before stamping)
        F_n, F_p = F[1].copy(), F[2].copy()
        cn = pk.c_nodes
        if cn.numel():
            rn, rp = pk.raw_continuity(cn, dpsi, dn, dp)
            idx = cn.cpu().numpy() - int(pk.node_off[0])
            F_n[idx] = rn.cpu().numpy()
            F_p[idx] = rp.cpu().numpy()
        cnodes = cn.cpu().numpy() - int(pk.node_off[0])
        self._dirichlet_rows = np.sort(np.concatenate([3 * cnodes, 3 * cnodes + 1,
                                                       3 * cnodes + 2]))
        cur = []
        for w in ("n", "p"):
            for a in range(self.dim):
                Jn, Jp = pk.edge_currents(a, dpsi, dn, dp)
                t = Jn if w == "n" else Jp
                cur.append(t.cpu().numpy().reshape(s.shape)[s.lo(a)].copy())
        pk.set_bias()          # restore the stored contact voltages
        return (Fi, J, *cur, F_n.reshape(s.shape), F_p.reshape(s.shape))


class Device2D(_Device):
    """2D device on a tensor-product Mesh2D (pytcad/device2d.py:138)."""
    dim = 2
    _current_len_exp = 1

    def add_contact(self, name, i, j, V=0.0):
        return self._add_contact(name, i, j, V=V)

    def add_gate(self, name, i, j, tox_cm, Vfb, Vg=0.0):
        return self._add_gate(name, (i, j), tox_cm, Vfb, Vg, None)


class Device3D(_Device):
    """3D device on a tensor-product Mesh3D (pytcad/device3d.py:414)."""
    dim = 3
    _current_len_exp = 2

    def add_contact(self, name, i, j, k, V=0.0):
        return self._add_contact(name, i, j, k, V=V)

    def add_gate(self, name, i, j, k, tox_cm, Vfb, Vg=0.0, normal_axis="z"):
        if normal_axis not in ("x", "y", "z"):
            raise ValueError(f"normal_axis must be 'x', 'y', or 'z', got {normal_axis!r}")
        return self._add_gate(name, (i, j, k), tox_cm, Vfb, Vg, normal_axis)

    Jn_z = property(lambda self: self._edge(2, "n"))
    Jp_z = property(lambda self: self._edge(2, "p"))
