"""Host set-up of one device instance and the HBM-resident pack of one or more
instances (the layout of include/tcad_b200.h).

``Setup`` is the once-per-device part of Device2D/Device3D.__init__
(pytcad/device2d.py:168-453, pytcad/device3d.py:437-724) for the plain path:
scaling, per-node coefficients and per-edge SG coefficients, evaluated in
numpy with the reference's formulas so the kernels receive bit-identical
inputs.  ``Pack`` uploads a list of set-ups back to back into device
memory and owns the state, Jacobian and Krylov workspace buffers.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .physics import (D0_REF, EPS0, EPS_OX_R, Q, SILICON, Semiconductor,
                      control_volume_widths, lifetime_scharfetter,
                      mobility_caughey_thomas, nie_effective, ohmic_values,
                      thermal_voltage)
from .options import Models


def _hmean(lo, hi):
    return 2.0 * lo * hi / (lo + hi)


class Contact:
    """Ohmic contact (pytcad/device2d.py:64-71 DirichletBC)."""
    kind = "contact"

    def __init__(self, nodes, V):
        self.nodes = np.asarray(nodes, dtype=np.int64).ravel()
        self.V = float(V)


class Gate:
    """Oxide gate, Robin on psi (pytcad/device2d.py:74-83, device3d.py:111-125)."""
    kind = "gate"

    def __init__(self, nodes, kappa, Vfb, Vg, w, normal_axis=None):
        self.nodes = np.asarray(nodes, dtype=np.int64).ravel()
        self.kappa = float(kappa)
        self.Vfb = float(Vfb)
        self.Vg = float(Vg)
        self.w = np.broadcast_to(np.asarray(w, dtype=float), self.nodes.shape).copy()
        self.normal_axis = normal_axis


class Setup:
    """Scaled geometry and coefficients of one device (host numpy)."""

    def __init__(self, coords, doping, Ntotal=None, T=300.0, material=SILICON,
                 models=None, Ns_override=None):
        self.dim = len(coords)
        self.models = models or Models()
        self.models.require_gpu_path()
        if not isinstance(material, Semiconductor):
            raise NotImplementedError(
                "tcad_b200: heterostructures (per-node material lists) are not on "
                "the GPU path; pass one Semiconductor")
        self.mat = material
        self.coords = [np.asarray(c, dtype=float) for c in coords]
        self.nax = [c.size for c in self.coords]               # Nx, Ny(, Nz)
        if min(self.nax) < 2:
            raise ValueError("every mesh axis needs at least 2 nodes")
        self.shape = tuple(reversed(self.nax))
        self.N = int(np.prod(self.nax))
        self.doping = np.asarray(doping, dtype=float).reshape(self.shape)
        self.Ntot = (np.abs(self.doping) if Ntotal is None
                     else np.asarray(Ntotal, dtype=float).reshape(self.shape))
        self.T = T
        mat = material
        # scaling (pytcad/device2d.py:319-347)
        self.VT = thermal_voltage(T)
        self.eps = mat.eps_r * EPS0
        self.ni = mat.ni(T)
        self.Ns = (max(float(np.abs(self.doping).max()), self.ni)
                   if Ns_override is None else float(Ns_override))
        self.LD = np.sqrt(self.eps * self.VT / (Q * self.Ns))
        self.J0 = Q * D0_REF * self.Ns / self.LD
        self.R0 = D0_REF * self.Ns / self.LD ** 2
        self.h = [np.diff(c / self.LD) for c in self.coords]
        self.dv = [control_volume_widths(h) for h in self.h]
        self.C = self.doping / self.Ns
        # per-node coefficients (pytcad/device2d.py:361-407)
        nt = self.Ntot
        self.nie = nie_effective(nt, mat, T, self.models.bgn)
        self.nie_s = self.nie / self.Ns
        if self.models.doping_mobility:
            mu_n = mobility_caughey_thomas(nt, mat, T, "n")
            mu_p = mobility_caughey_thomas(nt, mat, T, "p")
        else:
            mu_n = np.full(self.shape, mat.mu_n_max)
            mu_p = np.full(self.shape, mat.mu_p_max)
        self.tau_n = lifetime_scharfetter(nt, mat.tau_n0, mat.tau_Nref)
        self.tau_p = lifetime_scharfetter(nt, mat.tau_p0, mat.tau_Nref)
        # per-edge SG coefficients at the low node (pytcad/device2d.py:442-450)
        self.an, self.ap, self.dl = [], [], []
        for ax in range(self.dim):
            lo, hi = self.lo(ax), self.hi(ax)
            hb = self.bcast(self.h[ax], ax)
            dn = _hmean(mu_n[lo], mu_n[hi]) * self.VT / D0_REF
            dp = _hmean(mu_p[lo], mu_p[hi]) * self.VT / D0_REF
            an = np.zeros(self.shape); ap = np.zeros(self.shape); dl = np.zeros(self.shape)
            an[lo] = dn / hb
            ap[lo] = dp / hb
            dl[lo] = np.log(self.nie_s[hi] / self.nie_s[lo])
            self.an.append(an); self.ap.append(ap); self.dl.append(dl)
        self.bcs = {}

    # ---- axis helpers (axis 0 = x is the last array axis)
    def arr_axis(self, ax):
        return self.dim - 1 - ax

    def lo(self, ax):
        s = [slice(None)] * self.dim
        s[self.arr_axis(ax)] = slice(None, -1)
        return tuple(s)

    def hi(self, ax):
        s = [slice(None)] * self.dim
        s[self.arr_axis(ax)] = slice(1, None)
        return tuple(s)

    def bcast(self, v, ax):
        shp = [1] * self.dim
        shp[self.arr_axis(ax)] = v.size
        return v.reshape(shp)

    def flat(self, *ijk):
        out = np.atleast_1d(np.asarray(ijk[0], dtype=np.int64))
        stride = 1
        for a in range(1, self.dim):
            stride *= self.nax[a - 1]
            out = out + np.atleast_1d(np.asarray(ijk[a], dtype=np.int64)) * stride
        return out

    def bulk_guess(self):
        """Neutral-bulk potential (pytcad/device2d.py:744-759)."""
        return np.arcsinh(self.C / (2.0 * self.nie_s))

    def gate_kappa(self, tox_cm):
        """pytcad/device2d.py:676-680."""
        return EPS_OX_R * EPS0 * self.LD / (self.eps * tox_cm)

    def gate_weight(self, idx, normal_axis):
        """Face length (2D) or face area normal to `normal_axis` (3D,
        pytcad/device3d.py:939-947) the gate flux crosses."""
        dv = self.dv
        if self.dim == 2:
            return dv[0][idx[0]]
        if normal_axis == "z":
            return dv[0][idx[0]] * dv[1][idx[1]]
        if normal_axis == "y":
            return dv[0][idx[0]] * dv[2][idx[2]]
        return dv[1][idx[1]] * dv[2][idx[2]]

    # ---- boundary-condition arrays
    def contact_table(self):
        """Unique contact nodes (a later contact wins a shared node, as the
        reference's row stamping does), their contact index, ln(n0/nie),
        n0 and p0 (pytcad/contacts.py:21-38)."""
        names = [n for n, b in self.bcs.items() if b.kind == "contact"]
        owner = {}
        for ci, name in enumerate(names):
            for k in self.bcs[name].nodes:
                owner[int(k)] = ci
        nodes = np.array(sorted(owner), dtype=np.int64)
        cid = np.array([owner[int(k)] for k in nodes], dtype=np.int32)
        L, n0, p0 = ohmic_values(self.C.ravel()[nodes], self.nie_s.ravel()[nodes], 0.0,
                                 self.VT)
        return names, nodes, cid, L, n0, p0

    def gate_arrays(self):
        """Per-node kappa*w, V/VT - Vfb/VT (bias and equilibrium) and psi_b
        for every gate node (pytcad/device2d.py:1624-1637)."""
        gk = np.zeros(self.N); gv = np.zeros(self.N); gveq = np.zeros(self.N)
        gb = np.zeros(self.N); cnt = np.zeros(self.N, dtype=np.int64)
        acc_v = np.zeros(self.N); acc_veq = np.zeros(self.N)
        Cf, nief = self.C.ravel(), self.nie_s.ravel()
        for b in self.bcs.values():
            if b.kind != "gate":
                continue
            k = b.nodes
            kw = b.kappa * b.w
            v = b.Vg / self.VT - b.Vfb / self.VT
            veq = 0.0 - b.Vfb / self.VT
            first = cnt[k] == 0
            gk[k] = np.where(first, kw, gk[k] + kw)
            gv[k] = np.where(first, v, gv[k]); gveq[k] = np.where(first, veq, gveq[k])
            acc_v[k] += kw * v; acc_veq[k] += kw * veq
            gb[k] = np.arcsinh(Cf[k] / (2.0 * nief[k]))
            cnt[k] += 1
        multi = cnt > 1   # several gates on a node: kappa*w-weighted mean
        gv[multi] = acc_v[multi] / gk[multi]
        gveq[multi] = acc_veq[multi] / gk[multi]
        return cnt > 0, gk, gv, gveq, gb


NODE_ARRAYS = ("C", "nie", "nie_s", "tau_n", "tau_p")
BC_ARRAYS = ("bc_psi0", "bc_n0", "bc_p0", "bc_psi0_eq", "gate_k", "gate_v", "gate_veq",
             "gate_b")


def node_arrays(s):
    """Per-node coefficient arrays of a set-up, flattened, by pack name."""
    out = {name: getattr(s, name).ravel() for name in NODE_ARRAYS}
    for a in range(s.dim):
        for name in ("an", "ap", "dl"):
            out[f"{name}{a}"] = getattr(s, name)[a].ravel()
    return out


def axis_arrays(s, dim):
    """Per-axis (h, dv) of a set-up as packed: h padded with one 0 so that both
    have the node count; axes beyond dim get a single (0, 1) entry."""
    out = []
    for a in range(3):
        if a < dim:
            out.append((np.concatenate([s.h[a], [0.0]]), s.dv[a]))
        else:
            out.append((np.zeros(1), np.ones(1)))
    return out


def instance_par(s):
    par = np.zeros(_lib.NPAR)
    par[0] = s.Ns
    par[1] = s.R0
    par[2] = s.mat.Cn_auger
    par[3] = s.mat.Cp_auger
    par[4] = 1.0 if s.models.srh else 0.0
    par[5] = 1.0 if s.models.auger else 0.0
    return par


def choose_tile_z(setups, dim, sm_count=148, ctas_per_sm=3, waves=4.0):
    """Starting z depth of the 3D assembly tiles (tcad_b200.tune measures the
    best one at a pack's first coupled solve): the deeper of 4 and 2 planes
    whose tile count still fills `waves` waves of the GPU's CTA slots, else 1.
    A deeper tile re-evaluates fewer z-edges at its first plane, but deep
    tiles leave a long last wave: measured, 1-2 planes are best on a 1M-node
    mesh and 4 on an 8M-node one; 8 and 16 are slower on both."""
    if dim != 3:
        return 1
    slots = sm_count * ctas_per_sm * waves
    for tz in (4, 2):
        n = sum(-(-s.nax[0] // _lib.TILE_X) * -(-s.nax[1] // _lib.TILE_Y) * -(-s.nax[2] // tz)
                for s in setups)
        if n >= slots:
            return tz
    return 1


def instance_tiles(s, dim, tile_z=1):
    """Stencil tiles (i0, j0, k0) of one instance, x fastest."""
    nz = s.nax[2] if dim == 3 else 1
    kstep = tile_z if dim == 3 else 1
    k0, j0, i0 = np.meshgrid(np.arange(0, nz, kstep), np.arange(0, s.nax[1], _lib.TILE_Y),
                             np.arange(0, s.nax[0], _lib.TILE_X), indexing="ij")
    return np.stack([i0.ravel(), j0.ravel(), k0.ravel()], axis=1).astype(np.int32)


def instance_tables(setups, dim, node_off, axis_off, tiles=None, tile_z=1,
                    flat_nodes=None):
    """The per-instance tables of include/tcad_b200.h for instances placed at
    node_off[i] (increasing) with axis entries at axis_off[i, a]; 3D tiles
    `tile_z` planes deep, flat blocks of `flat_nodes` nodes."""
    ni = len(setups)
    flat_nodes = int(flat_nodes or _lib.FLAT_NODES)
    sizes = [s.N for s in setups]
    nflat = [-(-n // flat_nodes) for n in sizes]
    flat_off = np.concatenate(([0], np.cumsum(nflat))).astype(np.int64)
    flat_inst = np.repeat(np.arange(ni, dtype=np.int32), nflat)
    shape = np.ones((ni, 3), dtype=np.int32)
    for i, s in enumerate(setups):
        shape[i, :dim] = s.nax[:dim]
    tiles = tiles if tiles is not None else [instance_tiles(s, dim, tile_z) for s in setups]
    tl = (np.concatenate([np.concatenate([np.full((t.shape[0], 1), i, np.int32), t], axis=1)
                          for i, t in enumerate(tiles)]).ravel()
          if ni else np.zeros(0, np.int32))
    par = np.stack([instance_par(s) for s in setups]) if ni else np.zeros((0, _lib.NPAR))
    return dict(shape=shape.ravel(), node_off=np.asarray(node_off, np.int64),
                flat_off=flat_off, flat_inst=flat_inst, tile_z=int(tile_z),
                flat_nodes=flat_nodes,
                axis_off=np.asarray(axis_off, np.int64).ravel(), tile=tl.astype(np.int32),
                par=par.ravel())


def bc_node_arrays(s):
    """Boundary-condition node arrays of one instance (local node index):
    flag, psi0 at equilibrium on contacts, and the gate arrays; plus its
    contact table."""
    flag = np.zeros(s.N, dtype=np.uint8)
    psi0eq = np.zeros(s.N)
    names, nodes, cid, L, n0, p0 = s.contact_table()
    g_on, g_k, g_v, g_veq, g_b = s.gate_arrays()
    flag[g_on] |= _lib.BC_GATE
    flag[nodes] |= _lib.BC_CONTACT
    psi0eq[nodes] = 0.0 / s.VT + L
    arrs = dict(bcflag=flag, bc_psi0_eq=psi0eq, gate_k=g_k, gate_v=g_v, gate_veq=g_veq,
                gate_b=g_b)
    return arrs, (names, nodes, cid, L, n0, p0)


def gate_map(s):
    """What the bias update needs to recompute V/VT - Vfb/VT on an
    instance's gate nodes alone: the gates, each gate's slots among the gate
    nodes, its kappa*w, the nodes' summed kappa*w, VT; and the local gate
    nodes.  (None, None) when the instance has no gate."""
    gates = [b for b in s.bcs.values() if b.kind == "gate"]
    if not gates:
        return None, None
    on, gk, _, _, _ = s.gate_arrays()
    nodes = np.nonzero(on)[0]
    slot = np.full(s.N, -1, dtype=np.int64)
    slot[nodes] = np.arange(nodes.size)
    return (gates, [slot[b.nodes] for b in gates], [b.kappa * b.w for b in gates],
            gk[nodes], s.VT), nodes


def gate_values(gm):
    """V/VT - Vfb/VT on the gate nodes, Setup.gate_arrays' arithmetic in the
    same order (a node under several gates takes the kappa*w-weighted mean)."""
    gates, slots, kws, gk, VT = gm
    m = gk.size
    gv = np.zeros(m); acc = np.zeros(m); cnt = np.zeros(m, dtype=np.int64)
    for b, j, kw in zip(gates, slots, kws):
        v = b.Vg / VT - b.Vfb / VT
        first = cnt[j] == 0
        gv[j] = np.where(first, v, gv[j])
        acc[j] += kw * v
        cnt[j] += 1
    multi = cnt > 1
    gv[multi] = acc[multi] / gk[multi]
    return gv


def bias_vector(setup):
    """Every contact's V and gate's Vg, in BC order: the bias of a state."""
    return np.array([b.V if b.kind == "contact" else b.Vg for b in setup.bcs.values()],
                    dtype=float)


def secant_ratio(prev, cur, new, smax=2.0):
    """Step ratio s of the secant predictor: new - cur = s (cur - prev) with
    0 < s <= smax, else 0 (no prediction)."""
    if prev is None or cur is None or len(prev) != len(new) or len(cur) != len(new):
        return 0.0
    d1, d2 = cur - prev, new - cur
    n1 = float(d1 @ d1)
    if not n1 > 0.0:
        return 0.0
    s = float(d1 @ d2) / n1
    if not 0.0 < s <= smax:
        return 0.0
    if np.abs(d2 - s * d1).max() > 1e-9 * max(np.abs(d2).max(), 1e-12):
        return 0.0
    return s


class Pack:
    """Device-memory image of a list of Setups of one dimension, packed back
    to back."""

    # measure the 3D assembly tile depth at the first coupled solve
    # (tcad_b200.tune); results do not depend on it
    autotune = True

    def __init__(self, setups, device="cuda"):
        import torch
        self._init_common(setups, device)
        dim = self.dim
        sizes = [s.N for s in self.setups]
        node_off = np.concatenate(([0], np.cumsum(sizes))).astype(np.int64)
        self.N = int(node_off[-1])
        axes = [axis_arrays(s, dim) for s in self.setups]
        axis_off = np.zeros((len(self.setups), 3), dtype=np.int64)
        for a in range(3):
            lens = [ax[a][1].size for ax in axes]
            axis_off[:, a] = np.concatenate(([0], np.cumsum(lens)[:-1]))
        up = self._up
        t = {}
        for a in range(3):
            t[f"h{a}"] = up(np.concatenate([ax[a][0] for ax in axes]))
            t[f"dv{a}"] = up(np.concatenate([ax[a][1] for ax in axes]))
        per = [node_arrays(s) for s in self.setups]
        for name in per[0]:
            t[name] = up(np.concatenate([q[name] for q in per]))
        for name in BC_ARRAYS:
            t[name] = torch.zeros(self.N, dtype=torch.float64, device=self.device)
        t["bcflag"] = torch.zeros(self.N, dtype=torch.uint8, device=self.device)
        self.t = t
        self._set_tables(instance_tables(self.setups, dim, node_off[:-1], axis_off,
                                         tile_z=choose_tile_z(self.setups, dim)))
        # state and solver buffers
        z = lambda n: torch.zeros(n, dtype=torch.float64, device=self.device)  # noqa: E731
        self.psi, self.n, self.p = z(self.N), z(self.N), z(self.N)
        self.F = z(3 * self.N)
        self.J = z(_lib.NE[dim] * self.N)
        self.du = z(3 * self.N)
        wb = int(self.lib.tcad_block_workspace_bytes(self.pref, 2, 0))
        self.work = torch.empty(wb, dtype=torch.uint8, device=self.device)
        self.active = torch.ones(len(self.setups), dtype=torch.uint8, device=self.device)
        self.refresh_bcs()

    def predict(self, ratios):
        """Secant predictor per instance (tcad_state_extrapolate); saves the
        current state into the prev buffers first."""
        torch = self.torch
        if getattr(self, "_prev", None) is None:
            self._prev = tuple(torch.zeros_like(self.psi) for _ in range(3))
        r = self._up(np.asarray(ratios, dtype=float))
        rc = self.lib.tcad_state_extrapolate(
            self.pref, _lib.ptr(self.psi), _lib.ptr(self.n), _lib.ptr(self.p),
            *(_lib.ptr(t) for t in self._prev), _lib.ptr(r), self.sp())
        _lib.check(rc, "tcad_state_extrapolate")
        self._ratio_keep = r

    def restore_prev(self, insts=None):
        """State of the listed instances (all by default) back from the prev
        buffers (the state before the last prediction)."""
        insts = range(len(self.setups)) if insts is None else insts
        for i in insts:
            a, b = int(self.node_off[i]), int(self.node_off[i]) + self.setups[i].N
            for cur, prev in zip((self.psi, self.n, self.p), self._prev):
                cur[a:b].copy_(prev[a:b])

    def _init_common(self, setups, device):
        import torch
        self.torch = torch
        self.setups = list(setups)
        dims = {s.dim for s in self.setups}
        if len(dims) != 1:
            raise ValueError("a pack holds instances of one dimension")
        self.dim = dims.pop()
        self.lib = _lib.load()
        self.device = torch.device(device)
        self.last_h2d_bytes = 0

    def _up(self, a, dtype=None):
        torch = self.torch
        return torch.from_numpy(np.ascontiguousarray(a)).to(self.device,
                                                            dtype or torch.float64)

    def _set_tables(self, tb):
        """Upload the per-instance tables (instances at tb["node_off"], node
        arrays of length self.N) and fill the C struct."""
        torch = self.torch
        t = self.t
        ni = len(self.setups)
        self.node_off = np.concatenate([tb["node_off"][:ni], [self.N]]).astype(np.int64)
        self.flat_off = tb["flat_off"]
        self.n_flat = int(self.flat_off[-1])
        self.n_tiles = tb["tile"].size // 4
        t["shape"] = self._up(tb["shape"], torch.int32)
        t["node_off"] = self._up(self.node_off, torch.int64)
        t["flat_off"] = self._up(tb["flat_off"], torch.int64)
        t["flat_inst"] = self._up(tb["flat_inst"], torch.int32)
        t["axis_off"] = self._up(tb["axis_off"], torch.int64)
        t["tile"] = self._up(tb["tile"], torch.int32)
        t["par"] = self._up(tb["par"])
        dim = self.dim
        P = _lib.TcadPack()
        P.dim = dim; P.n_inst = ni; P.n_nodes = self.N
        P.n_flat = self.n_flat; P.n_tiles = self.n_tiles
        P.tile_z = self.tile_z = tb["tile_z"]
        P.flat_nodes = self.flat_nodes = tb["flat_nodes"]
        P.asm_stage = self.asm_stage = 0
        for f in ("shape", "node_off", "flat_off", "flat_inst", "axis_off", "tile", "par",
                  "C", "nie", "nie_s", "tau_n", "tau_p", "bcflag") + BC_ARRAYS:
            setattr(P, f, t[f].data_ptr())
        for a in range(3):
            P.h[a] = t[f"h{a}"].data_ptr()
            P.dv[a] = t[f"dv{a}"].data_ptr()
            src = a if a < dim else 0
            P.an[a] = t[f"an{src}"].data_ptr()
            P.ap[a] = t[f"ap{src}"].data_ptr()
            P.dl[a] = t[f"dl{src}"].data_ptr()
        self.P = P
        self.pref = ctypes.byref(P)

    # ---------------------------------------------------------------------
    def sp(self):
        return _lib.stream_ptr()

    def refresh_bcs(self):
        """(Re)build the boundary-condition arrays from every instance's BCs."""
        torch = self.torch
        N = self.N
        full = {"bcflag": np.zeros(N, dtype=np.uint8)}
        for name in ("bc_psi0_eq", "gate_k", "gate_v", "gate_veq", "gate_b"):
            full[name] = np.zeros(N)
        tables = []
        for i, s in enumerate(self.setups):
            off = int(self.node_off[i])
            arrs, ctab = bc_node_arrays(s)
            for name, a in arrs.items():
                full[name][off:off + s.N] = a
            tables.append(ctab)
        for name, a in full.items():
            self.t[name].copy_(self._up(a, torch.uint8 if name == "bcflag" else None))
        self._contact_tables(tables)
        self._build_gate_map()
        self.set_bias()

    def _contact_tables(self, tables):
        """Device contact lists from each instance's contact table (local node
        indices) placed at node_off[i]."""
        torch = self.torch
        c_nodes, c_cid, c_L, c_n0, c_p0 = [], [], [], [], []
        self.c_off = [0]
        self.contact_names = []
        self.cid_base = []
        base = 0
        for i, (names, nodes, cid, L, n0, p0) in enumerate(tables):
            off = int(self.node_off[i])
            self.contact_names.append(names)
            self.cid_base.append(base)
            c_nodes.append(off + nodes); c_cid.append(base + cid)
            self.c_off.append(self.c_off[-1] + nodes.size)
            c_L.append(L); c_n0.append(n0); c_p0.append(p0)
            base += len(names)
        self.n_contacts_total = base
        cat = lambda xs: np.concatenate(xs) if xs else np.zeros(0)  # noqa: E731
        self.c_nodes = self._up(cat(c_nodes), torch.int64)
        self.c_cid = self._up(cat(c_cid), torch.int32)
        self.c_L = self._up(cat(c_L))
        self.c_n0 = self._up(cat(c_n0))
        self.c_p0 = self._up(cat(c_p0))
        # per contact: device node list (for terminal currents)
        self.contact_lists = {}
        for i, s in enumerate(self.setups):
            off = int(self.node_off[i])
            for name, b in s.bcs.items():
                if b.kind == "contact":
                    self.contact_lists[(i, name)] = self._up(off + np.unique(b.nodes),
                                                             torch.int64)
        maxc = max([v.numel() for v in self.contact_lists.values()] + [1])
        self.cur_partial = torch.zeros(2 * maxc, dtype=torch.float64, device=self.device)
        self.cur_out = torch.zeros(max(len(self.contact_lists), 1), dtype=torch.float64,
                                   device=self.device)

    def _build_gate_map(self, cached=None):
        """Per instance with gates: gate map and global gate nodes (increasing)
        for set_bias; cached: optional per-instance (map, local nodes)."""
        self._gate_maps, self._gate_inst, idx = {}, [], []
        for i, s in enumerate(self.setups):
            gm, nodes = cached[i] if cached is not None else gate_map(s)
            if gm is None:
                continue
            self._gate_maps[i] = gm
            self._gate_inst.append(i)
            idx.append(int(self.node_off[i]) + nodes)
        self._gate_idx = self._up(np.concatenate(idx), self.torch.int64) if idx else None

    def _gate_values(self, i):
        return gate_values(self._gate_maps[i])

    def set_bias(self, voltages=None):
        """Contact targets at each contact's voltage and the gates' Vg terms.
        voltages: optional per-instance {name: V} overriding the stored V."""
        torch = self.torch
        vv = np.zeros(max(self.n_contacts_total, 1))
        for i, s in enumerate(self.setups):
            over = voltages[i] if voltages else {}
            for ci, name in enumerate(self.contact_names[i]):
                V = over.get(name, s.bcs[name].V) if over else s.bcs[name].V
                vv[self.cid_base[i] + ci] = V / s.VT
        vvt = torch.from_numpy(vv).to(self.device)
        rc = self.lib.tcad_set_contacts(
            self.pref, _lib.ptr(self.c_nodes), self.c_nodes.numel(), _lib.ptr(self.c_cid),
            _lib.ptr(vvt), _lib.ptr(self.c_L), _lib.ptr(self.c_n0), _lib.ptr(self.c_p0),
            _lib.ptr(self.t["bc_psi0"]), _lib.ptr(self.t["bc_n0"]), _lib.ptr(self.t["bc_p0"]),
            self.sp())
        _lib.check(rc, "tcad_set_contacts")
        # gate V/VT - Vfb/VT at the current Vg, recomputed on the gate nodes
        # only (the arithmetic of Setup.gate_arrays, in the same order) and
        # scattered into the node array on the device
        self.last_h2d_bytes = vv.nbytes
        if self._gate_idx is not None:
            vals = np.concatenate([self._gate_values(i) for i in self._gate_inst])
            vt = torch.from_numpy(vals).to(self.device)
            self.t["gate_v"].index_copy_(0, self._gate_idx, vt)
            self.last_h2d_bytes += vals.nbytes
            self._gvt = vt
        self._vvt = vvt  # keep alive until the kernel ran

    def stamp_contacts(self, active=None):
        """Contact nodes take their targets (all instances, or the instances
        with active[i] set: their contact nodes are contiguous in c_nodes)."""
        if active is None:
            ranges = [(0, self.c_nodes.numel())]
        else:
            ranges = [(self.c_off[i], self.c_off[i + 1]) for i, a in enumerate(active) if a]
        for a, b in ranges:
            if b <= a:
                continue
            rc = self.lib.tcad_stamp_contacts(
                self.pref, ctypes.c_void_p(self.c_nodes.data_ptr() + 8 * a), b - a,
                _lib.ptr(self.psi), _lib.ptr(self.n), _lib.ptr(self.p), self.sp())
            _lib.check(rc, "tcad_stamp_contacts")

    # ---- kernels -----------------------------------------------------------
    def assemble(self, mode, psi=None, n=None, p=None):
        rc = self.lib.tcad_sg_assemble(
            self.pref, _lib.ptr(self.psi if psi is None else psi),
            _lib.ptr(self.n if n is None else n), _lib.ptr(self.p if p is None else p),
            _lib.ptr(self.F), _lib.ptr(self.J), mode, self.sp())
        _lib.check(rc, "tcad_sg_assemble")

    def assemble_poisson(self, mode, psi=None, F=None, J=None):
        rc = self.lib.tcad_poisson_assemble(
            self.pref, _lib.ptr(self.psi if psi is None else psi),
            _lib.ptr(self.F if F is None else F), _lib.ptr(self.J if J is None else J),
            mode, self.sp())
        _lib.check(rc, "tcad_poisson_assemble")

    def contact_current(self, inst, name, psi=None, n=None, p=None, out_slot=0):
        """Deterministic sum of raw F_n + F_p over a contact's nodes (scaled)."""
        nodes = self.contact_lists[(inst, name)]
        rc = self.lib.tcad_contact_current(
            self.pref, _lib.ptr(self.psi if psi is None else psi),
            _lib.ptr(self.n if n is None else n), _lib.ptr(self.p if p is None else p),
            _lib.ptr(nodes), nodes.numel(), _lib.ptr(self.cur_partial),
            self.cur_partial.numel(), _lib.ptr(self.cur_out[out_slot:]), self.sp())
        _lib.check(rc, "tcad_contact_current")
        return self.cur_out[out_slot]

    def raw_continuity(self, nodes_dev, psi, n, p):
        """Raw (F_n, F_p) at a device node list."""
        torch = self.torch
        cnt = nodes_dev.numel()
        part = torch.zeros(2 * max(cnt, 1), dtype=torch.float64, device=self.device)
        out = torch.zeros(1, dtype=torch.float64, device=self.device)
        rc = self.lib.tcad_contact_current(self.pref, _lib.ptr(psi), _lib.ptr(n),
                                           _lib.ptr(p), _lib.ptr(nodes_dev), cnt,
                                           _lib.ptr(part), part.numel(), _lib.ptr(out),
                                           self.sp())
        _lib.check(rc, "tcad_contact_current")
        return part[:cnt], part[cnt:2 * cnt]

    def edge_currents(self, axis, psi=None, n=None, p=None):
        torch = self.torch
        Jn = torch.empty(self.N, dtype=torch.float64, device=self.device)
        Jp = torch.empty(self.N, dtype=torch.float64, device=self.device)
        rc = self.lib.tcad_edge_currents(
            self.pref, axis, _lib.ptr(self.psi if psi is None else psi),
            _lib.ptr(self.n if n is None else n), _lib.ptr(self.p if p is None else p),
            _lib.ptr(Jn), _lib.ptr(Jp), self.sp())
        _lib.check(rc, "tcad_edge_currents")
        return Jn, Jp

    def newton_opts(self, opts, equilibrium=False):
        o = _lib.NewtonOpts()
        o.max_iter = int(opts.max_iter)
        o.method = 1 if opts.linsolve == "gmres" and not equilibrium else 0
        o.method = 0  # the node-block path runs BiCGStab (GMRES: see linsolve.py)
        o.krylov_maxiter = int(getattr(opts, "linsolve_maxiter", 4000))
        o.restart = 0
        o.tol_update = float(opts.tol_update)
        o.max_dpsi = float(opts.max_dpsi)
        o.rtol = float(opts.linsolve_rtol)
        o.dens_floor = 1e-10
        o.verbose = 1 if opts.verbose else 0
        o.polish = 0 if equilibrium else int(getattr(opts, "polish", 0))
        o.forcing = 1 if getattr(opts, "forcing", "fixed") == "adaptive" else 0
        o.eta_max = float(getattr(opts, "eta_max", 1e-3))
        prec = getattr(opts, "precision", "fp64")
        o.precision = {"mixed": 32, "fp32_operator": 33}.get(prec, 64) if not equilibrium else 64
        o.density_scaling = 1 if getattr(opts, "krylov_unknowns", "relative") == "relative" else 0
        em = getattr(opts, "eta_min", None)
        if em is None:
            em = o.eta_max if o.precision in (64, 33) else opts.linsolve_rtol
        o.eta_min = float(em)
        o.scale_floor = float(getattr(opts, "krylov_scale_floor", 1e-10))
        pc = getattr(opts, "precond", "auto")
        # "ilu": ILU(0) everywhere (3D: per z-plane); "auto"/"schur": on 2D
        # packs ILU(0) for batches and for any instance whose node-block-Jacobi
        # solve fails, 3D packs keep node-block Jacobi
        o.precond = {"ilu": 1, "auto": 2, "schur": 2}.get(pc, 0)
        o.polish_eta = float(getattr(opts, "polish_eta", 1e-10))
        o.polish_scale_floor = float(getattr(opts, "polish_scale_floor", 0.0))
        o.red_black = 1 if getattr(opts, "krylov_system", "full") == "red_black" else 0
        return o

    def set_tile_z(self, tile_z):
        """Re-tile the 3D assembly `tile_z` planes deep (the tile list and
        the workspace's tile-list room follow)."""
        if self.dim != 3:
            return
        tiles = [instance_tiles(s, 3, tile_z) for s in self.setups]
        tl = np.concatenate([np.concatenate([np.full((t.shape[0], 1), i, np.int32), t], axis=1)
                             for i, t in enumerate(tiles)]).ravel().astype(np.int32)
        self.t["tile"] = self._up(tl, self.torch.int32)
        self.n_tiles = tl.size // 4
        P = self.P
        P.tile = self.t["tile"].data_ptr()
        P.n_tiles = self.n_tiles
        P.tile_z = self.tile_z = int(tile_z)
        wb = int(self.lib.tcad_block_workspace_bytes(self.pref, 2, 0))
        if wb > self.work.numel():
            self.work = self.torch.empty(wb, dtype=self.torch.uint8, device=self.device)

    def set_asm_stage(self, stage):
        """3D coupled assembly: 1 stages each next z-plane's coefficients in
        shared memory with asynchronous copies, 0 loads them in place (the
        same arithmetic either way)."""
        self.P.asm_stage = self.asm_stage = int(bool(stage)) if self.dim == 3 else 0

    def newton(self, opts, active=None, transient=None):
        """Coupled Newton on every (active) instance; `transient` = {dt (scaled
        time), theta, n_old, p_old[, fn_old, fp_old]} (device tensors) makes
        it one step of the theta scheme (tcad_newton_opts_t.dt)."""
        ni = len(self.setups)
        if self.autotune and self.dim == 3 and not getattr(self, "_tuned", False):
            from . import tune
            tune.tune_assembly(self)
            self._tuned = True
        if active is None:
            self.active.fill_(1)
        else:
            self.active.copy_(self.torch.as_tensor(np.asarray(active, np.uint8)))
        o = self.newton_opts(opts)
        if transient is not None:
            o.dt = float(transient["dt"])
            o.theta = float(transient.get("theta", 1.0))
            o.n_old = transient["n_old"].data_ptr()
            o.p_old = transient["p_old"].data_ptr()
            for f in ("fn_old", "fp_old"):
                t = transient.get(f)
                setattr(o, f, t.data_ptr() if t is not None else None)
        res = (_lib.NewtonResult * ni)()
        rc = self.lib.tcad_newton_solve(
            self.pref, _lib.ptr(self.psi), _lib.ptr(self.n), _lib.ptr(self.p),
            _lib.ptr(self.F), _lib.ptr(self.J), _lib.ptr(self.du), ctypes.byref(o),
            _lib.ptr(self.active), _lib.ptr(self.work), self.work.numel(), res, self.sp())
        _lib.check(rc, "tcad_newton_solve")
        return [dict(iters=r.iters, converged=bool(r.converged),
                     krylov_iters=r.krylov_iters, status=r.status, err=r.err,
                     relres=r.relres, fp64_from=r.fp64_from,
                     polish_iters=r.polish_iters) for r in res]

    def equilibrium(self, opts):
        ni = len(self.setups)
        o = self.newton_opts(opts, equilibrium=True)
        o.krylov_maxiter = max(o.krylov_maxiter, 20000)
        res = (_lib.NewtonResult * ni)()
        d = self.du[: self.N]
        rc = self.lib.tcad_equilibrium_solve(
            self.pref, _lib.ptr(self.psi), _lib.ptr(self.n), _lib.ptr(self.p),
            _lib.ptr(self.F), _lib.ptr(self.J), _lib.ptr(d), ctypes.byref(o),
            _lib.ptr(self.work), self.work.numel(), res, self.sp())
        _lib.check(rc, "tcad_equilibrium_solve")
        return [dict(iters=r.iters, converged=bool(r.converged),
                     krylov_iters=r.krylov_iters, status=r.status, err=r.err,
                     relres=r.relres, fp64_from=r.fp64_from,
                     polish_iters=r.polish_iters) for r in res]
