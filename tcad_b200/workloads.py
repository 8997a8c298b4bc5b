"""Synthetic device workloads with explicit node counts.

The reference publishes no dataset for this path; these builders generate the
devices its own builders would (pytcad/mosfet.py:26-87,
pytcad/finfet3d.py:61-152) on meshes with exact node counts, seeded where
random.  Doping profiles follow pytcad/mosfet.py:26-54 (Gaussian in depth x
erfc lateral roll-off).
"""
from __future__ import annotations

import numpy as np
from scipy.special import erfc

from .physics import Mesh2D, Mesh3D, Semiconductor, flatband_voltage, graded_nodes
from .options import Models


def sd_profile(x, y, x_edge, sigma_y, sigma_lat, Npeak, high_side):
    """Gaussian-in-depth x erfc-lateral source/drain profile, shape (Ny, Nx)
    (pytcad/mosfet.py:26-35)."""
    vertical = np.exp(-(y[:, None]) ** 2 / (2.0 * sigma_y ** 2))
    s = (x_edge - x) if high_side == "left" else (x - x_edge)
    lateral = 0.5 * erfc(-s[None, :] / (np.sqrt(2.0) * sigma_lat))
    return Npeak * vertical * lateral


def mosfet_doping(x, y, Lsd, Lg, Na, Nsd_peak, sigma_y, sigma_lat):
    """Net doping and total impurity concentration (pytcad/mosfet.py:38-54)."""
    channel = -Na * np.ones((y.size, x.size))
    source = sd_profile(x, y, Lsd, sigma_y, sigma_lat, Nsd_peak, "left")
    drain = sd_profile(x, y, Lsd + Lg, sigma_y, sigma_lat, Nsd_peak, "right")
    return channel + source + drain, np.abs(channel) + source + drain


def diode_x(nx, L=2.0e-4, xj=1.0e-4, ratio=1.05):
    """nx nodes on [0, L], cell widths a symmetric geometric series growing by
    `ratio` away from the junction xj on both sides."""
    half = (nx - 1) // 2
    w = ratio ** np.arange(half)
    w = w / w.sum() * xj
    right = np.concatenate(([0.0], np.cumsum(w)))
    x = np.concatenate([xj - right[::-1], xj + right[1:]])
    x[0], x[-1] = 0.0, L
    return x


def diode2d(dev_cls, nx=201, ny=101):
    """Plain-method CPU-runnable workload: silicon abrupt p-n diode, 2 um x
    1 um, N_A 1e17 | N_D 1e18, constant mobility, SRH tau 1e-7 s, ohmic left
    and right edges.  Sweep: 0 .. 0.7 V in 0.05 V steps on "anode"."""
    x = diode_x(nx)
    y = np.linspace(0.0, 1.0e-4, ny)
    dop = np.where(np.meshgrid(x, y)[0] < 1.0e-4, -1e17, 1e18)
    mat = Semiconductor(tau_n0=1e-7, tau_p0=1e-7, tau_Nref=1e300)
    dev = dev_cls(Mesh2D(x, y), dop, material=mat,
                  models=Models(doping_mobility=False, srh=True, auger=False, bgn=False))
    dev.add_contact("anode", np.zeros(ny, int), np.arange(ny))
    dev.add_contact("cathode", np.full(ny, nx - 1), np.arange(ny))
    return dev


DIODE_SWEEP = [round(0.05 * i, 10) for i in range(15)]


def trigate3d(dev_cls, nx=160, ny=96, nz=64, Lg=40e-7, Lsd=40e-7, Hfin=40e-7,
              Wfin=20e-7, Na=1e18, Nsd_peak=1e20, sigma=10e-7, tox=1e-7,
              models=None):
    """n-channel tri-gate structure (pytcad/finfet3d.py:61-152 pattern) on an
    exact nx x ny x nz tensor mesh: p-body Na, Gaussian source/drain implants
    of peak Nsd_peak (sigma both in depth and laterally), gate length Lg,
    Robin gates (t_ox) on the top face (normal y) and both sidewalls (normal
    z) over the channel, ohmic source / drain on the n+ part of the x-end
    faces and a body contact on the fin bottom.  Models() defaults."""
    L = 2 * Lsd + Lg
    x = graded_nodes(nx, L, [Lsd, Lsd + Lg], 1.06)
    y = graded_nodes(ny, Hfin, [0.0], 1.02)
    z = graded_nodes(nz, Wfin, [0.0, Wfin], 1.04)
    dop2, nt2 = mosfet_doping(x, y, Lsd, Lg, Na, Nsd_peak, sigma, sigma)
    doping = np.broadcast_to(dop2, (nz, ny, nx)).copy()
    ntot = np.broadcast_to(nt2, (nz, ny, nx)).copy()
    dev = dev_cls(Mesh3D(x, y, z), doping, Ntotal=ntot, models=models or Models())
    J, K = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")
    for name, i in (("source", 0), ("drain", nx - 1)):
        ntype = dop2[J.ravel(), i] > 0
        dev.add_contact(name, np.full(int(ntype.sum()), i), J.ravel()[ntype], K.ravel()[ntype])
    bi, bk = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    body_p = dop2[ny - 1, bi.ravel()] < 0
    dev.add_contact("body", bi.ravel()[body_p], np.full(int(body_p.sum()), ny - 1),
                    bk.ravel()[body_p])
    ig = np.where((x > Lsd) & (x < Lsd + Lg))[0]
    Vfb = flatband_voltage(-Na, tox, "n+poly")
    ti, tk = np.meshgrid(ig, np.arange(nz), indexing="ij")
    dev.add_gate("gate_top", ti.ravel(), np.zeros(ti.size, int), tk.ravel(), tox_cm=tox,
                 Vfb=Vfb, normal_axis="y")
    li, lj = np.meshgrid(ig, np.arange(1, ny), indexing="ij")
    dev.add_gate("gate_left", li.ravel(), lj.ravel(), np.zeros(li.size, int), tox_cm=tox,
                 Vfb=Vfb, normal_axis="z")
    dev.add_gate("gate_right", li.ravel(), lj.ravel(), np.full(li.size, nz - 1),
                 tox_cm=tox, Vfb=Vfb, normal_axis="z")
    return dev


TRIGATE_VG = [round(0.05 * i, 10) for i in range(21)]
TRIGATE_VD = [0.05, 0.7]


def trigate_bias(Vd, Vg):
    return {"drain": Vd, "gate_top": Vg, "gate_left": Vg, "gate_right": Vg}


def trigate_schedule():
    """The bias points of the Id-Vg workload, in solve order: each Vd sweep
    starts from equilibrium (pytcad/finfet3d.py:246-263)."""
    pts = []
    for vd in TRIGATE_VD:
        for q, vg in enumerate(TRIGATE_VG):
            pts.append((vd, vg, q == 0))
    return pts
