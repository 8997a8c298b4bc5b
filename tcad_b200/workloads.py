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


def mosfet2d(dev_cls, nx=120, ny=60, Lg=100e-7, Lsd=None, depth=None, Na=1e17,
             Nsd_peak=1e20, tox=2e-7, sigma=None, ratio_x=1.08, ratio_y=1.06,
             models=None):
    """n-channel MOSFET on an exact nx x ny mesh, the structure of
    pytcad/mosfet.py:57-87 (build_mosfet): source/drain ohmic contacts on the
    surface over x <= Lsd / x >= Lsd+Lg, body contact on the bottom row, an
    oxide gate over the channel (n+poly flat-band), Gaussian-erfc S/D."""
    Lsd = Lg if Lsd is None else Lsd
    depth = 2.0 * Lg + 50e-7 if depth is None else depth
    sigma = Lg / 4.0 if sigma is None else sigma
    L = 2 * Lsd + Lg
    x = graded_nodes(nx, L, [Lsd, Lsd + Lg], ratio_x)
    y = graded_nodes(ny, depth, [0.0], ratio_y)
    dop, ntot = mosfet_doping(x, y, Lsd, Lg, Na, Nsd_peak, sigma, sigma)
    dev = dev_cls(Mesh2D(x, y), dop, Ntotal=ntot, models=models or Models())
    i_src = np.where(x <= Lsd)[0]
    i_drn = np.where(x >= Lsd + Lg)[0]
    i_gate = np.where((x > Lsd) & (x < Lsd + Lg))[0]
    dev.add_contact("source", i_src, np.zeros_like(i_src))
    dev.add_contact("drain", i_drn, np.zeros_like(i_drn))
    dev.add_contact("body", np.arange(nx), np.full(nx, ny - 1))
    Vfb = flatband_voltage(-Na, tox, "n+poly")
    dev.add_gate("gate", i_gate, np.zeros_like(i_gate), tox_cm=tox, Vfb=Vfb)
    return dev


def mosfet_batch_params(count=512, seed=2026, nx=(80, 400), ny=(40, 200), Lg=(30e-7, 200e-7),
                        Na=(1e16, 1e18), Npk=(1e19, 1e20), V=(0.0, 1.2)):
    """Seeded draws of the batched 2D MOSFET workload: per instance nx, ny
    uniform integers, Lg uniform, body doping and S/D peak log-uniform, and its
    own (Vg, Vd) uniform."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        out.append(dict(
            nx=int(rng.integers(nx[0], nx[1] + 1)), ny=int(rng.integers(ny[0], ny[1] + 1)),
            Lg=float(rng.uniform(*Lg)),
            Na=float(10.0 ** rng.uniform(np.log10(Na[0]), np.log10(Na[1]))),
            Nsd_peak=float(10.0 ** rng.uniform(np.log10(Npk[0]), np.log10(Npk[1]))),
            Vg=float(rng.uniform(*V)), Vd=float(rng.uniform(*V))))
    return out


def pin3d(dev_cls, nx=256, ny=256, nz=128, L=1.0e-4, W=0.5e-4, H=0.25e-4, x1=0.3e-4,
          x2=0.7e-4, NA=1e19, ND=1e19, Ni=1e14, lam=20e-7, ratio=1.03, models=None):
    """3D p-i-n diode on an exact nx x ny x nz tensor mesh: p+ (NA) for
    x < x1, intrinsic background Ni (n-type) between, n+ (ND) for x > x2,
    each transition an erfc of length lam; x graded toward the two
    junctions, y and z uniform; ohmic anode on the x = 0 face and cathode on
    the x = L face.  SRH + Auger with doping mobility (BGN off)."""
    x = graded_nodes(nx, L, [x1, x2], ratio)
    y = np.linspace(0.0, W, ny)
    z = np.linspace(0.0, H, nz)
    pa = 0.5 * NA * erfc((x - x1) / lam)
    nd = 0.5 * ND * erfc((x2 - x) / lam)
    net1 = nd + Ni - pa
    tot1 = nd + Ni + pa
    shape = (nz, ny, nx)
    dop = np.broadcast_to(net1[None, None, :], shape).copy()
    ntot = np.broadcast_to(tot1[None, None, :], shape).copy()
    m = models or Models(doping_mobility=True, srh=True, auger=True, bgn=False)
    dev = dev_cls(Mesh3D(x, y, z), dop, Ntotal=ntot, models=m)
    J, K = np.meshgrid(np.arange(ny), np.arange(nz), indexing="xy")
    J, K = J.ravel(), K.ravel()
    dev.add_contact("anode", np.zeros_like(J), J, K)
    dev.add_contact("cathode", np.full_like(J, nx - 1), J, K)
    return dev


PIN_SWEEP = [round(0.1 * k, 10) for k in range(10)]


def ramp(target, steps):
    """The explicit bias ramp both sides use: equal steps from 0 to the
    target, `steps` of them (the reference has no ramp of its own; every
    instance jumps from equilibrium through the same schedule)."""
    return [{k: v * (s + 1) / steps for k, v in target.items()} for s in range(steps)]
