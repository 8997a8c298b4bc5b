"""Shared test helpers: load the golden fixtures and rebuild the same device
for the oracle (CPU) or for the GPU product from the stored definition."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    with np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False) as f:
        return {k: f[k] for k in f.files}


def coords(g):
    return (g["x"], g["y"]) if int(g["dim"]) == 2 else (g["x"], g["y"], g["z"])


def bcs(g):
    """[(name, kind, flat node idx, vals)] in the fixture's insertion order."""
    out = []
    ptr = g["bc_ptr"]
    for b, name in enumerate(g["bc_names"]):
        out.append((str(name), str(g["bc_kinds"][b]),
                    g["bc_idx"][ptr[b]:ptr[b + 1]], g["bc_vals"][b]))
    return out


def unflat(g, k):
    nx, ny = g["x"].size, g["y"].size
    i = k % nx
    j = (k // nx) % ny
    if int(g["dim"]) == 2:
        return (i, j)
    return (i, j, k // (nx * ny))


def oracle_device(g, material=None):
    from oracle import OracleDevice, OracleModels, SILICON_PARAMS
    m = g["models"]
    mat = dict(SILICON_PARAMS)
    if material:
        mat.update(material)
    dev = OracleDevice(coords(g), g["doping"], Ntotal=g["Ntot"], T=float(g["T"]),
                       models=OracleModels(*[bool(v) for v in m]), material=mat)
    for name, kind, k, v in bcs(g):
        ijk = unflat(g, k)
        if kind == "contact":
            dev.add_contact(name, *ijk, V=v[0])
        else:
            dev.gates[name] = None
            _add_gate_kappa(dev, name, ijk, v)
    return dev


def _add_gate_kappa(dev, name, ijk, v):
    """Gate from the stored kappa (the reference stores kappa, not t_ox)."""
    kappa, Vfb, Vg, ax = v
    idx = [np.asarray(a, dtype=np.int64) for a in ijk]
    dv = dev.dv
    if dev.dim == 2:
        w = dv[0][idx[0]]
    else:
        axis = "xyz"[int(ax)]
        if axis == "z":
            w = dv[0][idx[0]] * dv[1][idx[1]]
        elif axis == "y":
            w = dv[0][idx[0]] * dv[2][idx[2]]
        else:
            w = dv[1][idx[1]] * dv[2][idx[2]]
    dev.gates[name] = [dev.flat(*ijk), float(kappa), float(Vfb), float(Vg), w]


def csr(g, prefix=""):
    import scipy.sparse as sp
    n = g[prefix + "J_indptr"].size - 1
    return sp.csr_matrix((g[prefix + "J_data"], g[prefix + "J_indices"],
                          g[prefix + "J_indptr"]), shape=(n, n))


def rownorm_err(A, B):
    """max over rows of ||A_r - B_r||_1 / ||B_r||_1 (normwise per row)."""
    D = (A - B).tocsr()
    Bc = B.tocsr()
    num = np.asarray(abs(D).sum(axis=1)).ravel()
    den = np.asarray(abs(Bc).sum(axis=1)).ravel()
    den = np.where(den == 0, 1.0, den)
    return float((num / den).max())


# Elementwise Jacobian bar.  1e-12 is the drop-in's bar for assembled
# entries; it holds for every entry except where the reference's own
# arithmetic amplifies an ulp of its math library: B'(x) = B(x) (1/x -
# 1/(1 - e^-x)) (pytcad/kernels.py:98-109) cancels about 4 digits at
# |x| = 1e-4, so one ulp of difference between two expm1 implementations
# (glibc's expm1 is itself not correctly rounded in ~1 of 1,300 arguments of
# that band) moves B' by up to 2 x 2^-52 / (|x| |B'|) = 4.4e-12.  Entries
# built from such a B' get TOL_ENTRY_CANCEL; the tests require that they are
# rare (TOL_ENTRY_FRACTION of the entries at most).
TOL_ENTRY = 1e-12
TOL_ENTRY_CANCEL = 5e-12
TOL_ENTRY_FRACTION = 1e-4


def elem_err(A, B, floor_rel=0.0):
    """Elementwise max |A_ij - B_ij| / |B_ij| over B's non-zero entries that
    are at least floor_rel x their row's largest |entry|.  A floor excludes
    entries formed where a sum of terms may cancel; the coupled Jacobian's
    duplicate sums add terms of one sign, so its default is 0 (every
    entry).  Entries of A outside B's pattern must be zero.  Returns
    (max error, entries compared, fraction of compared entries above
    TOL_ENTRY)."""
    A = A.tocsr().copy()
    B = B.tocsr().copy()
    for M in (A, B):
        M.sum_duplicates()
        M.sort_indices()
    n = B.shape[1]

    def keys(M):
        r = np.repeat(np.arange(M.shape[0], dtype=np.int64), np.diff(M.indptr))
        return r * n + M.indices.astype(np.int64), r

    ka, _ = keys(A)
    kb, rb = keys(B)
    pos = np.searchsorted(ka, kb)
    pos_c = np.minimum(pos, max(ka.size - 1, 0))
    hit = (pos < ka.size) & (ka[pos_c] == kb) if ka.size else np.zeros(kb.size, bool)
    av = np.where(hit, A.data[pos_c] if ka.size else 0.0, 0.0)
    extra = np.ones(ka.size, bool)
    extra[pos_c[hit]] = False
    assert not np.any(A.data[extra] != 0.0), "entries outside the reference pattern"
    absb = np.abs(B.data)
    rowmax = np.zeros(B.shape[0])
    np.maximum.at(rowmax, rb, absb)
    sel = (absb >= floor_rel * rowmax[rb]) & (absb > 0)
    err = np.abs(av - B.data)[sel] / absb[sel]
    frac = float((err > TOL_ENTRY).mean()) if err.size else 0.0
    return (float(err.max()) if err.size else 0.0), int(sel.sum()), frac


def vec_err(a, b, scale=None):
    """max |a-b| / max(|b|, scale) -- scale guards entries that cancel."""
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    s = np.abs(b) if scale is None else np.maximum(np.abs(b), scale)
    s = np.where(s == 0, 1.0, s)
    return float((np.abs(a - b) / s).max())


def gpu_device(g, material=None):
    """The same device on the GPU path (tcad_b200), BCs with the stored kappa."""
    import tcad_b200 as tb
    from tcad_b200.pack import Contact, Gate
    m = g["models"]
    mat = tb.Semiconductor(**(material or {}))
    models = tb.Models(doping_mobility=bool(m[0]), srh=bool(m[1]), auger=bool(m[2]),
                       bgn=bool(m[3]))
    if int(g["dim"]) == 2:
        dev = tb.Device2D(tb.Mesh2D(g["x"], g["y"]), g["doping"], Ntotal=g["Ntot"],
                          T=float(g["T"]), material=mat, models=models)
    else:
        dev = tb.Device3D(tb.Mesh3D(g["x"], g["y"], g["z"]), g["doping"],
                          Ntotal=g["Ntot"], T=float(g["T"]), material=mat, models=models)
    s = dev.setup
    for name, kind, k, v in bcs(g):
        if kind == "contact":
            dev.bcs[name] = Contact(k, v[0])
        else:
            idx = [np.asarray(a, dtype=np.int64) for a in unflat(g, k)]
            axis = "xyz"[int(v[3])] if int(g["dim"]) == 3 else None
            dev.bcs[name] = Gate(k, v[0], v[1], v[2], s.gate_weight(idx, axis), axis)
    dev._bcs_changed()
    return dev


def current_err(I, g, floor_frac=1e-9):
    """Relative distance of currents I to the reference's: the smaller of the
    distances to its converged state and to the other state of its Newton
    limit cycle (fixture key I_alt; equal to I where there is no cycle).
    Points with a current below floor_frac x the sweep's largest compare on
    that scale (the V = 0 point carries a round-off-level current)."""
    I = np.asarray(I, dtype=float)
    ref = np.asarray(g["I"], dtype=float)
    alt = np.asarray(g["I_alt"], dtype=float) if "I_alt" in g else ref
    scale = np.maximum(np.abs(ref), floor_frac * np.abs(ref).max())
    scale = np.where(scale == 0, 1.0, scale)
    return float((np.minimum(np.abs(I - ref), np.abs(I - alt)) / scale).max())


def oracle_from_device(dev):
    """The oracle device with the same set-up, contacts and gates as a
    tcad_b200 device (built by a workload builder)."""
    from oracle import OracleDevice, OracleModels
    s = dev.setup
    m = s.models
    mat = {k: getattr(s.mat, k) for k in s.mat.__dataclass_fields__ if k != "name"}
    ora = OracleDevice(s.coords, s.doping, Ntotal=s.Ntot, T=s.T,
                       models=OracleModels(m.doping_mobility, m.srh, m.auger, m.bgn),
                       material=mat)
    for name, b in dev.bcs.items():
        if b.kind == "contact":
            ora.contacts[name] = [b.nodes.copy(), b.V]
        else:
            ora.gates[name] = [b.nodes.copy(), b.kappa, b.Vfb, b.Vg, b.w.copy()]
    return ora


def field_errs(psi, n, p, psi_ref, n_ref, p_ref):
    """(max |dpsi|, max |d phi_n|, max |d phi_p|) in scaled units (x VT for
    volts): phi_n = psi - ln(n / nie), phi_p = psi + ln(p / nie), so the
    n_ie of the device cancels out of the differences."""
    psi, n, p = (np.asarray(a, float).ravel() for a in (psi, n, p))
    psi_ref, n_ref, p_ref = (np.asarray(a, float).ravel() for a in (psi_ref, n_ref, p_ref))
    dpsi = psi - psi_ref
    return (float(np.abs(dpsi).max()),
            float(np.abs(dpsi - (np.log(n) - np.log(n_ref))).max()),
            float(np.abs(dpsi + (np.log(p) - np.log(p_ref))).max()))


def current_noise(dev, contact, rel=4.4e-16, trials=8, seed=0, state=None):
    """How much of a terminal current the last bits of the state decide: the
    spread (max - min) of the contact's current over `trials` random
    relative perturbations of psi, n and p at the rounding level (each value
    times 1 + rel u, u uniform in [-1, 1]), evaluated by the device's own
    current sum on perturbed copies (the state is not touched); `state`: a
    (psi, n, p) of host arrays to use instead of the device's own.  At
    low-current points the current is a difference of contact fluxes many
    decades larger, so two solvers whose states agree to the last bits can
    still report currents this far apart (the 41x11 diode at 0.07 V: states
    within 4e-15, currents 7.7e-4 apart; the oracle's own sum at the GPU
    state gives the GPU's value)."""
    import torch
    pk = dev.pack
    g = torch.Generator(device=pk.device).manual_seed(seed)
    scale = dev.J0 * dev.LD ** dev._current_len_exp
    base = ((pk.psi, pk.n, pk.p) if state is None else
            [torch.as_tensor(np.asarray(a, float).ravel(), device=pk.device) for a in state])
    vals = []
    for _ in range(trials):
        pert = [t * (1.0 + rel * (2.0 * torch.rand(t.shape, generator=g, device=pk.device,
                                                   dtype=t.dtype) - 1.0))
                for t in base]
        vals.append(float(pk.contact_current(0, contact, *pert).item()) * scale)
    return max(vals) - min(vals)


def current_tol(I_ref, noise, rel=1e-6, floor=0.0):
    """Tolerance of a current comparison: rel x max(|I_ref|, floor), or ten
    times the current's rounding-level spread (current_noise) where that is
    larger."""
    return max(rel * max(abs(I_ref), floor), 10.0 * noise)
