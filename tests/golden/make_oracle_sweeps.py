"""Generate the oracle fixtures of the larger parity cases in this directory.

These cases are too many or too large to re-run on the reference's own
direct path inside a GPU test, so they are solved once here by the oracle
(``oracle/dd_oracle.py``, itself pinned bit-exact to the reference's
assembly and to its converged states by tests/test_oracle_golden.py) and
committed as small .npz files:

* ``trigate_ds.npz`` -- the tri-gate Id-Vg workload (tcad_b200.workloads.
  trigate3d) down-scaled to 40 x 24 x 16 nodes (15,360; the bench's --small
  size): equilibrium, then Vg = 0 .. 1.0 V in 0.05 V steps at Vd = 0.05 V and
  at Vd = 0.7 V, each sweep from equilibrium (pytcad/finfet3d.py:246-263);
* ``pin_ds.npz`` -- the p-i-n forward sweep (tcad_b200.workloads.pin3d,
  SRH + Auger, doping mobility) down-scaled to 48 x 24 x 12 nodes: 0 .. 0.9 V
  in 0.1 V steps;
* ``mosfet_batch_oracle.npz`` -- eight instances of the seeded 512-MOSFET
  batch (tcad_b200.workloads.mosfet_batch_params, seed 2026): the smallest
  and largest meshes, the extreme body and source/drain dopings, the
  shortest gate and the highest bias; each from equilibrium through the
  same 4-step ramp (tcad_b200.workloads.ramp) as the batched GPU solve,
  Newton steps solved by SuperLU;
* ``trigate_mid.npz`` -- the tri-gate at 64 x 40 x 28 (71,680 nodes), the
  down-scaled size of the headline sweep: equilibrium, then Vg = 0 and
  0.05 V at Vd = 0.05 V and Vg = 0 at Vd = 0.7 V, each branch from
  equilibrium -- three points, not a sweep: a coupled Newton step took
  ~12 minutes here (equilibrium 5 min; the three points 1.0, 1.2 and 2.6 h
  with two branches in parallel).

The sweep meshes are the largest whose sweeps the oracle's direct solves finish
in minutes per point on one host core: a SuperLU factorisation of the coupled
3D system grows from 0.5 s at 3,840 nodes to about a minute at 30k and
several minutes at the 71,680-node 64 x 40 x 28 mesh,
where a 42-point sweep would take days.

Every converged state is solved to the update test 1e-12 (a stock
NewtonOptions value, as for the reference-run sweep fixtures: at 1e-8 the
update test saturates at the 1e-10 density floor).  Each fixture holds the
terminal currents and (psi, n, p) at a seeded sample of nodes (the whole
fields would be several MB).

Usage:  python tests/golden/make_oracle_sweeps.py [mosfets] [trigate] [pin] [trigate_mid]
"""
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

TOL = 1e-12
N_SAMPLE_2D = 512
N_SAMPLE_3D = 1024
BATCH_RAMP = 4
TRIGATE_SHAPE = (40, 24, 16)
TRIGATE_FIELD_POINTS = (0, 4, 8, 12, 16, 20)   # Vg indices whose fields are stored
PIN_SHAPE = (48, 24, 12)


def _log(msg):
    print(f"[{time.strftime('%H:%M:%S')}] {msg}", flush=True)


def sample_nodes(N, count, seed):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(N, size=min(count, N), replace=False)).astype(np.int64)


def _oracle(dev):
    import fixtures as fx
    return fx.oracle_from_device(dev)


def _fields(ora, idx):
    return (ora.psi.ravel()[idx].copy(), ora.n.ravel()[idx].copy(),
            ora.p.ravel()[idx].copy())


def batch_selection(params):
    """Indices of the batch instances the fixture covers."""
    size = np.array([q["nx"] * q["ny"] for q in params])
    na = np.array([q["Na"] for q in params])
    npk = np.array([q["Nsd_peak"] for q in params])
    lg = np.array([q["Lg"] for q in params])
    vv = np.array([q["Vg"] + q["Vd"] for q in params])
    pick = [int(size.argmin()), int(size.argmax()), int(na.argmin()), int(na.argmax()),
            int(npk.argmin()), int(npk.argmax()), int(lg.argmin()), int(vv.argmax())]
    out = []
    for k in pick:
        if k not in out:
            out.append(k)
    return out


def job_mosfet(i):
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    q = W.mosfet_batch_params(512)[i]
    dev = W.mosfet2d(tb.Device2D, nx=q["nx"], ny=q["ny"], Lg=q["Lg"], Na=q["Na"],
                     Nsd_peak=q["Nsd_peak"])
    ora = _oracle(dev)
    idx = sample_nodes(ora.N, N_SAMPLE_2D, 1000 + i)
    t = time.time()
    ora.solve_equilibrium()
    steps = 0
    for volts in W.ramp({"gate": q["Vg"], "drain": q["Vd"]}, BATCH_RAMP):
        ora.solve_bias(volts, tol=TOL)
        steps += ora.newton_iters
    conv = bool(ora.last_converged)
    _log(f"mosfet {i} ({q['nx']}x{q['ny']}): {steps} steps, {time.time() - t:.1f} s, "
         f"converged={conv}")
    return dict(i=i, idx=idx, I_drain=ora.terminal_current("drain"),
                I_source=ora.terminal_current("source"), fields=np.stack(_fields(ora, idx)),
                converged=conv, steps=steps)


def job_mosfets():
    from tcad_b200 import workloads as W
    sel = batch_selection(W.mosfet_batch_params(512))
    with mp.get_context("spawn").Pool(min(4, len(sel))) as pool:
        res = pool.map(job_mosfet, sel)
    n = max(r["idx"].size for r in res)
    idx = np.full((len(res), n), -1, dtype=np.int64)
    fields = np.zeros((len(res), 3, n))
    for a, r in enumerate(res):
        idx[a, :r["idx"].size] = r["idx"]
        fields[a, :, :r["idx"].size] = r["fields"]
    np.savez_compressed(os.path.join(HERE, "mosfet_batch_oracle.npz"), tol=TOL,
                        inst=np.array([r["i"] for r in res]), idx=idx, fields=fields,
                        I_drain=np.array([r["I_drain"] for r in res]),
                        I_source=np.array([r["I_source"] for r in res]),
                        converged=np.array([r["converged"] for r in res]),
                        steps=np.array([r["steps"] for r in res]), ramp=BATCH_RAMP)


def job_trigate(vd_index):
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    dev = W.trigate3d(tb.Device3D, *TRIGATE_SHAPE)
    ora = _oracle(dev)
    idx = sample_nodes(ora.N, N_SAMPLE_3D, 402416)
    t = time.time()
    ora.solve_equilibrium()
    _log(f"trigate equilibrium {time.time() - t:.1f} s ({ora.eq_iters} steps)")
    psi_eq = ora.psi.ravel()[idx].copy()
    vd = W.TRIGATE_VD[vd_index]
    I = {c: [] for c in ("drain", "source", "body")}
    F, iters = [], []
    for q, vg in enumerate(W.TRIGATE_VG):
        t = time.time()
        ora.solve_bias(W.trigate_bias(vd, vg), tol=TOL)
        assert ora.last_converged, (vd, vg)
        for c in I:
            I[c].append(ora.terminal_current(c))
        iters.append(ora.newton_iters)
        if q in TRIGATE_FIELD_POINTS:
            F.append(np.stack(_fields(ora, idx)))
        _log(f"trigate Vd={vd} Vg={vg}: {ora.newton_iters} steps, {time.time() - t:.1f} s, "
             f"Id={I['drain'][-1]:.9e}")
    return dict(idx=idx, psi_eq=psi_eq, I_drain=np.array(I["drain"]),
                I_source=np.array(I["source"]), I_body=np.array(I["body"]),
                fields=np.array(F), iters=np.array(iters))


def job_trigate_both():
    from tcad_b200 import workloads as W
    with mp.get_context("spawn").Pool(2) as pool:
        a, b = pool.map(job_trigate, [0, 1])
    assert np.array_equal(a["idx"], b["idx"])
    np.savez_compressed(
        os.path.join(HERE, "trigate_ds.npz"), shape=np.array(TRIGATE_SHAPE), tol=TOL,
        Vg=np.array(W.TRIGATE_VG), Vd=np.array(W.TRIGATE_VD), idx=a["idx"],
        psi_eq=a["psi_eq"], field_points=np.array(TRIGATE_FIELD_POINTS),
        **{k: np.stack([a[k], b[k]]) for k in ("I_drain", "I_source", "I_body", "fields",
                                               "iters")})


def job_pin():
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    dev = W.pin3d(tb.Device3D, *PIN_SHAPE)
    ora = _oracle(dev)
    idx = sample_nodes(ora.N, N_SAMPLE_3D, 482412)
    t = time.time()
    ora.solve_equilibrium(tol=TOL)
    _log(f"pin equilibrium {time.time() - t:.1f} s ({ora.eq_iters} steps)")
    psi_eq = ora.psi.ravel()[idx].copy()
    I, F, iters = [], [], []
    for V in W.PIN_SWEEP:
        t = time.time()
        ora.solve_bias({"anode": V}, tol=TOL)
        assert ora.last_converged, V
        I.append(ora.terminal_current("anode"))
        iters.append(ora.newton_iters)
        F.append(np.stack(_fields(ora, idx)))
        _log(f"pin V={V}: {ora.newton_iters} steps, {time.time() - t:.1f} s, I={I[-1]:.9e}")
    np.savez_compressed(os.path.join(HERE, "pin_ds.npz"), shape=np.array(PIN_SHAPE), tol=TOL,
                        idx=idx, psi_eq=psi_eq, V=np.array(W.PIN_SWEEP), I_anode=np.array(I),
                        fields=np.array(F), iters=np.array(iters))


MID_SHAPE = (64, 40, 28)
MID_POINTS = {0: [0.0, 0.05], 1: [0.0]}    # Vd index -> Vg values, from equilibrium


def job_trigate_mid_branch(vd_index):
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    dev = W.trigate3d(tb.Device3D, *MID_SHAPE)
    ora = _oracle(dev)
    idx = sample_nodes(ora.N, N_SAMPLE_3D, 642816)
    t = time.time()
    ora.solve_equilibrium()
    _log(f"trigate-mid equilibrium {time.time() - t:.1f} s ({ora.eq_iters} steps)")
    psi_eq = ora.psi.ravel()[idx].copy()
    vd = W.TRIGATE_VD[vd_index]
    out = []
    for vg in MID_POINTS[vd_index]:
        t = time.time()
        ora.solve_bias(W.trigate_bias(vd, vg), tol=TOL)
        assert ora.last_converged, (vd, vg)
        out.append(dict(vd=vd, vg=vg, I_drain=ora.terminal_current("drain"),
                        I_source=ora.terminal_current("source"),
                        I_body=ora.terminal_current("body"),
                        fields=np.stack(_fields(ora, idx)), iters=ora.newton_iters))
        _log(f"trigate-mid Vd={vd} Vg={vg}: {ora.newton_iters} steps, {time.time() - t:.1f} s, "
             f"Id={out[-1]['I_drain']:.9e}")
    return dict(idx=idx, psi_eq=psi_eq, points=out)


def job_trigate_mid():
    """The tri-gate at 64 x 40 x 28 (71,680 nodes; a SuperLU step takes
    minutes here): equilibrium, then the first points of each Vd branch."""
    with mp.get_context("spawn").Pool(2) as pool:
        a, b = pool.map(job_trigate_mid_branch, [0, 1])
    assert np.array_equal(a["idx"], b["idx"])
    pts = a["points"] + b["points"]
    np.savez_compressed(
        os.path.join(HERE, "trigate_mid.npz"), shape=np.array(MID_SHAPE), tol=TOL,
        idx=a["idx"], psi_eq=a["psi_eq"], vd=np.array([q["vd"] for q in pts]),
        vg=np.array([q["vg"] for q in pts]),
        I_drain=np.array([q["I_drain"] for q in pts]),
        I_source=np.array([q["I_source"] for q in pts]),
        I_body=np.array([q["I_body"] for q in pts]),
        fields=np.stack([q["fields"] for q in pts]), iters=np.array([q["iters"] for q in pts]))


JOBS = {"mosfets": job_mosfets, "trigate": job_trigate_both, "pin": job_pin,
        "trigate_mid": job_trigate_mid}


if __name__ == "__main__":
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    names = [a for a in sys.argv[1:] if a in JOBS] or [j for j in JOBS if j != "trigate_mid"]
    for name in names:
        JOBS[name]()
