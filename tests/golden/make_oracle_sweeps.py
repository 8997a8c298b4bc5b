"""Generate the oracle fixtures of the larger parity cases in this directory.

These cases are too many or too large to re-run on the reference's own
direct path inside a GPU test, so they are solved once here by the oracle
(``oracle/dd_oracle.py``, itself pinned bit-exact to the reference's
assembly and to its converged states by tests/test_oracle_golden.py) and
committed as small .npz files:

* ``mosfet_batch_oracle.npz`` -- eight instances of the seeded 512-MOSFET
  batch (tcad_b200.workloads.mosfet_batch_params, seed 2026): the smallest
  and largest meshes, the extreme body and source/drain dopings, the
  shortest gate and the highest bias; each from equilibrium through the
  same 4-step ramp (tcad_b200.workloads.ramp) as the batched GPU solve,
  Newton steps solved by SuperLU.

Every converged state is solved to the update test 1e-12 (a stock
NewtonOptions value, as for the reference-run sweep fixtures: at 1e-8 the
update test saturates at the 1e-10 density floor).  Each fixture holds the
terminal currents and (psi, n, p) at a seeded sample of nodes (the whole
fields would be several MB).

Usage:  python tests/golden/make_oracle_sweeps.py [mosfets]
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
BATCH_RAMP = 4


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


JOBS = {"mosfets": job_mosfets}


if __name__ == "__main__":
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    names = [a for a in sys.argv[1:] if a in JOBS] or list(JOBS)
    for name in names:
        JOBS[name]()
