"""The continuous-batching service (tcad_b200.serve): every request's result
is the one it gets alone, whether it shares rounds with other requests or
waits for arena room.  Alone means the drop-in Device2D/Device3D path on a
fresh device with the same options.  Tolerances: currents within 1e-6
relative, psi within 1e-9 V."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_I = 1e-6
TOL_PSI_V = 1e-9

MOS = [dict(nx=41, ny=17, Lg=60e-7, Na=3e17, Nsd_peak=5e19, Vg=0.9, Vd=0.6),
       dict(nx=29, ny=23, Lg=100e-7, Na=1e16, Nsd_peak=1e20, Vg=0.4, Vd=1.0),
       dict(nx=57, ny=12, Lg=35e-7, Na=1e18, Nsd_peak=1e19, Vg=1.1, Vd=0.2),
       dict(nx=33, ny=31, Lg=150e-7, Na=5e16, Nsd_peak=2e19, Vg=0.0, Vd=0.8)]


def _mosfet(q):
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    return W.mosfet2d(tb.Device2D, nx=q["nx"], ny=q["ny"], Lg=q["Lg"], Na=q["Na"],
                      Nsd_peak=q["Nsd_peak"])


def _cases():
    """(key, device builder, points, report, contact) of the mix: four
    single-bias MOSFET solves (3-step ramp), one warm-started Id-Vg sweep and
    one small tri-gate solve."""
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    out = []
    for i, q in enumerate(MOS):
        pts = W.ramp({"gate": q["Vg"], "drain": q["Vd"]}, 3)
        out.append((f"mos{i}", lambda q=q: _mosfet(q), pts, [False, False, True], "drain"))
    sweep = W.ramp({"drain": 0.5}, 2) + [{"gate": vg, "drain": 0.5}
                                         for vg in np.linspace(0.0, 0.8, 5)]
    out.append(("sweep", lambda: _mosfet(MOS[0]), sweep, [False, False] + [True] * 5,
                "drain"))
    tri = [W.trigate_bias(0.3, 0.4), W.trigate_bias(0.6, 0.8)]
    out.append(("tri", lambda: W.trigate3d(tb.Device3D, 24, 16, 12), tri, [False, True],
                "drain"))
    return out


def _alone(build, pts, report, contact, opts):
    dev = build()
    dev.solve_equilibrium()
    I = []
    for v, rep in zip(pts, report):
        dev.solve_bias(v, opts)
        assert dev.last_converged
        if rep:
            I.append(dev.terminal_current(contact))
    return np.array(I), dev.psi.copy(), dev.VT


def _check(reqs, ref):
    for r in reqs:
        assert r.error is None, r.error
        I, psi, VT = ref[r.key]
        assert all(r.converged)
        got = np.array(r.currents)
        assert np.all(np.abs(got - I) <= TOL_I * np.abs(I)), (r.key, got, I)
        assert np.abs(r.state[0] - psi).max() * VT < TOL_PSI_V, r.key


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_served_results_equal_alone(precision):
    import tcad_b200 as tb
    from tcad_b200.serve import Request, Server
    opts = tb.NewtonOptions(precision=precision)
    cases = _cases()
    ref = {key: _alone(build, pts, rep, c, opts) for key, build, pts, rep, c in cases}
    srv = Server(budget={2: 64 << 20, 3: 64 << 20}, opts=opts).start()
    try:
        reqs = []
        for j, (key, build, pts, rep, c) in enumerate(cases):
            reqs.append(srv.submit(Request(key, build().setup, pts, c, rep,
                                           return_state=True)))
            if j == 2:                 # the rest arrive while these are on the GPU
                time.sleep(0.05)
        assert srv.wait_idle(300)
        for r in reqs:
            assert r.done.is_set()
        _check(reqs, ref)
        w2 = srv.workers[2]
        assert w2.rounds >= 3 and max(e[2] for e in w2.round_log) >= 2
    finally:
        srv.stop()


def test_admission_waits_for_arena_room():
    """A 2D arena with room for about two of the MOSFETs: the others queue,
    are admitted as devices retire (idle ones are evicted), and still get
    their alone results."""
    import tcad_b200 as tb
    from tcad_b200.serve import Request, Server, bytes_per_node
    opts = tb.NewtonOptions()
    cases = [c for c in _cases() if c[0].startswith("mos")]
    ref = {key: _alone(build, pts, rep, c, opts) for key, build, pts, rep, c in cases}
    sizes = sorted(q["nx"] * q["ny"] for q in MOS)
    budget = (sizes[-1] + sizes[-2] + 64) * bytes_per_node(2)
    srv = Server(budget={2: budget}, opts=opts).start()
    try:
        reqs = [srv.submit(Request(key, build().setup, pts, c, rep, return_state=True))
                for key, build, pts, rep, c in cases]
        assert srv.wait_idle(300)
        _check(reqs, ref)
        w2 = srv.workers[2]
        assert max(e[2] for e in w2.round_log) <= 2
    finally:
        srv.stop()


def test_repeated_device_stays_resident():
    """A second request on the same device key reuses the resident arrays
    (no second upload of its coefficients) and restarts from equilibrium."""
    import tcad_b200 as tb
    from tcad_b200.serve import Request, Server
    from tcad_b200 import workloads as W
    opts = tb.NewtonOptions()
    q = MOS[1]
    pts = W.ramp({"gate": q["Vg"], "drain": q["Vd"]}, 3)
    ref = {"m": _alone(lambda: _mosfet(q), pts, [False, False, True], "drain", opts)}
    srv = Server(budget={2: 64 << 20}, opts=opts).start()
    try:
        setup = _mosfet(q).setup
        r1 = srv.submit(Request("m", setup, pts, "drain", [False, False, True],
                                return_state=True))
        assert srv.wait_idle(120)
        h1 = srv.workers[2].h2d_bytes
        r2 = srv.submit(Request("m", setup, pts, "drain", [False, False, True],
                                return_state=True))
        assert srv.wait_idle(120)
        _check([r1, r2], ref)
        grew = srv.workers[2].h2d_bytes - h1
        assert grew < 8 * setup.N * 2      # guess + bias values, not the coefficients
    finally:
        srv.stop()


def test_requests_sharing_a_setup_keep_their_own_bias():
    """Two requests on different keys built from ONE Setup object (a design
    served to two clients at once) are solved at their own biases."""
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    from tcad_b200.serve import Request, Server
    opts = tb.NewtonOptions()
    q = MOS[0]
    pa = W.ramp({"gate": 0.9, "drain": 0.6}, 3)
    pb = W.ramp({"gate": 0.3, "drain": 1.0}, 3)
    ref = {"a": _alone(lambda: _mosfet(q), pa, [False, False, True], "drain", opts),
           "b": _alone(lambda: _mosfet(q), pb, [False, False, True], "drain", opts)}
    setup = _mosfet(q).setup
    srv = Server(budget={2: 64 << 20}, opts=opts).start()
    try:
        ra = srv.submit(Request("a", setup, pa, "drain", [False, False, True],
                                return_state=True))
        rb = srv.submit(Request("b", setup, pb, "drain", [False, False, True],
                                return_state=True))
        assert srv.wait_idle(120)
        _check([ra, rb], ref)
    finally:
        srv.stop()


def test_served_requests_match_the_oracle():
    """One request of each kind served together -- a single-bias 2D MOSFET
    solve (3-step ramp), a warm-started 2D Id-Vg sweep, a small 3D tri-gate
    solve -- against the oracle's exact-Newton solutions of the same
    devices and bias points (update test 1e-12): every reported current
    within 1e-6 and the final psi within 1e-9 V."""
    import fixtures as fx
    import tcad_b200 as tb
    from tcad_b200.serve import Request, Server
    opts = tb.NewtonOptions()
    cases = [c for c in _cases() if c[0] in ("mos1", "sweep", "tri")]
    ref = {}
    for key, build, pts, rep, contact in cases:
        dev = build()
        ora = fx.oracle_from_device(dev)
        ora.solve_equilibrium(tol=1e-12)
        I = []
        for v, r_ in zip(pts, rep):
            ora.solve_bias(v, tol=1e-12)
            assert ora.last_converged, (key, v)
            if r_:
                I.append(ora.terminal_current(contact))
        ref[key] = (np.array(I), ora.psi.copy(), dev.VT)
    srv = Server(budget={2: 64 << 20, 3: 64 << 20}, opts=opts).start()
    try:
        reqs = [srv.submit(Request(key, build().setup, pts, contact, rep, return_state=True))
                for key, build, pts, rep, contact in cases]
        assert srv.wait_idle(timeout=300)
    finally:
        srv.stop()
    _check(reqs, ref)
