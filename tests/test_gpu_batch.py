"""Packed batches: every instance's result equals its result solved alone
(psi within 1e-9 V, currents within 1e-6 relative), for uneven instance
sizes and per-instance biases, in FP64 and mixed precision."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PARAMS = [dict(nx=41, ny=17, Lg=60e-7, Na=3e17, Nsd_peak=5e19, Vg=0.9, Vd=0.6),
          dict(nx=29, ny=23, Lg=100e-7, Na=1e16, Nsd_peak=1e20, Vg=0.4, Vd=1.0),
          dict(nx=57, ny=12, Lg=35e-7, Na=1e18, Nsd_peak=1e19, Vg=1.1, Vd=0.2),
          dict(nx=33, ny=31, Lg=150e-7, Na=5e16, Nsd_peak=2e19, Vg=0.0, Vd=0.8)]


def _build(q):
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    return W.mosfet2d(tb.Device2D, nx=q["nx"], ny=q["ny"], Lg=q["Lg"], Na=q["Na"],
                      Nsd_peak=q["Nsd_peak"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_alone(precision):
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    from tcad_b200.batch import DeviceBatch
    opts = tb.NewtonOptions(precision=precision)
    steps = 3
    alone_I, alone_psi = [], []
    for q in PARAMS:
        dev = _build(q)
        dev.solve_equilibrium()
        for volts in W.ramp({"gate": q["Vg"], "drain": q["Vd"]}, steps):
            dev.solve_bias(volts, opts)
            assert dev.last_converged
        alone_I.append(dev.terminal_current("drain"))
        alone_psi.append(dev.psi.copy())
    batch = DeviceBatch([_build(q) for q in PARAMS])
    batch.solve_equilibrium()
    ramps = [W.ramp({"gate": q["Vg"], "drain": q["Vd"]}, steps) for q in PARAMS]
    for s in range(steps):
        res = batch.solve_bias([r[s] for r in ramps], opts)
        assert all(r["converged"] for r in res)
    I = batch.terminal_currents("drain")
    for i, q in enumerate(PARAMS):
        psi = batch.state(i)[0]
        VT = batch.devices[i].VT
        assert np.abs(psi - alone_psi[i]).max() * VT < 1e-9
        assert abs(I[i] - alone_I[i]) <= 1e-6 * abs(alone_I[i])


def test_batch_mask_keeps_inactive_state():
    """An instance masked out of a solve keeps its state bit for bit."""
    import tcad_b200 as tb
    from tcad_b200.batch import DeviceBatch
    batch = DeviceBatch([_build(q) for q in PARAMS[:2]])
    batch.solve_equilibrium()
    before = [t.copy() for t in batch.state(1)]
    res = batch.solve_bias([{"gate": 0.5, "drain": 0.1}, {"gate": 0.5, "drain": 0.1}],
                           tb.NewtonOptions(), active=[1, 0])
    assert res[0]["converged"]
    after = batch.state(1)
    for a, b in zip(before, after):
        assert np.array_equal(a, b)


def test_gate_bias_upload_matches_setup():
    """set_bias recomputes V/VT - Vfb/VT on the gate nodes alone and
    scatters it: the device array equals the full-mesh host recomputation
    bit for bit, including nodes under two gates (the tri-gate corners)."""
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    from tcad_b200.pack import Pack
    devs = [_build(PARAMS[0]), W.trigate3d(tb.Device3D, 24, 16, 12)]
    for d, volts in ((devs[0], {"gate": 0.7}),
                     (devs[1], {"gate_top": 0.3, "gate_left": 0.8, "gate_right": 0.55})):
        pk = Pack([d.setup])
        d._apply_voltages(volts)
        pk.set_bias()
        want = d.setup.gate_arrays()[2]
        assert np.array_equal(pk.t["gate_v"].cpu().numpy(), want)
        assert pk.last_h2d_bytes < 8 * d.N / 4


def test_batch_matches_oracle():
    """Eight instances of the seeded 512-MOSFET batch (the smallest and
    largest meshes, the extreme dopings, the shortest gate, the highest
    bias) solved in ONE pack through the same 4-step ramp from equilibrium
    as the oracle's exact-Newton run (tests/golden/mosfet_batch_oracle.npz,
    made by tests/golden/make_oracle_sweeps.py): every instance's drain
    current within 1e-6, psi within 1e-9 V and the quasi-Fermi levels within
    1e-8 V at the fixture's sampled nodes."""
    import fixtures as fx
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    from tcad_b200.batch import DeviceBatch
    g = fx.load("mosfet_batch_oracle")
    params = W.mosfet_batch_params(512)
    sel = [params[int(i)] for i in g["inst"]]
    batch = DeviceBatch([_build(q) for q in sel])
    opts = tb.NewtonOptions()
    batch.solve_equilibrium(opts)
    steps = int(g["ramp"])
    ramps = [W.ramp({"gate": q["Vg"], "drain": q["Vd"]}, steps) for q in sel]
    for s in range(steps):
        res = batch.solve_bias([r[s] for r in ramps], opts)
    assert all(r["converged"] for r in res)
    I = batch.terminal_currents("drain")
    rel = np.abs(I - g["I_drain"]) / np.abs(g["I_drain"])
    assert rel.max() < 1e-6, rel
    for a in range(len(sel)):
        idx = g["idx"][a]
        idx = idx[idx >= 0]
        st = [t.ravel()[idx] for t in batch.state(a)]
        ref = g["fields"][a][:, :idx.size]
        e_psi, e_n, e_p = fx.field_errs(*st, *ref)
        VT = batch.devices[a].VT
        assert e_psi * VT < 1e-9, (a, e_psi * VT)
        assert max(e_n, e_p) * VT < 1e-8, (a, e_n * VT, e_p * VT)
