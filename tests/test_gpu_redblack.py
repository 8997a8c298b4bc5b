"""BiCGStab on the red-black Schur complement of the block-scaled system
(tcad_block_krylov method 2, NewtonOptions.krylov_system="red_black"): the red
nodes, (i + j + k) even, are eliminated exactly, so the solve must meet the
full system's own stopping test ||b - A x|| <= rtol ||b||, and Newton sweeps
run on it must land on the oracle's results as the full-system path does --
2D and 3D, even and odd node counts along x (pad slots), single instances
and ragged batches."""
import ctypes
import contextlib

import numpy as np
import pytest

import fixtures as fx
from test_gpu_scale import _check_currents, _check_fields

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def _per_step(lib):
    """Single-instance packs small enough are solved in one cooperative
    launch; turning that off sends them through the per-step Schur loop."""
    prev = lib.tcad_set_krylov_fused(0)
    try:
        yield
    finally:
        lib.tcad_set_krylov_fused(prev)


def _scaled_system(dev):
    """The device's block-scaled Newton system at a biased bulk-guess state."""
    import torch
    from tcad_b200 import _lib
    pk = dev.pack
    s = dev.setup
    g = s.bulk_guess()
    pk.psi.copy_(dev._to_dev(g))
    pk.n.copy_(dev._to_dev(s.nie_s * np.exp(g)))
    pk.p.copy_(dev._to_dev(s.nie_s * np.exp(-g)))
    pk.set_bias()
    sp = pk.sp()
    _lib.check(pk.lib.tcad_sg_assemble(pk.pref, _lib.ptr(pk.psi), _lib.ptr(pk.n),
                                       _lib.ptr(pk.p), _lib.ptr(pk.F), _lib.ptr(pk.J),
                                       _lib.MODE_ELIMINATE, sp), "assemble")
    st = torch.zeros(1, dtype=torch.int32, device=pk.device)
    _lib.check(pk.lib.tcad_block_jacobi_setup_rel(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F),
                                                  _lib.ptr(st), _lib.ptr(pk.n),
                                                  _lib.ptr(pk.p), 1e-10, sp), "bj")
    assert int(st.item()) == _lib.TCAD_OK
    return pk


def _solve(pk, method, rtol, maxit):
    import torch
    from tcad_b200 import _lib
    x = torch.full_like(pk.du, float("nan"))
    it, st, rr = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_double(0.0)
    with _per_step(pk.lib):
        _lib.check(pk.lib.tcad_block_krylov(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F),
                                            _lib.ptr(x), method, rtol, maxit, 0,
                                            _lib.ptr(pk.work), pk.work.numel(),
                                            ctypes.byref(it), ctypes.byref(st),
                                            ctypes.byref(rr), pk.sp()), "krylov")
    torch.cuda.synchronize()
    return x, it.value, st.value, rr.value


def _true_relres(pk, x):
    import torch
    from tcad_b200 import _lib
    y = torch.empty_like(x)
    _lib.check(pk.lib.tcad_block_spmv(pk.pref, _lib.ptr(pk.J), _lib.ptr(x), _lib.ptr(y),
                                      pk.sp()), "spmv")
    torch.cuda.synchronize()
    return float(torch.linalg.norm(pk.F - y) / torch.linalg.norm(pk.F))


def _devices():
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    return {"diode2d_201x101": lambda: W.diode2d(tb.Device2D, 201, 101),
            "mosfet2d_128x64": lambda: W.mosfet2d(tb.Device2D, 128, 64),
            "trigate3d_40x24x20": lambda: W.trigate3d(tb.Device3D, 40, 24, 20),
            "trigate3d_41x23x19": lambda: W.trigate3d(tb.Device3D, 41, 23, 19)}


@pytest.mark.parametrize("name", ["diode2d_201x101", "mosfet2d_128x64", "trigate3d_40x24x20",
                                  "trigate3d_41x23x19"])
def test_schur_solve_meets_the_full_systems_test(name):
    """Method 2 converges to the full system's tolerance -- the reported and
    the independently recomputed ||b - A x|| / ||b|| -- and agrees with the
    full-system solve (method 0) to what that tolerance allows."""
    from tcad_b200 import _lib
    pk = _scaled_system(_devices()[name]())
    rtol = 1e-11
    x0, it0, st0, rr0 = _solve(pk, 0, rtol, 20000)
    x2, it2, st2, rr2 = _solve(pk, 2, rtol, 20000)
    assert st2 == _lib.TCAD_OK and rr2 <= rtol, (st2, rr2)
    assert _true_relres(pk, x2) <= 1.01 * rtol
    assert bool(x2.isfinite().all())
    if st0 == _lib.TCAD_OK:
        # both within rtol of the same system: their difference is the
        # operator's inverse applied to two residuals of at most rtol ||b||
        d = float((x2 - x0).abs().max() / x0.abs().max())
        assert d < 1e-5, d
        assert it2 < it0, (it2, it0)


def test_schur_solve_iteration_cap_reports_noconv():
    from tcad_b200 import _lib
    pk = _scaled_system(_devices()["trigate3d_40x24x20"]())
    x, it, st, rr = _solve(pk, 2, 1e-30, 40)
    assert st == _lib.TCAD_ERR_NOCONV and it == 40 and rr > 0.0
    assert bool(x.isfinite().all())


def test_other_methods_refused():
    import torch
    from tcad_b200 import _lib
    pk = _scaled_system(_devices()["diode2d_201x101"]())
    x = torch.zeros_like(pk.du)
    it, st, rr = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_double(0.0)
    for method in (1, 3):
        rc = pk.lib.tcad_block_krylov(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F), _lib.ptr(x),
                                      method, 1e-8, 10, 0, _lib.ptr(pk.work), pk.work.numel(),
                                      ctypes.byref(it), ctypes.byref(st), ctypes.byref(rr),
                                      pk.sp())
        assert rc == _lib.TCAD_ERR_ARG


def test_diode_c1_sweep_red_black():
    """The 201x101 diode sweep (odd Nx: pad slots) through the Schur solves,
    against the reference's currents and fields."""
    import tcad_b200 as tb
    g = fx.load("diode_c1")
    dev = fx.gpu_device(g, material=dict(tau_n0=1e-7, tau_p0=1e-7, tau_Nref=1e300))
    opts = tb.NewtonOptions(krylov_system="red_black")
    with _per_step(dev.pack.lib):
        dev.solve_equilibrium()
        I = []
        for V in g["V"]:
            dev.solve_bias({"anode": float(V)}, opts)
            assert dev.last_converged, V
            I.append(dev.terminal_current("anode"))
            tag = "%03d" % int(round(V * 100))
            if "psi_" + tag in g:
                assert np.abs(dev.psi.ravel() - g["psi_" + tag]).max() * dev.VT < 1e-9
    assert fx.current_err(I, g) < 1e-6


def test_pin_downscaled_sweep_red_black():
    """The 48 x 24 x 12 p-i-n sweep (the case whose low-bias currents need
    the polishing steps) through the Schur solves, against the oracle."""
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    g = fx.load("pin_ds")
    dev = W.pin3d(tb.Device3D, *(int(v) for v in g["shape"]))
    opts = tb.NewtonOptions(krylov_system="red_black")
    idx = g["idx"]
    I, noise = [], []
    with _per_step(dev.pack.lib):
        dev.solve_equilibrium()
        for k, V in enumerate(g["V"]):
            dev.solve_bias({"anode": float(V)}, opts)
            assert dev.last_converged, V
            I.append(dev.terminal_current("anode"))
            noise.append(fx.current_noise(dev, "anode"))
            st = [t.ravel()[idx] for t in (dev.psi, dev.n, dev.p)]
            _check_fields(dev.VT, st, g["fields"][k], V)
    _check_currents(I, g["I_anode"], noise)


def test_trigate_downscaled_batch_red_black():
    """Both tri-gate Vd branches (40 x 24 x 16) in one 2-instance pack through
    the Schur solves: every current within 1e-6 of the oracle's (on 1e-9 x
    the branch's largest terminal current)."""
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    from tcad_b200.batch import DeviceBatch
    g = fx.load("trigate_ds")
    shape = tuple(int(v) for v in g["shape"])
    opts = tb.NewtonOptions(krylov_system="red_black")
    b = DeviceBatch([W.trigate3d(tb.Device3D, *shape) for _ in W.TRIGATE_VD])
    b.solve_equilibrium(opts)
    cur = {c: np.zeros((2, len(W.TRIGATE_VG))) for c in ("drain", "source", "body")}
    for q, vg in enumerate(W.TRIGATE_VG):
        res = b.solve_bias([W.trigate_bias(vd, vg) for vd in W.TRIGATE_VD], opts)
        assert all(r["converged"] for r in res), vg
        for c in cur:
            cur[c][:, q] = b.terminal_currents(c)
    for a in range(2):
        top = max(np.abs(g["I_" + c][a]).max() for c in cur)
        for c in cur:
            ref = g["I_" + c][a]
            err = float((np.abs(cur[c][a] - ref) / np.maximum(np.abs(ref), 1e-9 * top)).max())
            assert err < 1e-6, (c, a, err)


def test_ragged_2d_batch_red_black_equals_alone():
    """Four MOSFETs of different odd Nx in one pack, node-block Jacobi with
    the Schur solves, against each device solved alone on the full system:
    psi within 1e-9 V, drain currents within 1e-6."""
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    from tcad_b200.batch import DeviceBatch
    from test_gpu_batch import PARAMS, _build
    full = tb.NewtonOptions(precond="block_jacobi")
    rb = tb.NewtonOptions(precond="block_jacobi", krylov_system="red_black")
    steps = 3
    alone_I, alone_psi = [], []
    for q in PARAMS:
        dev = _build(q)
        dev.solve_equilibrium()
        for volts in W.ramp({"gate": q["Vg"], "drain": q["Vd"]}, steps):
            dev.solve_bias(volts, full)
            assert dev.last_converged
        alone_I.append(dev.terminal_current("drain"))
        alone_psi.append(dev.psi.copy())
    batch = DeviceBatch([_build(q) for q in PARAMS])
    batch.solve_equilibrium()
    ramps = [W.ramp({"gate": q["Vg"], "drain": q["Vd"]}, steps) for q in PARAMS]
    for k in range(steps):
        res = batch.solve_bias([r[k] for r in ramps], rb)
        assert all(r["converged"] for r in res), k
    I = batch.terminal_currents("drain")
    for a in range(len(PARAMS)):
        assert abs(I[a] - alone_I[a]) <= 1e-6 * abs(alone_I[a]), (a, I[a], alone_I[a])
        assert np.abs(batch.state(a)[0] - alone_psi[a]).max() * batch.devices[a].VT < 1e-9


def _solve_counted(pk, method, rtol, maxit, fused):
    import torch
    from tcad_b200 import _lib
    lib = pk.lib
    prev = lib.tcad_set_krylov_fused(1 if fused else 0)
    try:
        x = torch.full_like(pk.du, float("nan"))
        it, st, rr = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_double(0.0)
        torch.cuda.synchronize()
        n0 = lib.tcad_launch_count()
        _lib.check(lib.tcad_block_krylov(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F), _lib.ptr(x),
                                         method, rtol, maxit, 0, _lib.ptr(pk.work),
                                         pk.work.numel(), ctypes.byref(it), ctypes.byref(st),
                                         ctypes.byref(rr), pk.sp()), "krylov")
        torch.cuda.synchronize()
        n = lib.tcad_launch_count() - n0
    finally:
        lib.tcad_set_krylov_fused(prev)
    return x, it.value, st.value, rr.value, n


@pytest.mark.parametrize("name", ["diode2d_201x101", "trigate3d_40x24x20", "trigate3d_41x23x19"])
@pytest.mark.parametrize("rtol,maxit", [(1e-10, 4000), (1e-30, 60)])
def test_schur_single_launch_bit_identical_to_per_step(name, rtol, maxit):
    """The red-black solve of a small single-instance pack in one
    cooperative launch (p and s formed on the fly by the red passes, five
    grid barriers per iteration) against its one-launch-per-step loop: the
    same bodies, scalar updates and reduction order, so solution, iteration
    count, status and residual are bit-identical."""
    pk = _scaled_system(_devices()[name]())
    xa, ita, sta, rra, na = _solve_counted(pk, 2, rtol, maxit, fused=False)
    xb, itb, stb, rrb, nb = _solve_counted(pk, 2, rtol, maxit, fused=True)
    assert (ita, sta, rra) == (itb, stb, rrb)
    assert np.array_equal(xa.cpu().numpy(), xb.cpu().numpy())
    assert nb == 2 and na > 10          # colour repack + the single launch


def test_schur_single_launch_give_up_falls_back():
    """With the test hook the single launch's first grid barrier runs out
    its time limit; the host solves again one launch per step, bit for bit
    the per-step answer, and the next single launch succeeds."""
    pk = _scaled_system(_devices()["trigate3d_40x24x20"]())
    lib = pk.lib
    x0, it0, st0, rr0, _ = _solve_counted(pk, 2, 1e-10, 4000, fused=False)
    g0 = lib.tcad_krylov_fused_gave_up()
    prev = lib.tcad_set_krylov_fused_test(1)
    try:
        x1, it1, st1, rr1, n1 = _solve_counted(pk, 2, 1e-10, 4000, fused=True)
    finally:
        lib.tcad_set_krylov_fused_test(prev)
    assert lib.tcad_krylov_fused_gave_up() == g0 + 1
    assert n1 > 3
    assert (it1, st1, rr1) == (it0, st0, rr0)
    assert np.array_equal(x1.cpu().numpy(), x0.cpu().numpy())
    x2, it2, st2, rr2, n2 = _solve_counted(pk, 2, 1e-10, 4000, fused=True)
    assert n2 == 2 and lib.tcad_krylov_fused_gave_up() == g0 + 1
    assert np.array_equal(x2.cpu().numpy(), x0.cpu().numpy())


def test_newton_sweep_single_launch_equals_per_step():
    """A whole 201x101 diode sweep with the red-black default: single
    launch and one launch per step give bit-identical states."""
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    states = []
    for fused in (False, True):
        dev = W.diode2d(tb.Device2D, 201, 101)
        lib = dev.pack.lib
        prev = lib.tcad_set_krylov_fused(1 if fused else 0)
        try:
            dev.solve_equilibrium()
            for v in (0.2, 0.4, 0.6):
                dev.solve_bias({"anode": v}, tb.NewtonOptions())
                assert dev.last_converged
            states.append([t.copy() for t in (dev.psi, dev.n, dev.p)])
        finally:
            lib.tcad_set_krylov_fused(prev)
    for a, b in zip(*states):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ["mosfet2d_128x64", "trigate3d_41x23x19"])
def test_equilibrium_pcg_red_black_matches_whole_system(name):
    """The equilibrium Newton with its PCG on the red-black Schur complement
    (the default) lands on the whole-system PCG's potential (within 1e-10 V)
    in fewer PCG iterations."""
    import tcad_b200 as tb
    res = {}
    for system in ("full", "red_black"):
        dev = _devices()[name]()
        dev.solve_equilibrium(tb.NewtonOptions(krylov_system=system))
        eq = dev.last_equilibrium
        assert eq["converged"], system
        res[system] = (dev.psi.copy(), eq["krylov_iters"], dev.VT)
    (pa, ka, vt), (pb, kb, _) = res["full"], res["red_black"]
    assert np.abs(pa - pb).max() * vt < 1e-10
    assert kb < ka, (kb, ka)


def test_equilibrium_pcg_red_black_batch_equals_alone():
    """Ragged 2D batch (odd Nx) equilibrium through the red-black PCG: each
    instance's potential equals its solo solve's within 1e-10 V."""
    import tcad_b200 as tb
    from tcad_b200.batch import DeviceBatch
    from test_gpu_batch import PARAMS, _build
    alone = []
    for q in PARAMS:
        dev = _build(q)
        dev.solve_equilibrium()
        alone.append(dev.psi.copy())
    b = DeviceBatch([_build(q) for q in PARAMS])
    b.solve_equilibrium()
    for a in range(len(PARAMS)):
        assert np.abs(b.state(a)[0] - alone[a]).max() * b.devices[a].VT < 1e-10
