"""The allocation-free Krylov entry point against the workspace one.

tcad_block_krylov_noalloc serves callers that cannot allocate device memory
on demand (a serving process whose HBM is already owned by its own pool, a
cgo / JNI / N-API host without a device allocator, a loop that must not pay
cudaMalloc's device-wide synchronisation): its scratch is a fixed 5 MiB
device array inside the library.  Through the C ABI, two calls in a row must
give the answers of tcad_block_krylov (caller-provided workspace), and a pack
beyond the array's limit must be refused.  Kept in its own file so that it
runs after every other test.
"""
import ctypes

import numpy as np
import pytest

import fixtures as fx

pytestmark = pytest.mark.gpu

TOL = 1e-12   # the assembly-parity tolerance of the other GPU tests


def _prepared(name="asm2d"):
    """A fixture device at its perturbed, biased state: assembled with the
    Dirichlet elimination, diagonal blocks inverted, rhs block-scaled."""
    from tcad_b200 import _lib
    g = fx.load(name)
    dev = fx.gpu_device(g)
    pk = dev.pack
    psi, n, p = (dev._to_dev(g[k]) for k in ("st_psi", "st_n", "st_p"))
    volts = {"right": float(g["V_right"])} if "V_right" in g else \
        {"drain": float(g["V_drain"])}
    pk.set_bias([volts])
    pk.assemble(_lib.MODE_ELIMINATE, psi, n, p)
    _bj_setup(pk)
    return dev, pk


def _bj_setup(pk):
    import torch
    from tcad_b200 import _lib
    st = torch.zeros(pk.P.n_inst, dtype=torch.int32, device=pk.device)
    rc = pk.lib.tcad_block_jacobi_setup(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F),
                                        _lib.ptr(st), _lib.stream_ptr())
    assert rc == _lib.TCAD_OK and not st.any()


def _prepared_batch():
    """Two MOSFETs of different sizes in one pack, each at equilibrium with
    its own new bias stamped on its contacts: the first Newton system of a
    batched bias step, block-scaled."""
    import tcad_b200 as tb
    from tcad_b200 import _lib
    from tcad_b200 import workloads as W
    from tcad_b200.batch import DeviceBatch
    devs = [W.mosfet2d(tb.Device2D, nx=41, ny=17, Lg=60e-7),
            W.mosfet2d(tb.Device2D, nx=29, ny=23, Lg=100e-7, Na=1e16)]
    batch = DeviceBatch(devs)
    batch.solve_equilibrium()
    for d, v in zip(devs, ({"gate": 0.3, "drain": 0.1}, {"gate": 0.5, "drain": 0.2})):
        d._apply_voltages(v)
    pk = batch.pack
    pk.set_bias()
    pk.stamp_contacts()
    pk.assemble(_lib.MODE_ELIMINATE)
    _bj_setup(pk)
    return batch, pk


def _results(ni):
    return ((ctypes.c_int32 * ni)(), (ctypes.c_int32 * ni)(), (ctypes.c_double * ni)())


@pytest.mark.parametrize("case", ["asm2d", "asm3d", "batch2"])
def test_noalloc_matches_workspace_entry_point_twice(case):
    """2D and 3D single-device packs and a two-instance pack (per-instance
    reductions and their tickets): the answer of tcad_block_krylov, twice."""
    import torch
    from tcad_b200 import _lib
    _, pk = _prepared_batch() if case == "batch2" else _prepared(case)
    ni = pk.P.n_inst
    lib, sp = pk.lib, _lib.stream_ptr()
    rtol, maxiter = 1e-10, 4000
    # reference answer: the workspace entry point
    x_ref = torch.zeros_like(pk.du)
    it0, st0, rr0 = _results(ni)
    rc = lib.tcad_block_krylov(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F), _lib.ptr(x_ref), 0,
                               rtol, maxiter, 0, _lib.ptr(pk.work), pk.work.numel(),
                               it0, st0, rr0, sp)
    assert rc == _lib.TCAD_OK and all(st0[i] == _lib.TCAD_OK for i in range(ni))
    ref = x_ref.cpu().numpy()
    assert np.isfinite(ref).all() and np.abs(ref).max() > 0
    for call in range(2):
        x = torch.full_like(pk.du, float("nan"))     # every entry must be written
        it, st, rr = _results(ni)
        rc = lib.tcad_block_krylov_noalloc(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F),
                                           _lib.ptr(x), rtol, maxiter, it, st, rr, sp)
        torch.cuda.synchronize()
        assert rc == _lib.TCAD_OK, call
        for i in range(ni):
            assert st[i] == _lib.TCAD_OK and it[i] == it0[i], (call, i)
            assert abs(rr[i] - rr0[i]) <= TOL, (call, i)
        got = x.cpu().numpy()
        assert np.abs(got - ref).max() <= TOL * np.abs(ref).max(), call


def test_noalloc_refuses_packs_beyond_its_scratch():
    import tcad_b200 as tb
    from tcad_b200 import _lib
    x = np.linspace(0.0, 1e-4, 300)
    y = np.linspace(0.0, 1e-4, 120)          # 36,000 nodes > 32,768
    dev = tb.Device2D(tb.Mesh2D(x, y), np.full((120, 300), 1e17))
    pk = dev.pack
    it, st, rr = _results(1)
    rc = pk.lib.tcad_block_krylov_noalloc(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F),
                                          _lib.ptr(pk.du), 1e-10, 10, it, st, rr,
                                          _lib.stream_ptr())
    assert rc == _lib.TCAD_ERR_ARG


def test_noalloc_refuses_too_many_instances():
    """33 small devices: few nodes, but more instances than the scratch's
    per-instance tables hold (TCAD_STATIC_MAX_INST = 32)."""
    import tcad_b200 as tb
    from tcad_b200 import _lib
    from tcad_b200.batch import DeviceBatch
    x = np.linspace(0.0, 1e-5, 8)
    y = np.linspace(0.0, 1e-5, 6)
    devs = [tb.Device2D(tb.Mesh2D(x, y), np.full((6, 8), 1e17)) for _ in range(33)]
    pk = DeviceBatch(devs).pack
    assert pk.P.n_nodes <= 32768 and pk.P.n_inst == 33
    it, st, rr = _results(33)
    rc = pk.lib.tcad_block_krylov_noalloc(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F),
                                          _lib.ptr(pk.du), 1e-10, 10, it, st, rr,
                                          _lib.stream_ptr())
    assert rc == _lib.TCAD_ERR_ARG
