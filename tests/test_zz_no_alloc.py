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
    """The 2D fixture device at its perturbed, biased state: assembled with
    the Dirichlet elimination, diagonal blocks inverted, rhs block-scaled."""
    import torch
    from tcad_b200 import _lib
    g = fx.load(name)
    dev = fx.gpu_device(g)
    pk = dev.pack
    psi, n, p = (dev._to_dev(g[k]) for k in ("st_psi", "st_n", "st_p"))
    pk.set_bias([{"right": float(g["V_right"])}])
    pk.assemble(_lib.MODE_ELIMINATE, psi, n, p)
    st = torch.zeros(1, dtype=torch.int32, device=pk.device)
    rc = pk.lib.tcad_block_jacobi_setup(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F),
                                        _lib.ptr(st), _lib.stream_ptr())
    assert rc == _lib.TCAD_OK and int(st.item()) == 0
    return dev, pk


def _results(ni):
    return ((ctypes.c_int32 * ni)(), (ctypes.c_int32 * ni)(), (ctypes.c_double * ni)())


def test_noalloc_matches_workspace_entry_point_twice():
    import torch
    from tcad_b200 import _lib
    dev, pk = _prepared()
    lib, sp = pk.lib, _lib.stream_ptr()
    rtol, maxiter = 1e-10, 4000
    # reference answer: the workspace entry point
    x_ref = torch.zeros_like(pk.du)
    it0, st0, rr0 = _results(1)
    rc = lib.tcad_block_krylov(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F), _lib.ptr(x_ref), 0,
                               rtol, maxiter, 0, _lib.ptr(pk.work), pk.work.numel(),
                               it0, st0, rr0, sp)
    assert rc == _lib.TCAD_OK and st0[0] == _lib.TCAD_OK
    ref = x_ref.cpu().numpy()
    assert np.isfinite(ref).all() and np.abs(ref).max() > 0
    for call in range(2):
        x = torch.full_like(pk.du, float("nan"))     # every entry must be written
        it, st, rr = _results(1)
        rc = lib.tcad_block_krylov_noalloc(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F),
                                           _lib.ptr(x), rtol, maxiter, it, st, rr, sp)
        torch.cuda.synchronize()
        assert rc == _lib.TCAD_OK, call
        assert st[0] == _lib.TCAD_OK and it[0] == it0[0], call
        got = x.cpu().numpy()
        assert np.abs(got - ref).max() <= TOL * np.abs(ref).max(), call
        assert abs(rr[0] - rr0[0]) <= TOL, call


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
