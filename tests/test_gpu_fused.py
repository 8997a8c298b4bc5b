"""The fused BiCGStab (one cooperative launch for a single-instance pack whose
flat blocks fit on the GPU at once) against the launch-per-step kernels: the
same block bodies and scalar updates in the same order, so solution,
iteration count, status and residual are bit-identical, and so is a whole
Newton sweep."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scaled_system(dev):
    """The device's block-scaled Newton system at its bulk-guess state."""
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
    _lib.check(pk.lib.tcad_block_jacobi_setup(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F),
                                              _lib.ptr(st), sp), "bj")
    assert int(st.item()) == _lib.TCAD_OK
    return pk


def _krylov(pk, fused, rtol=1e-10, maxit=4000):
    import torch
    from tcad_b200 import _lib
    lib = pk.lib
    prev = lib.tcad_set_krylov_fused(1 if fused else 0)
    try:
        x = torch.full_like(pk.du, float("nan"))
        it, st, rr = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_double(0.0)
        torch.cuda.synchronize()
        L0 = lib.tcad_launch_count()
        _lib.check(lib.tcad_block_krylov(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F), _lib.ptr(x),
                                         0, rtol, maxit, 0, _lib.ptr(pk.work), pk.work.numel(),
                                         ctypes.byref(it), ctypes.byref(st), ctypes.byref(rr),
                                         pk.sp()), "krylov")
        torch.cuda.synchronize()
        launches = lib.tcad_launch_count() - L0
    finally:
        lib.tcad_set_krylov_fused(prev)
    return x, it.value, st.value, rr.value, launches


def _devices():
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    return {"diode2d_201x101": lambda: W.diode2d(tb.Device2D, 201, 101),
            "mosfet2d_512x256": lambda: W.mosfet2d(tb.Device2D, 512, 256),
            "trigate3d_40x24x20": lambda: W.trigate3d(tb.Device3D, 40, 24, 20)}


@pytest.mark.parametrize("name", ["diode2d_201x101", "mosfet2d_512x256", "trigate3d_40x24x20"])
@pytest.mark.parametrize("rtol,maxit", [(1e-10, 4000), (1e-30, 60)])
def test_fused_bit_identical_to_per_step(name, rtol, maxit):
    from tcad_b200 import _lib
    pk = _scaled_system(_devices()[name]())
    xa, ita, sta, rra, La = _krylov(pk, False, rtol, maxit)
    xb, itb, stb, rrb, Lb = _krylov(pk, True, rtol, maxit)
    assert (ita, sta, rra) == (itb, stb, rrb)
    assert bool((xa == xb).all())
    assert Lb == 1 and La > 5                 # the fused solve is one launch
    if maxit == 60:
        assert sta == _lib.TCAD_ERR_NOCONV and ita == 60
    else:   # converged, or (block Jacobi on a hard start) out of iterations
        assert (sta == _lib.TCAD_OK and rra <= rtol) or \
            (sta == _lib.TCAD_ERR_NOCONV and ita == maxit)


def test_too_large_for_one_launch_runs_per_step():
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    pk = _scaled_system(W.diode2d(tb.Device2D, 601, 301))   # 354 flat blocks of 512
    x, it, st, rr, L = _krylov(pk, True, 1e-30, 8)
    assert L > 1 and it == 8


def test_newton_sweep_bit_identical():
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    lib = None
    states = []
    for fused in (False, True):
        dev = W.diode2d(tb.Device2D, 201, 101)
        lib = dev.pack.lib
        prev = lib.tcad_set_krylov_fused(1 if fused else 0)
        try:
            dev.solve_equilibrium()
            cur = []
            for v in (0.1, 0.2, 0.3):
                dev.solve_bias({"anode": v}, tb.NewtonOptions(krylov_system="full"))
                assert dev.last_converged
                cur.append(dev.terminal_current("anode"))
            states.append((dev.psi_gpu.clone(), dev.n_gpu.clone(), dev.p_gpu.clone(), cur))
        finally:
            lib.tcad_set_krylov_fused(prev)
    a, b = states
    for u, v in zip(a[:3], b[:3]):
        assert bool((u == v).all())
    assert a[3] == b[3]


def test_fused_give_up_falls_back_bit_identical():
    """The fused solve's failure path: with the test hook, the first grid
    barrier waits for an arrival that never comes until its 1 s limit runs
    out; the kernel returns, the host sees the flag and solves again with
    one launch per step.  The answer is the launch-per-step one bit for bit,
    and the GPU stays usable (the next fused solve succeeds)."""
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    pk = _scaled_system(W.diode2d(tb.Device2D, 201, 101))
    lib = pk.lib
    x0, it0, st0, rr0, _ = _krylov(pk, fused=False)
    g0 = lib.tcad_krylov_fused_gave_up()
    prev = lib.tcad_set_krylov_fused_test(1)
    try:
        x1, it1, st1, rr1, n1 = _krylov(pk, fused=True)
    finally:
        lib.tcad_set_krylov_fused_test(prev)
    assert lib.tcad_krylov_fused_gave_up() == g0 + 1
    assert n1 > 2                     # the fused launch, then the per-step launches
    assert (it1, st1) == (it0, st0) and rr1 == rr0
    assert np.array_equal(x1.cpu().numpy(), x0.cpu().numpy())
    x2, it2, st2, rr2, n2 = _krylov(pk, fused=True)
    assert n2 == 1 and lib.tcad_krylov_fused_gave_up() == g0 + 1
    assert np.array_equal(x2.cpu().numpy(), x0.cpu().numpy())
