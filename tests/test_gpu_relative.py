"""The relative-unknown node-block-Jacobi set-up is the similarity transform
of the plain one: with S = diag(1, max(n, floor), max(p, floor)) per node,
A^_rel = S^-1 A^_abs S and b^_rel = S^-1 b^_abs (to rounding)."""
import numpy as np
import pytest

import fixtures as fx

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["asm2d", "asm3d"])
def test_relative_setup_is_similarity(name):
    import torch
    from tcad_b200 import _lib
    g = fx.load(name)
    dev = fx.gpu_device(g)
    pk = dev.pack
    psi, n, p = (dev._to_dev(g[k]) for k in ("st_psi", "st_n", "st_p"))
    volts = {"right": float(g["V_right"])} if "V_right" in g else \
        {"drain": float(g["V_drain"])}
    dev._apply_voltages(volts)
    pk.set_bias()
    pk.assemble(_lib.MODE_ELIMINATE, psi, n, p)
    J0, F0 = pk.J.clone(), pk.F.clone()
    st = torch.zeros(1, dtype=torch.int32, device=pk.device)
    sp = _lib.stream_ptr()
    Ja, Fa = J0.clone(), F0.clone()
    assert pk.lib.tcad_block_jacobi_setup(pk.pref, _lib.ptr(Ja), _lib.ptr(Fa), _lib.ptr(st),
                                          sp) == 0
    floor = 1e-10
    Jr, Fr = J0.clone(), F0.clone()
    assert pk.lib.tcad_block_jacobi_setup_rel(pk.pref, _lib.ptr(Jr), _lib.ptr(Fr),
                                              _lib.ptr(st), _lib.ptr(n), _lib.ptr(p), floor,
                                              sp) == 0
    assert int(st.item()) == 0
    N = pk.N
    S = torch.cat([torch.ones_like(n), n.clamp(min=floor), p.clamp(min=floor)])
    x = torch.randn(3 * N, dtype=torch.float64, device=pk.device)
    yr = torch.empty_like(x)
    ya = torch.empty_like(x)
    assert pk.lib.tcad_block_spmv(pk.pref, _lib.ptr(Jr), _lib.ptr(x), _lib.ptr(yr), sp) == 0
    Sx = S * x
    assert pk.lib.tcad_block_spmv(pk.pref, _lib.ptr(Ja), _lib.ptr(Sx), _lib.ptr(ya), sp) == 0
    want = (ya / S).cpu().numpy()
    got = yr.cpu().numpy()
    # the scaling is applied per stored entry, so rounding differs: compare
    # each component against that component's magnitude
    for c in range(3):
        sl = slice(c * N, (c + 1) * N)
        assert np.abs(got[sl] - want[sl]).max() <= 1e-12 * np.abs(want[sl]).max(), c
    bw = (Fa / S).cpu().numpy()
    bg = Fr.cpu().numpy()
    for c in range(3):
        sl = slice(c * N, (c + 1) * N)
        assert np.abs(bg[sl] - bw[sl]).max() <= 1e-13 * np.abs(bw[sl]).max(), c


@pytest.mark.parametrize("flat_nodes", [256, 512, 2048])
def test_flat_block_size_does_not_change_results(flat_nodes):
    """The flat-block size is a launch shape only: the SpMV is the same to
    the bit, whatever the size."""
    import torch
    from tcad_b200 import _lib
    from tcad_b200.pack import instance_tables
    g = fx.load("asm3d")
    dev = fx.gpu_device(g)
    pk = dev.pack
    pk.assemble(_lib.MODE_ELIMINATE, *(dev._to_dev(g[k]) for k in ("st_psi", "st_n", "st_p")))
    st = torch.zeros(1, dtype=torch.int32, device=pk.device)
    sp = _lib.stream_ptr()
    assert pk.lib.tcad_block_jacobi_setup(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F),
                                          _lib.ptr(st), sp) == 0
    x = torch.randn(3 * pk.N, dtype=torch.float64, device=pk.device)
    y0 = torch.empty_like(x)
    assert pk.lib.tcad_block_spmv(pk.pref, _lib.ptr(pk.J), _lib.ptr(x), _lib.ptr(y0), sp) == 0
    ax = np.zeros((1, 3), dtype=np.int64)
    pk._set_tables(instance_tables(pk.setups, pk.dim, [0], ax, tile_z=pk.tile_z,
                                   flat_nodes=flat_nodes))
    assert pk.n_flat == -(-pk.N // flat_nodes)
    y1 = torch.empty_like(x)
    assert pk.lib.tcad_block_spmv(pk.pref, _lib.ptr(pk.J), _lib.ptr(x), _lib.ptr(y1), sp) == 0
    assert torch.equal(y0, y1)
