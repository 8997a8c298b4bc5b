"""Block ILU(0) of the block-scaled 2D operator (tcad_block_ilu_setup /
tcad_block_ilu_apply, and NewtonOptions(precond="ilu")).

For the 5-point block stencil ILU(0) is exact in its pattern: the factor's
diagonal blocks are D~_k = I - G_k (B_kW Q_W G_W B_WE + B_kS Q_S G_S B_SN)
in natural order (G = stored inverse diagonal block, B = neighbour blocks,
Q = D~^-1).  The tests recompute that recursion on the host, check
M (M^-1 r) = r with M = (D~ + L^) D~^-1 (D~ + U^) built on the host, and run a
Newton sweep with the preconditioner against the reference's currents."""
import numpy as np
import pytest

import fixtures as fx

pytestmark = pytest.mark.gpu


def _nb(Jh, k, d):
    b = Jh[9 + 5 * d: 14 + 5 * d, k]
    B = np.zeros((3, 3))
    B[0, 0], B[1, 0], B[1, 1], B[2, 0], B[2, 2] = b
    return B


def test_ilu_factor_and_apply_match_host():
    import torch
    from tcad_b200 import _lib
    g = fx.load("asm2d")
    dev = fx.gpu_device(g)
    pk = dev.pack
    psi, n, p = (dev._to_dev(g[k]) for k in ("st_psi", "st_n", "st_p"))
    dev._apply_voltages({"right": float(g["V_right"])})
    pk.set_bias()
    pk.assemble(_lib.MODE_ELIMINATE, psi, n, p)
    st = torch.zeros(1, dtype=torch.int32, device=pk.device)
    sp = _lib.stream_ptr()
    assert pk.lib.tcad_block_jacobi_setup_rel(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F),
                                              _lib.ptr(st), _lib.ptr(n), _lib.ptr(p), 1e-10,
                                              sp) == 0
    N = pk.N
    assert pk.lib.tcad_block_ilu_bytes(pk.pref) == 9 * 8 * N
    Q = torch.zeros(9 * N, dtype=torch.float64, device=pk.device)
    assert pk.lib.tcad_block_ilu_setup(pk.pref, _lib.ptr(pk.J), _lib.ptr(Q), _lib.ptr(st),
                                       sp) == 0
    assert int(st.item()) == 0
    r = torch.randn(3 * N, dtype=torch.float64, device=pk.device)
    out = torch.zeros_like(r)
    assert pk.lib.tcad_block_ilu_apply(pk.pref, _lib.ptr(pk.J), _lib.ptr(Q), _lib.ptr(r),
                                       _lib.ptr(out), sp) == 0
    Jh = pk.J.cpu().numpy().reshape(-1, N)
    Qg = Q.cpu().numpy().reshape(9, N)
    nx, ny = dev.setup.nax[0], dev.setup.nax[1]
    G = [Jh[0:9, k].reshape(3, 3) for k in range(N)]
    Qh = [None] * N
    Dt = [None] * N
    for j in range(ny):
        for i in range(nx):
            k = j * nx + i
            S = np.zeros((3, 3))
            if i > 0:
                m = k - 1
                S += _nb(Jh, k, 0) @ Qh[m] @ G[m] @ _nb(Jh, m, 1)
            if j > 0:
                m = k - nx
                S += _nb(Jh, k, 2) @ Qh[m] @ G[m] @ _nb(Jh, m, 3)
            Dt[k] = np.eye(3) - G[k] @ S
            Qh[k] = np.linalg.inv(Dt[k])
    Qh_arr = np.stack([q.ravel() for q in Qh], axis=1)
    assert np.abs(Qg - Qh_arr).max() <= 1e-10 * np.abs(Qh_arr).max()
    # M (M^-1 r) = r
    x = out.cpu().numpy().reshape(3, N).T
    u = np.zeros_like(x)
    for j in range(ny):
        for i in range(nx):
            k = j * nx + i
            t = np.zeros(3)
            if i < nx - 1:
                t += _nb(Jh, k, 1) @ x[k + 1]
            if j < ny - 1:
                t += _nb(Jh, k, 3) @ x[k + nx]
            u[k] = Dt[k] @ x[k] + G[k] @ t
    v = np.stack([Qh[k] @ u[k] for k in range(N)])
    w = np.zeros_like(v)
    for j in range(ny):
        for i in range(nx):
            k = j * nx + i
            t = np.zeros(3)
            if i > 0:
                t += _nb(Jh, k, 0) @ v[k - 1]
            if j > 0:
                t += _nb(Jh, k, 2) @ v[k - nx]
            w[k] = Dt[k] @ v[k] + G[k] @ t
    rh = r.cpu().numpy().reshape(3, N).T
    assert np.abs(w - rh).max() <= 1e-9 * np.abs(rh).max()


def _apply_M_host(Jh, Qg, x, nx, ny):
    """M x = (D~ + L^) D~^-1 (D~ + U^) x, vectorised over nodes (x: [N, 3])."""
    N = nx * ny
    G = Jh[0:9].T.reshape(N, 3, 3)
    Q = Qg.T.reshape(N, 3, 3)
    Dt = np.linalg.inv(Q)

    def nbmat(d):
        b = Jh[9 + 5 * d: 14 + 5 * d].T
        B = np.zeros((N, 3, 3))
        B[:, 0, 0], B[:, 1, 0], B[:, 1, 1], B[:, 2, 0], B[:, 2, 2] = b.T
        return B

    idx = np.arange(N).reshape(ny, nx)
    def shift(v, di, dj):       # value of node (i+di, j+dj), zero outside
        out = np.zeros_like(v)
        vv = v.reshape(ny, nx, 3)
        oo = out.reshape(ny, nx, 3)
        oo[max(0, -dj):ny - max(0, dj), max(0, -di):nx - max(0, di)] = \
            vv[max(0, dj):ny - max(0, -dj), max(0, di):nx - max(0, -di)]
        return out
    mv = lambda A, v: np.einsum("nij,nj->ni", A, v)  # noqa: E731
    u = mv(Dt, x) + mv(G, mv(nbmat(1), shift(x, 1, 0)) + mv(nbmat(3), shift(x, 0, 1)))
    v = mv(Q, u)
    return mv(Dt, v) + mv(G, mv(nbmat(0), shift(v, -1, 0)) + mv(nbmat(2), shift(v, 0, -1)))


@pytest.mark.parametrize("shape", [(64, 40), (300, 270)])
def test_ilu_apply_inverts_M(shape):
    """M (M^-1 r) = r on a MOSFET at a biased Newton state; (300, 270) has
    anti-diagonals longer than a block (the general sweep), (64, 40) the
    register-pipelined one."""
    import torch
    import tcad_b200 as tb
    from tcad_b200 import _lib, workloads as W
    dev = W.mosfet2d(tb.Device2D, *shape, Lg=60e-7)
    dev.solve_equilibrium()
    dev._apply_voltages({"gate": 0.6, "drain": 0.4})
    pk = dev.pack
    pk.set_bias()
    pk.stamp_contacts()
    pk.assemble(_lib.MODE_ELIMINATE)
    st = torch.zeros(1, dtype=torch.int32, device=pk.device)
    sp = _lib.stream_ptr()
    assert pk.lib.tcad_block_jacobi_setup_rel(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F),
                                              _lib.ptr(st), _lib.ptr(pk.n), _lib.ptr(pk.p),
                                              1e-10, sp) == 0
    N = pk.N
    Q = torch.zeros(9 * N, dtype=torch.float64, device=pk.device)
    assert pk.lib.tcad_block_ilu_setup(pk.pref, _lib.ptr(pk.J), _lib.ptr(Q), _lib.ptr(st),
                                       sp) == 0
    assert int(st.item()) == 0
    r = torch.randn(3 * N, dtype=torch.float64, device=pk.device)
    out = torch.zeros_like(r)
    assert pk.lib.tcad_block_ilu_apply(pk.pref, _lib.ptr(pk.J), _lib.ptr(Q), _lib.ptr(r),
                                       _lib.ptr(out), sp) == 0
    Jh = pk.J.cpu().numpy().reshape(-1, N)
    x = out.cpu().numpy().reshape(3, N).T
    w = _apply_M_host(Jh, Q.cpu().numpy().reshape(9, N), x, *shape)
    rh = r.cpu().numpy().reshape(3, N).T
    assert np.abs(w - rh).max() <= 1e-6 * np.abs(rh).max()   # rounding: kappa(M) ~ 1e10


def test_ilu_newton_sweep_parity_and_fewer_iterations():
    import tcad_b200 as tb
    g = fx.load("mosfet_small")
    res = {}
    for pc in ("block_jacobi", "ilu"):
        dev = fx.gpu_device(g)
        dev.solve_equilibrium()
        opts = tb.NewtonOptions(precond=pc)
        I, kr = [], 0
        for v in g["Vg"]:
            dev.solve_bias({"drain": float(g["Vd"]), "gate": float(v)}, opts)
            assert dev.last_converged
            I.append(dev.terminal_current("drain"))
            kr += dev.last_newton["krylov_iters"]
        assert fx.current_err(I, g) < 1e-6, pc
        res[pc] = kr
    assert res["ilu"] < res["block_jacobi"]


def test_ilu_3d_planes_invert_their_blocks():
    """On a 3D pack ILU(0) is taken per z-plane (in-plane couplings): M is
    block-diagonal over planes and M (M^-1 r) = r holds plane by plane."""
    import torch
    import tcad_b200 as tb
    from tcad_b200 import _lib, workloads as W
    dev = W.trigate3d(tb.Device3D, 24, 16, 12)
    dev.solve_equilibrium()
    dev._apply_voltages(W.trigate_bias(0.3, 0.5))
    pk = dev.pack
    pk.set_bias()
    pk.stamp_contacts()
    pk.assemble(_lib.MODE_ELIMINATE)
    st = torch.zeros(1, dtype=torch.int32, device=pk.device)
    sp = _lib.stream_ptr()
    assert pk.lib.tcad_block_jacobi_setup_rel(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F),
                                              _lib.ptr(st), _lib.ptr(pk.n), _lib.ptr(pk.p),
                                              1e-10, sp) == 0
    N = pk.N
    Q = torch.zeros(9 * N, dtype=torch.float64, device=pk.device)
    assert pk.lib.tcad_block_ilu_setup(pk.pref, _lib.ptr(pk.J), _lib.ptr(Q), _lib.ptr(st),
                                       sp) == 0
    assert int(st.item()) == 0
    r = torch.randn(3 * N, dtype=torch.float64, device=pk.device)
    out = torch.zeros_like(r)
    assert pk.lib.tcad_block_ilu_apply(pk.pref, _lib.ptr(pk.J), _lib.ptr(Q), _lib.ptr(r),
                                       _lib.ptr(out), sp) == 0
    nx, ny, nz = dev.setup.nax
    Jh = pk.J.cpu().numpy().reshape(-1, N)
    Qh = Q.cpu().numpy().reshape(9, N)
    x = out.cpu().numpy().reshape(3, N).T
    rh = r.cpu().numpy().reshape(3, N).T
    P = nx * ny
    for z in range(nz):
        sl = slice(z * P, (z + 1) * P)
        w = _apply_M_host(Jh[:, sl], Qh[:, sl], x[sl], nx, ny)
        assert np.abs(w - rh[sl]).max() <= 1e-8 * np.abs(rh).max(), z


def test_ilu_3d_newton_sweep_parity():
    import tcad_b200 as tb
    g = fx.load("trigate_small")
    dev = fx.gpu_device(g)
    dev.solve_equilibrium()
    opts = tb.NewtonOptions(precond="ilu")
    gates = [b for b in dev.bcs if b.startswith("gate")]
    I = []
    for v in g["Vg"]:
        dev.solve_bias({"drain": float(g["Vd"]), **{gt: float(v) for gt in gates}}, opts)
        assert dev.last_converged
        I.append(dev.terminal_current("drain"))
    assert fx.current_err(I, g) < 1e-6
