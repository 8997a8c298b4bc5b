"""GPU linsolve.solve_linear against scipy's direct solve, following the
reference's own gates (tests/test_m22_linsolve.py G3-G6 and the block-Jacobi
exactness pin)."""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.linalg import spsolve

import fixtures as fx

pytestmark = pytest.mark.gpu


def _random_spd_system(n, seed):
    rng = np.random.default_rng(seed)
    A = sp.random(n, n, density=min(1.0, 5.0 / n), random_state=rng,
                  data_rvs=lambda k: rng.standard_normal(k)).tocsr()
    A = A + A.T
    A = A + sp.diags(np.abs(A).sum(axis=1).A1 + 1.0)
    return A.tocsr(), rng.standard_normal(n)


@pytest.mark.parametrize("method", ["gmres", "bicgstab"])
def test_iterative_agrees_with_direct(method):
    from tcad_b200 import solve_linear
    for n, seed in ((30, 10), (300, 11), (2001, 12)):
        A, b = _random_spd_system(n, seed)
        ref = spsolve(A.tocsc(), b)
        x, info = solve_linear(A, b, method=method, rtol=1e-10)
        assert info["converged"] and info["method"] == method
        assert np.linalg.norm(x - ref) / np.linalg.norm(ref) <= 1e-6
        x3, info3 = solve_linear(A, b, method=method, rtol=1e-10, block_size=3)
        assert np.linalg.norm(x3 - ref) / np.linalg.norm(ref) <= 1e-6
        assert info3["precond"] == ("block_jacobi" if n % 3 == 0 else "jacobi")


@pytest.mark.parametrize("method", ["gmres", "bicgstab"])
def test_device_jacobian(method):
    """A real coupled device Jacobian (the 2D fixture, eliminated)."""
    from tcad_b200 import solve_linear
    from oracle import eliminate_csr
    g = fx.load("asm2d")
    dev = fx.gpu_device(g)
    F, J, *_ = dev._residual_jacobian(g["st_psi"], g["st_n"], g["st_p"],
                                      {"right": float(g["V_right"])})
    Jd, rhs = eliminate_csr(J, -F, dev._dirichlet_rows)
    ref = spsolve(Jd.tocsc(), rhs)
    x, info = solve_linear(Jd, rhs, method=method, rtol=1e-10, block_size=3)
    assert info["converged"]
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) <= 1e-6


def test_non_convergence_raises():
    from tcad_b200 import solve_linear, LinearSolveError
    n = 200
    rng = np.random.default_rng(99)
    A = sp.random(n, n, density=0.05, random_state=rng,
                  data_rvs=lambda k: rng.standard_normal(k)).tocsr()
    A = A + sp.eye(n) * 1e-3
    b = rng.standard_normal(n)
    for method in ("gmres", "bicgstab"):
        with pytest.raises(LinearSolveError):
            solve_linear(A, b, method=method, rtol=1e-14, maxiter=1)


def test_singular_and_non_finite_raise():
    from tcad_b200 import solve_linear, LinearSolveError
    A = sp.csr_matrix((10, 10))
    for method in ("gmres", "bicgstab", "direct"):
        with pytest.raises(LinearSolveError):
            solve_linear(A, np.ones(10), method=method)
    A2, b2 = _random_spd_system(10, 1)
    b2[3] = np.nan
    with pytest.raises(LinearSolveError):
        solve_linear(A2, b2, method="gmres")
    with pytest.raises(ValueError):
        solve_linear(A2, np.ones(10), method="cholesky")


def test_block_jacobi_exact_on_block_diagonal():
    """With exact node-block inverses, a block-diagonal system is solved by
    the first preconditioned step (the reference pins the apply to 1e-10)."""
    from tcad_b200 import solve_linear
    rng = np.random.default_rng(3)
    nb = 200
    blocks = [rng.standard_normal((3, 3)) * 3 + np.eye(3) * 10.0 for _ in range(nb)]
    A = sp.block_diag(blocks, format="csr")
    b = rng.standard_normal(3 * nb)
    x, info = solve_linear(A, b, method="bicgstab", rtol=1e-12, block_size=3)
    ref = np.concatenate([np.linalg.solve(B, b[3 * k:3 * k + 3]) for k, B in enumerate(blocks)])
    assert np.abs(x - ref).max() < 1e-10
    assert info["iterations"] <= 1


def test_block_jacobi_unsticks_coupled_3d_jacobian():
    """The reference's G6 pin (test_m22_linsolve.py:301-331): the 21^3 coupled
    Jacobian converges with GMRES + node-block-Jacobi in < 100 iterations."""
    import tcad_b200 as tb
    from tcad_b200 import solve_linear
    n = 20
    m = np.linspace(0.0, 2.0e-4, n + 1)
    dev = tb.Device3D(tb.Mesh3D(m, m, m), np.full((n + 1,) * 3, 1e16),
                      models=tb.Models(srh=False))
    jj, kk = np.meshgrid(np.arange(n + 1), np.arange(n + 1))
    jj, kk = jj.ravel(), kk.ravel()
    dev.add_contact("l", np.zeros_like(jj), jj, kk, V=0.0)
    dev.add_contact("r", np.full_like(jj, n), jj, kk, V=0.1)
    dev.solve_equilibrium()
    F, J, *_ = dev._residual_jacobian(dev.psi, dev.n, dev.p, {"r": 0.1})
    x, info = solve_linear(J, -F, method="gmres", rtol=1e-8, maxiter=500, block_size=3)
    assert info["converged"] and info["iterations"] < 100
