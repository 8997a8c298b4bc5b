"""Oracle parity at the headline size: the coupled SG assembly of the full
160 x 96 x 64 tri-gate (983,040 nodes, 38M Jacobian entries; the bench's
default workload) on the GPU against the oracle's assembly of the same device
and state (oracle/dd_oracle.py, pinned bit-exact to the reference's assembly
by tests/test_oracle_golden.py).  Every tile, the measured tile depth and the
1,920 flat blocks of the full mesh are covered, which the small fixtures do
not reach.

Two states: the equilibrium the GPU solves, at zero bias; and a perturbed
state (smooth +-0.3 potential, +-50 % densities) at Vd = 0.7 V, Vg = 0.6 V.
Bar: the Jacobian within 1e-12 relative entry by entry and per row, the
residual within 1e-12 per row on its natural scale (|J| |x| + |F|)."""
import numpy as np
import pytest

import fixtures as fx

pytestmark = pytest.mark.gpu

TOL_ASM = 1e-12


def _rownorm_vec(F, J, x, Fref):
    scale = np.asarray(abs(J) @ np.abs(x)).ravel() + np.abs(Fref)
    scale = np.where(scale == 0, 1.0, scale)
    return float((np.abs(F - Fref) / scale).max())


def _states(dev):
    s = dev.setup
    psi = dev.psi.copy()
    n = s.nie_s * np.exp(psi)
    p = s.nie_s * np.exp(-psi)
    yield psi, n, p, {}
    zz, yy, xx = np.meshgrid(*(np.linspace(0.0, 1.0, m) for m in s.shape), indexing="ij")
    w = np.sin(7.0 * xx + 3.0 * yy) * np.cos(5.0 * zz + 1.0)
    yield (psi + 0.3 * w, n * (1.0 + 0.5 * w), p * (1.0 - 0.5 * w),
           {"drain": 0.7, "gate_top": 0.6, "gate_left": 0.6, "gate_right": 0.6})


def test_trigate_full_mesh_assembly():
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    dev = W.trigate3d(tb.Device3D)
    assert dev.N == 160 * 96 * 64
    dev.solve_equilibrium()
    assert dev.last_equilibrium["converged"]
    for psi, n, p, volts in _states(dev):
        dev._apply_voltages(volts)
        out = dev._residual_jacobian(psi, n, p, {k: v for k, v in volts.items()
                                                 if k in ("drain", "source", "body")})
        F, J, F_n, F_p = out[0], out[1], out[-2], out[-1]
        ora = fx.oracle_from_device(dev)
        Fo, Jo, Fno, Fpo = ora.residual_jacobian(psi, n, p, {k: v for k, v in volts.items()
                                                             if k in ora.contacts})
        assert np.array_equal(np.sort(dev._dirichlet_rows), np.sort(ora.fixed))
        e_elem, n_cmp = fx.elem_err(J, Jo)
        assert n_cmp == np.count_nonzero(Jo.data) and e_elem < TOL_ASM, (e_elem, n_cmp)
        assert fx.rownorm_err(J, Jo) < TOL_ASM
        x = np.stack([psi.ravel(), n.ravel(), p.ravel()], axis=1).ravel()
        assert _rownorm_vec(F, Jo, x, Fo) < TOL_ASM
        for mine, ref in ((F_n.ravel(), Fno.ravel()), (F_p.ravel(), Fpo.ravel())):
            assert fx.vec_err(mine, ref, 1e-12 * np.abs(ref).max()) < 1e-10
        del out, F, J, Fo, Jo
