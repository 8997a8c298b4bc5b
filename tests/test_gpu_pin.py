"""The 3D p-i-n workload (SRH + Auger, doping mobility, erfc junctions) on a
small mesh against the oracle: equilibrium and a forward sweep, psi within
1e-9 V, quasi-Fermi levels within 1e-8 V, anode currents within 1e-6."""
import numpy as np
import pytest

import fixtures as fx

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pin3d_small_sweep_matches_oracle(precision):
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    dev = W.pin3d(tb.Device3D, 20, 6, 5)
    ora = fx.oracle_from_device(dev)
    ora.solve_equilibrium(tol=1e-12)
    dev.solve_equilibrium()
    VT = dev.VT
    assert np.abs(dev.psi.ravel() - ora.psi.ravel()).max() * VT < 1e-9
    opts = tb.NewtonOptions(precision=precision)
    for V in (0.1, 0.2, 0.3, 0.4, 0.5):
        ora.solve_bias({"anode": V}, tol=1e-12)
        dev.solve_bias({"anode": V}, opts)
        assert dev.last_converged, V
        assert np.abs(dev.psi.ravel() - ora.psi.ravel()).max() * VT < 1e-9, V
        nie = dev.nie_s.ravel()
        for c, sgn in (("n", -1.0), ("p", 1.0)):
            mine = dev.psi.ravel() + sgn * np.log(getattr(dev, c).ravel() / nie)
            ref = ora.psi.ravel() + sgn * np.log(getattr(ora, c).ravel() / nie)
            assert np.abs(mine - ref).max() * VT < 1e-8, (V, c)
        I, Iref = dev.terminal_current("anode"), ora.terminal_current("anode")
        assert abs(I - Iref) <= 1e-6 * abs(Iref), (V, I, Iref)
