"""Small-signal AC on the GPU Jacobian against the reference's own
y_parameters (pytcad/ac2d.py:237-342; fixture tests/golden/ac_small.npz: the
small 2D MOSFET biased on at Vd = 0.5 V, Vg = 0.8 V, four ports -- source,
drain, body, gate -- at 1 Hz .. 100 GHz).  The DC point is solved on the GPU
from equilibrium with the default options; Y must agree entry by entry
within 1e-6 of the larger of |Y_ij| and 1e-6 x the largest entry at that
frequency.  The floor covers the body row at 1 Hz: ~1e-11 against ~100, a
sum of contact fluxes that cancel, where a Krylov solve to 1e-12 leaves
~2e-11 and the reference's own SuperLU round-off is of that order too."""
import numpy as np
import pytest

import fixtures as fx

pytestmark = pytest.mark.gpu


def _device(g):
    dev = fx.gpu_device(g)
    dev.solve_equilibrium()
    dev.solve_bias({"drain": float(g["Vd"]), "gate": float(g["Vg"])})
    assert dev.last_converged
    return dev


def test_y_parameters_match_reference():
    from tcad_b200.ac import y_parameters
    g = fx.load("ac_small")
    dev = _device(g)
    assert np.abs(dev.psi.ravel() - g["psi_dc"]).max() * dev.VT < 1e-9
    r = y_parameters(dev, g["freqs"])
    assert list(r.port_names) == [str(p) for p in g["ports"]]
    Yref = g["Y"]
    for kf in range(Yref.shape[0]):
        for i in range(Yref.shape[1]):
            scale = np.maximum(np.abs(Yref[kf, i]), 1e-6 * np.abs(Yref[kf]).max())
            err = np.abs(r.Y[kf, i] - Yref[kf, i]) / scale
            assert err.max() < 1e-6, (g["freqs"][kf], i, err)


def test_y_parameters_low_frequency_is_the_dc_conductance():
    """At 1 Hz the ohmic-port Y is the DC small-signal conductance: the
    drain row's derivative w.r.t. the drain voltage, by a central
    difference of GPU terminal currents (+-1 mV), within the difference's
    own truncation error."""
    from tcad_b200.ac import y_parameters
    g = fx.load("ac_small")
    dev = _device(g)
    r = y_parameters(dev, [1.0])
    ports = list(r.port_names)
    i_d = ports.index("drain")
    Vd, Vg = float(g["Vd"]), float(g["Vg"])
    I = []
    for dv in (-1e-3, 1e-3):
        dev.solve_bias({"drain": Vd + dv, "gate": Vg})
        I.append(dev.terminal_current("drain"))
    gdd = (I[1] - I[0]) / 2e-3
    assert abs(r.Y[0, i_d, i_d].real - gdd) <= 1e-4 * abs(gdd)
