"""The launch-shape autotuner (tcad_b200.tune): the 3D tile depth it picks
changes which CTA evaluates a node, never the arithmetic, so the assembled
residual/Jacobian and a whole Newton solve are bit-identical at every depth."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device():
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    return W.trigate3d(tb.Device3D, 40, 24, 20)


def _bulk_state(dev):
    pk = dev.pack
    s = dev.setup
    g = s.bulk_guess()
    pk.psi.copy_(dev._to_dev(g))
    pk.n.copy_(dev._to_dev(s.nie_s * np.exp(g)))
    pk.p.copy_(dev._to_dev(s.nie_s * np.exp(-g)))
    pk.set_bias()
    return pk


def _assemble(pk):
    from tcad_b200 import _lib
    rc = pk.lib.tcad_sg_assemble(pk.pref, _lib.ptr(pk.psi), _lib.ptr(pk.n), _lib.ptr(pk.p),
                                 _lib.ptr(pk.F), _lib.ptr(pk.J), _lib.MODE_ELIMINATE, pk.sp())
    _lib.check(rc, "tcad_sg_assemble")
    return pk.F.clone(), pk.J.clone()


def test_assembly_bit_identical_at_every_depth():
    pk = _bulk_state(_device())
    ref = None
    for tz in (1, 2, 3, 8, 16):
        pk.set_tile_z(tz)
        F, J = _assemble(pk)
        if ref is None:
            ref = (F, J)
        else:
            assert bool((F == ref[0]).all()) and bool((J == ref[1]).all()), tz


def test_tuner_picks_a_candidate_and_caches_it():
    from tcad_b200 import tune
    tune.clear()
    pk = _bulk_state(_device())
    best = tune.tune_tile_z(pk)
    assert best in tune.CANDIDATES and pk.tile_z == best
    assert set(tune.last_timings) == set(tune.CANDIDATES)
    assert all(t > 0.0 for t in tune.last_timings.values())
    tune.last_timings.clear()
    pk2 = _bulk_state(_device())
    assert tune.tune_tile_z(pk2) == best and pk2.tile_z == best
    assert not tune.last_timings          # served from the cache, nothing re-measured


def test_newton_solve_bit_identical_at_two_depths():
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    states = []
    for tz in (1, 8):
        dev = _device()
        dev.pack.autotune = False
        dev.pack.set_tile_z(tz)
        dev.solve_equilibrium()
        dev.solve_bias(W.trigate_bias(0.05, 0.4), tb.NewtonOptions())
        assert dev.last_converged
        states.append((dev.psi_gpu.clone(), dev.n_gpu.clone(), dev.p_gpu.clone()))
    for a, b in zip(*states):
        assert bool((a == b).all())
