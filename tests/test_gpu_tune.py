"""The launch-shape autotuner (tcad_b200.tune): the 3D tile depth and the
plane staging it picks change which CTA evaluates a node and where its
coefficients are read from, never the arithmetic, so the assembled
residual/Jacobian and a whole Newton solve are bit-identical at every
setting."""
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


@pytest.mark.parametrize("biased", [False, True])
def test_assembly_bit_identical_at_every_depth_and_staging(biased):
    """Every (depth, staging) pair, at the bulk guess and at a biased,
    perturbed state with gates on (the staged west/south halo copies, the
    last-plane empty copy group and the z-edges at the top plane included)."""
    from tcad_b200 import workloads as W
    dev = _device()
    pk = _bulk_state(dev)
    if biased:
        dev._apply_voltages(W.trigate_bias(0.7, 0.6))
        pk.set_bias()
        g = pk.psi.clone()
        w = dev._to_dev(np.sin(np.arange(dev.N) * 0.37))
        pk.psi.copy_(g + 0.2 * w)
        pk.n.mul_(1.0 + 0.3 * w)
        pk.p.mul_(1.0 - 0.3 * w)
    ref = None
    for st in (0, 1):
        pk.set_asm_stage(st)
        for tz in (1, 2, 3, 8, 16):
            pk.set_tile_z(tz)
            F, J = _assemble(pk)
            if ref is None:
                ref = (F, J)
            else:
                assert bool((F == ref[0]).all()) and bool((J == ref[1]).all()), (tz, st)


def test_tuner_picks_a_candidate_and_caches_it():
    from tcad_b200 import tune
    tune.clear()
    pk = _bulk_state(_device())
    best = tune.tune_assembly(pk)
    assert best[0] in tune.CANDIDATES and best[1] in tune.STAGES
    assert (pk.tile_z, pk.asm_stage) == best
    assert set(tune.last_timings) == {(tz, st) for tz in tune.CANDIDATES for st in tune.STAGES}
    assert all(t > 0.0 for t in tune.last_timings.values())
    tune.last_timings.clear()
    pk2 = _bulk_state(_device())
    assert tune.tune_assembly(pk2) == best and (pk2.tile_z, pk2.asm_stage) == best
    assert not tune.last_timings          # served from the cache, nothing re-measured


def test_newton_solve_bit_identical_at_two_settings():
    import tcad_b200 as tb
    from tcad_b200 import workloads as W
    states = []
    for tz, stg in ((1, 0), (8, 1)):
        dev = _device()
        dev.pack.autotune = False
        dev.pack.set_tile_z(tz)
        dev.pack.set_asm_stage(stg)
        dev.solve_equilibrium()
        dev.solve_bias(W.trigate_bias(0.05, 0.4), tb.NewtonOptions())
        assert dev.last_converged
        states.append((dev.psi_gpu.clone(), dev.n_gpu.clone(), dev.p_gpu.clone()))
    for a, b in zip(*states):
        assert bool((a == b).all())
