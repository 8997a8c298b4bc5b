"""The per-instance tables every kernel launch trusts (tcad_b200.pack): flat
blocks of one instance each, sized to the instance, and stencil tiles that
cover every node of every instance exactly once at any tile depth -- the
depth the tuner re-tiles with included.  Pure numpy, no GPU."""
from types import SimpleNamespace as NS

import numpy as np
import pytest

from tcad_b200 import _lib
from tcad_b200.pack import instance_tables, instance_tiles, secant_ratio

MESHES_3D = [(40, 24, 20), (33, 9, 7), (64, 8, 1), (1, 1, 3), (97, 17, 16)]
MESHES_2D = [(201, 101), (33, 9), (1, 1), (64, 40)]


def _setups(shapes):
    mat = NS(Cn_auger=2.8e-31, Cp_auger=9.9e-32)
    models = NS(srh=True, auger=False)
    return [NS(nax=s, N=int(np.prod(s)), Ns=1e18, R0=1.0, mat=mat, models=models)
            for s in shapes]


@pytest.mark.parametrize("dim,shapes", [(3, MESHES_3D), (2, MESHES_2D)])
@pytest.mark.parametrize("flat_nodes", [512, 256, 1000])
def test_flat_blocks_never_straddle_instances(dim, shapes, flat_nodes):
    st = _setups(shapes)
    tb = _tables(st, dim, flat_nodes=flat_nodes)
    off, inst = tb["flat_off"], tb["flat_inst"]
    assert off[0] == 0 and np.all(np.diff(off) >= 1)
    for i, s in enumerate(st):
        nb = off[i + 1] - off[i]
        assert nb == -(-s.N // flat_nodes)                       # ceil(N / flat_nodes)
        assert np.all(inst[off[i]:off[i + 1]] == i)
    assert inst.size == off[-1]


def _tables(st, dim, tile_z=1, flat_nodes=None):
    node_off = np.concatenate(([0], np.cumsum([s.N for s in st])[:-1]))
    return instance_tables(st, dim, node_off, np.zeros((len(st), 3), np.int64),
                           tile_z=tile_z, flat_nodes=flat_nodes)


@pytest.mark.parametrize("tile_z", [1, 2, 3, 4, 8, 16])
def test_tiles_cover_every_node_once(tile_z):
    st = _setups(MESHES_3D)
    tb = _tables(st, 3, tile_z=tile_z)
    assert tb["tile_z"] == tile_z
    tl = tb["tile"].reshape(-1, 4)
    for i, s in enumerate(st):
        nx, ny, nz = s.nax
        hits = np.zeros((nz, ny, nx), np.int32)
        for _, i0, j0, k0 in tl[tl[:, 0] == i]:
            assert k0 % tile_z == 0 and i0 % _lib.TILE_X == 0 and j0 % _lib.TILE_Y == 0
            hits[k0:k0 + tile_z, j0:j0 + _lib.TILE_Y, i0:i0 + _lib.TILE_X] += 1
        assert np.all(hits == 1), (s.nax, tile_z)


def test_instance_tiles_2d_ignore_depth():
    s = NS(nax=(64, 40), N=64 * 40)
    assert np.array_equal(instance_tiles(s, 2, 1), instance_tiles(s, 2, 8))
    assert np.all(instance_tiles(s, 2, 8)[:, 2] == 0)


def test_secant_ratio_only_for_parallel_steps():
    a, b = np.array([0.0, 0.1]), np.array([0.0, 0.2])
    assert secant_ratio(a, b, np.array([0.0, 0.3])) == pytest.approx(1.0)
    assert secant_ratio(a, b, np.array([0.0, 0.25])) == pytest.approx(0.5)
    assert secant_ratio(a, b, np.array([0.1, 0.3])) == 0.0          # not parallel
    assert secant_ratio(a, b, np.array([0.0, 0.1])) == 0.0          # reversal
    assert secant_ratio(a, b, np.array([0.0, 0.6])) == 0.0          # beyond smax = 2
    assert secant_ratio(None, b, np.array([0.0, 0.3])) == 0.0
