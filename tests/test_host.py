"""CPU tests: host-side set-up and the C ABI (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

import fixtures as fx

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("name", ["asm2d", "asm3d", "trigate_small", "mosfet_small"])
def test_setup_matches_oracle_bitwise(name):
    """The coefficient arrays handed to the kernels equal the oracle's (and
    hence the reference's) bit for bit."""
    from tcad_b200.pack import Setup
    import tcad_b200 as tb
    g = fx.load(name)
    ora = fx.oracle_device(g)
    m = g["models"]
    s = Setup(fx.coords(g), g["doping"], Ntotal=g["Ntot"], T=float(g["T"]),
              models=tb.Models(doping_mobility=bool(m[0]), srh=bool(m[1]),
                               auger=bool(m[2]), bgn=bool(m[3])))
    for a in ("Ns", "LD", "J0", "R0", "VT"):
        assert getattr(s, a) == getattr(ora, a), a
    for a in ("C", "nie", "nie_s", "tau_n", "tau_p"):
        assert np.array_equal(getattr(s, a), getattr(ora, a)), a
    for ax in range(s.dim):
        assert np.array_equal(s.h[ax], ora.h[ax]) and np.array_equal(s.dv[ax], ora.dv[ax])
        lo = s.lo(ax)
        assert np.array_equal(s.an[ax][lo], ora.an[ax])
        assert np.array_equal(s.ap[ax][lo], ora.ap[ax])
        assert np.array_equal(s.dl[ax][lo], ora.dlnnie[ax])
        hi_edge = [slice(None)] * s.dim
        hi_edge[s.arr_axis(ax)] = -1
        assert not s.an[ax][tuple(hi_edge)].any()


def test_contact_table_matches_ohmic_values():
    from tcad_b200.pack import Setup
    import tcad_b200 as tb
    from oracle import ohmic_values
    g = fx.load("trigate_small")
    s = Setup(fx.coords(g), g["doping"], Ntotal=g["Ntot"], models=tb.Models())
    from tcad_b200.pack import Contact
    for name, kind, k, v in fx.bcs(g):
        if kind == "contact":
            s.bcs[name] = Contact(k, 0.3)
    names, nodes, cid, L, n0, p0 = s.contact_table()
    psi0, on0, op0 = ohmic_values(s.C.ravel()[nodes], s.nie_s.ravel()[nodes], 0.3, s.VT)
    assert np.array_equal(0.3 / s.VT + L, psi0)
    assert np.array_equal(n0, on0) and np.array_equal(p0, op0)


def test_refuses_unimplemented_models():
    import tcad_b200 as tb
    with pytest.raises(NotImplementedError):
        tb.Models(fd=True).require_gpu_path()
    with pytest.raises(NotImplementedError):
        tb.Models(S_n=1e3).require_gpu_path()


def _header_functions():
    src = open(os.path.join(ROOT, "include", "tcad_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tcad_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_header_symbol():
    """The .so loads (no GPU needed to dlopen) and exports every function the
    header declares; the ctypes binding covers the same set."""
    from tcad_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        import __graft_entry__
        __graft_entry__.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = _header_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(_lib.exported_names()) | {"tcad_pack_sizeof", "tcad_version"}
    assert lib.tcad_pack_sizeof() == ctypes.sizeof(_lib.TcadPack)


def _header_struct_fields(tag):
    """Field names of `typedef struct <tag> { ... }` in the header, in order
    (array fields by their name)."""
    src = open(os.path.join(ROOT, "include", "tcad_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    body = re.search(r"typedef struct " + tag + r"\s*\{(.*?)\}", src, flags=re.S).group(1)
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if decl:
            names.append(re.search(r"(\w+)\s*(\[\d+\])?$", decl).group(1))
    return names


@pytest.mark.parametrize("tag,cls", [("tcad_pack", "TcadPack"),
                                     ("tcad_newton_opts", "NewtonOpts"),
                                     ("tcad_newton_result", "NewtonResult")])
def test_ctypes_structs_mirror_the_header(tag, cls):
    """The ctypes mirrors list the header's fields in the header's order (a
    field added on one side only would shift every later one)."""
    from tcad_b200 import _lib
    assert [f[0] for f in getattr(_lib, cls)._fields_] == _header_struct_fields(tag)


def test_tile_depth_prior():
    """The starting 3D tile depth: the deeper of 4 and 2 planes that fills 4
    waves of 3 CTAs on 148 SMs, else 1 (2D: 1)."""
    from types import SimpleNamespace as NS
    from tcad_b200.pack import choose_tile_z
    mesh = lambda *nax: NS(nax=nax)  # noqa: E731
    assert choose_tile_z([mesh(160, 96, 64)], 3) == 2        # 960 tiles at 4, 1,920 at 2
    assert choose_tile_z([mesh(256, 256, 128)], 3) == 4      # 8,192 tiles at 4
    assert choose_tile_z([mesh(40, 24, 20)], 3) == 1
    assert choose_tile_z([mesh(160, 96, 64)] * 2, 3) == 4    # a pack of two: 1,920 at 4
    assert choose_tile_z([mesh(512, 256)], 2) == 1


def test_product_does_not_import_oracle():
    for dirpath, _, files in os.walk(os.path.join(ROOT, "tcad_b200")):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh")):
                txt = open(os.path.join(dirpath, f)).read()
                assert "import oracle" not in txt and "from oracle" not in txt, f


def test_range_allocator_first_fit_and_coalescing():
    from tcad_b200.serve import RangeAllocator
    a = RangeAllocator(1000, align=10)
    x = a.alloc(95)          # rounds to 100
    y = a.alloc(200)
    z = a.alloc(300)
    assert (x, y, z) == (0, 100, 300)
    assert a.alloc(500) is None and a.largest() == 400
    a.release(y, 200)
    assert a.alloc(150) == 100           # first fit into the hole
    a.release(100, 150)
    a.release(x, 95)
    assert a.free[0] == (0, 300)         # coalesced with the hole
    a.release(z, 300)
    assert a.free == [(0, 1000)] and a.free_total() == 1000


def test_arena_bytes_per_node():
    from tcad_b200.serve import bytes_per_node
    # coefficients + BC + state + previous state + F + J + du (doubles),
    # bcflag, FP64 and FP32 Krylov workspace, ILU(0) factor and vectors,
    # the equilibrium PCG's red-black extension
    assert 1490 <= bytes_per_node(2) <= 1580
    assert 1210 <= bytes_per_node(3) <= 1300


def test_arena_estimate_covers_the_workspace():
    """The serving arena's per-node estimate holds the library's own
    workspace (sized without the coupled red-black extension) with the node
    arrays it does not count."""
    import ctypes
    from tcad_b200 import _lib
    from tcad_b200.serve import bytes_per_node
    lib = _lib.load(require_gpu=False)
    for dim in (2, 3):
        P = _lib.TcadPack()
        P.dim, P.n_inst, P.n_nodes = dim, 64, 1 << 20
        P.n_flat, P.flat_nodes, P.tile_z = (1 << 20) // 256 + 64, _lib.FLAT_NODES, 2
        wb = lib.tcad_block_workspace_bytes(ctypes.byref(P), 0, 0)
        arrays = (1 + 3 * dim + 3 + 3 + 3 + 3 + _lib.NE[dim] + 3) * 8   # not in wb
        assert wb / P.n_nodes <= bytes_per_node(dim) - arrays + 64, (dim, wb / P.n_nodes)
