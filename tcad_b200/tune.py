"""Launch-shape autotuner for the coupled assembly.

The 3D assembly's tile depth (`tile_z`: how many z-planes one CTA of the
fused SG assembly marches) trades the z-edge that every tile re-evaluates at
its first plane against the number of CTAs and the tail of the last wave.
The best depth depends on the mesh and on the GPU, so it is measured: each
candidate depth assembles the pack's current state (CUDA events on the
pack's stream, after one untimed launch), the fastest is kept for the pack
and remembered for the process under the pack's mesh-shape key.

The depth only decides which CTA evaluates a node, never the arithmetic:
every candidate gives the same residual and Jacobian bit for bit, so tuning
cannot change a result.
"""
from . import _lib

CANDIDATES = (1, 2, 4, 8, 16)

_cache = {}
last_timings = {}   # candidate depth -> us, of the last measured key


def shape_key(pack):
    return (pack.dim,) + tuple(tuple(int(a) for a in s.nax[:pack.dim]) for s in pack.setups)


def time_assembly(pack, reps=3):
    """Mean device time (us) of one coupled assembly of the pack's state
    into its F/J buffers, after one untimed launch."""
    torch = pack.torch
    args = (pack.pref, _lib.ptr(pack.psi), _lib.ptr(pack.n), _lib.ptr(pack.p),
            _lib.ptr(pack.F), _lib.ptr(pack.J), _lib.MODE_ELIMINATE, pack.sp())
    _lib.check(pack.lib.tcad_sg_assemble(*args), "tcad_sg_assemble")
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        _lib.check(pack.lib.tcad_sg_assemble(*args), "tcad_sg_assemble")
    b.record()
    b.synchronize()
    return a.elapsed_time(b) * 1e3 / reps


def tune_tile_z(pack, candidates=CANDIDATES, reps=3):
    """Set the pack's 3D tile depth to the fastest candidate for its meshes
    (measured once per mesh-shape key and process) and return it.  The
    pack's F and J are scratch here: call it before a solve, which assembles
    first.  Timings are kept in `last_timings`."""
    if pack.dim != 3:
        return 1
    key = shape_key(pack)
    if key not in _cache:
        nz = max(int(s.nax[2]) for s in pack.setups)
        cands = [tz for tz in candidates if tz <= max(nz, 1)] or [1]
        times = {}
        for tz in cands:
            pack.set_tile_z(tz)
            times[tz] = time_assembly(pack, reps)
        last_timings.clear()
        last_timings.update(times)
        _cache[key] = min(cands, key=lambda tz: (times[tz], tz))
    best = _cache[key]
    if pack.tile_z != best:
        pack.set_tile_z(best)
    return best


def clear():
    _cache.clear()
    last_timings.clear()
