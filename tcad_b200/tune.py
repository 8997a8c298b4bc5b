"""Launch-shape autotuner for the coupled assembly.

Two knobs of the 3D assembly are measured per mesh: the tile depth (below)
and the plane staging (`asm_stage`: the next z-plane's edge and node
coefficients copied into shared memory asynchronously while the current
plane computes, at 2 CTAs per SM, or loaded in place at 3 CTAs per SM).
Neither changes the arithmetic, so both are tuned on timing alone.

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
STAGES = (0, 1)

_cache = {}
last_timings = {}   # candidate (depth, staging) -> us, of the last measured key


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


def tune_assembly(pack, candidates=CANDIDATES, stages=STAGES, reps=3):
    """Set the pack's 3D tile depth and plane staging to the fastest
    candidate pair for its meshes (measured once per mesh-shape key and
    process) and return it.  The pack's F and J are scratch here: call it
    before a solve, which assembles first.  Timings are kept in
    `last_timings`."""
    if pack.dim != 3:
        return (1, 0)
    key = shape_key(pack)
    if key not in _cache:
        nz = max(int(s.nax[2]) for s in pack.setups)
        cands = [tz for tz in candidates if tz <= max(nz, 1)] or [1]
        times = {}
        for st in stages:
            pack.set_asm_stage(st)
            for tz in cands:
                pack.set_tile_z(tz)
                times[(tz, st)] = time_assembly(pack, reps)
        last_timings.clear()
        last_timings.update(times)
        _cache[key] = min(times, key=lambda c: (times[c], c))
    tz, st = _cache[key]
    if pack.tile_z != tz:
        pack.set_tile_z(tz)
    pack.set_asm_stage(st)
    return tz, st


def tune_tile_z(pack, candidates=CANDIDATES, reps=3):
    """The tile depth alone, unstaged (tune_assembly with stages (0,))."""
    return tune_assembly(pack, candidates, (0,), reps)[0] if pack.dim == 3 else 1


def clear():
    _cache.clear()
    last_timings.clear()
