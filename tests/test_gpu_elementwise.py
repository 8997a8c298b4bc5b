"""Elementwise parity of the SG device functions against the reference.

The assembly kernels evaluate the Bernoulli function, its derivative and the
SRH/Auger recombination rate inside one translation unit compiled with the
assembly's rounding (-fmad=false).  tcad_eval_bernoulli / _recombination run
those same device functions on arrays, so these tests compare them, value by
value, with the reference's own outputs in tests/golden/elem.npz
(pytcad/kernels.py:88-109 bernoulli / dbernoulli at 816 arguments, including
the series threshold 1e-4 (1 +- 1e-12), the clip at 700 / 701 and 1e-300;
pytcad/materials.py:474-518 recombination at 64 random states).

Bar: 1e-12 relative per element (the drop-in's assembly tolerance), with no
normwise averaging."""
import numpy as np
import pytest

import fixtures as fx

pytestmark = pytest.mark.gpu

TOL_ELEM = 1e-12


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def test_bernoulli_elementwise():
    import torch
    from tcad_b200 import _lib
    lib = _lib.load()
    g = fx.load("elem")
    x = g["x"]
    n = x.size
    half = n // 2
    assert np.array_equal(x[half:], -x[:half])   # the fixture holds +x and -x
    mirror = np.concatenate([np.arange(half, n), np.arange(half)])
    xd = torch.tensor(x, dtype=torch.float64, device="cuda")
    out = torch.empty(4 * n, dtype=torch.float64, device="cuda")
    rc = lib.tcad_eval_bernoulli(_lib.ptr(xd), n, _lib.ptr(out), _lib.stream_ptr())
    assert rc == _lib.TCAD_OK
    Bp, Bm, dBp, dBm = out.cpu().numpy().reshape(4, n)
    refs = (g["B"], g["B"][mirror], g["dB"], g["dB"][mirror])
    errs = [_rel(v, r) for v, r in zip((Bp, Bm, dBp, dBm), refs)]
    for name, e in zip(("B(x)", "B(-x)", "B'(x)", "B'(-x)"), errs):
        k = int(np.argmax(e))
        assert e[k] <= TOL_ELEM, f"{name}: {e[k]:.3e} at x={x[k]!r}"
    # the values themselves agree to a few ulp
    assert errs[0].max() < 1e-15 and errs[1].max() < 1e-15


@pytest.mark.parametrize("auger,key", [(True, "R_aug"), (False, "R_srh")])
def test_recombination_elementwise(auger, key):
    import torch
    import tcad_b200 as tb
    from tcad_b200 import _lib
    lib = _lib.load()
    g = fx.load("elem")
    mat = tb.Semiconductor()
    cnt = g["rn"].size
    par = np.zeros(_lib.NPAR)
    par[0], par[1] = 1.0, 1.0          # Ns = R0 = 1: physical rates
    par[2], par[3] = mat.Cn_auger, mat.Cp_auger
    par[4], par[5] = 1.0, 1.0 if auger else 0.0

    def t(a):
        return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    args = [t(g[k]) for k in ("rn", "rp", "rnie", "rtn", "rtp")]
    pd = t(par)
    out = torch.empty(3 * cnt, dtype=torch.float64, device="cuda")
    rc = lib.tcad_eval_recombination(*[_lib.ptr(a) for a in args], cnt, _lib.ptr(pd),
                                     _lib.ptr(out), _lib.stream_ptr())
    assert rc == _lib.TCAD_OK
    o = out.cpu().numpy().reshape(3, cnt)
    ref = g[key]
    for r in range(3):
        assert _rel(o[r], ref[r]).max() <= 1e-15, (r, _rel(o[r], ref[r]).max())
