"""linsolve drop-in on the GPU (pytcad/linsolve.py).

``solve_linear(A, b, *, method, rtol, atol, maxiter, x0, restart, block_size,
precond)`` keeps the reference's signature, return value ``(x, info)`` and
error contract (pytcad/linsolve.py:725-985): "gmres" and "bicgstab" run on
the GPU (libtcad_b200 ``tcad_csr_krylov``), right-preconditioned by node-
block-Jacobi when ``block_size`` is given (pytcad/linsolve.py:363-427), and
are accepted only when the true residual satisfies
``||A x - b|| / ||b|| <= max(rtol, 1e-6)``; otherwise LinearSolveError.

Not on this path, raising LinearSolveError (the class every reference caller
already handles): the CPU direct solvers ("direct", "petsc", "mumps") and
"gpu_direct" (a cuSOLVER library call in the reference).  Where the
reference builds an ILU or AMG preconditioner (block_size None, or a failed
block inverse, pytcad/linsolve.py:526-585), the GPU uses point Jacobi.
"""
from __future__ import annotations

import ctypes

import numpy as np
import scipy.sparse as sp

_METHODS = ("direct", "gmres", "bicgstab", "gpu_direct", "petsc", "mumps")
_PRECOND = ("auto", "block_jacobi", "schur")


class LinearSolveError(RuntimeError):
    """Singular / non-finite input or iterative non-convergence
    (pytcad/linsolve.py:344-351): a failed solve never returns a half-solved
    state."""


def solve_linear(A, b, *, method="direct", rtol=1e-10, atol=0.0, maxiter=500,
                 x0=None, restart=None, block_size=None, precond="auto"):
    """Solve A x = b on the GPU.  Returns (x, info) with info keys
    method, iterations, converged, residual (and precond: the preconditioner
    that ran -- "block_jacobi", "jacobi" or "none")."""
    if method not in _METHODS:
        raise ValueError(f"unknown method {method!r}; choose from {_METHODS}")
    if precond not in _PRECOND:
        raise ValueError(f"unknown precond {precond!r}; choose from {_PRECOND}")
    if method not in ("gmres", "bicgstab"):
        raise LinearSolveError(
            f"solve_linear(method={method!r}) is not available on the GPU path "
            "(tcad_b200 solves with GMRES/BiCGStab + node-block-Jacobi)")
    import torch
    from . import _lib
    lib = _lib.load()
    A = sp.csr_matrix(A) if not sp.issparse(A) else A.tocsr()
    b = np.asarray(b, dtype=float).ravel()
    n = A.shape[0]
    if A.shape != (n, n) or b.size != n:
        raise ValueError(f"shape mismatch: A {A.shape}, b {b.shape}")
    if not np.all(np.isfinite(b)):
        raise LinearSolveError(f"solve_linear({method!r}): b contains non-finite values")
    if not np.all(np.isfinite(A.data)):
        raise LinearSolveError(f"solve_linear({method!r}): A contains non-finite values")
    if A.nnz == 0 or np.any(np.diff(A.indptr) == 0):
        raise LinearSolveError(f"solve_linear({method!r}): A has an empty row (singular)")
    if A.nnz >= 2 ** 31 or n >= 2 ** 31:
        raise ValueError("solve_linear: matrix too large for 32-bit CSR indices")
    dev = torch.device("cuda")
    up = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
    ip = up(A.indptr.astype(np.int32), torch.int32)
    ix = up(A.indices.astype(np.int32), torch.int32)
    dv = up(A.data.astype(np.float64), torch.float64)
    bd = up(b, torch.float64)
    xd = (torch.zeros(n, dtype=torch.float64, device=dev) if x0 is None
          else up(np.asarray(x0, dtype=float).ravel(), torch.float64))
    meth = 1 if method == "gmres" else 0
    rst = int(min(restart or 100, n))
    bs = int(block_size) if block_size else 0
    wb = int(lib.tcad_csr_workspace_bytes(n, meth, rst))
    work = torch.empty(wb, dtype=torch.uint8, device=dev)
    iters = ctypes.c_int32(0)
    resid = ctypes.c_double(0.0)
    pc = ctypes.c_int32(0)
    rc = lib.tcad_csr_krylov(n, _lib.ptr(ip), _lib.ptr(ix), _lib.ptr(dv), _lib.ptr(bd),
                             _lib.ptr(xd), meth, bs, float(rtol), float(atol), int(maxiter),
                             rst, _lib.ptr(work), wb, ctypes.byref(iters),
                             ctypes.byref(resid), ctypes.byref(pc), _lib.stream_ptr())
    if rc not in (_lib.TCAD_OK, _lib.TCAD_ERR_NOCONV):
        _lib.check(rc, f"solve_linear({method!r})")
    x = xd.cpu().numpy()
    res = float(resid.value)
    converged = rc == _lib.TCAD_OK and bool(np.all(np.isfinite(x))) and res <= max(rtol, 1e-6)
    if not converged:
        raise LinearSolveError(
            f"{method} did not converge within {maxiter} iterations (relative "
            f"residual={res:.3e}, target rtol={rtol:.3e}) -- refusing to return the "
            "unconverged iterate")
    return x, {"method": method, "iterations": int(iters.value), "converged": True,
               "residual": res,
               "precond": {6: "block_jacobi", 3: "block_jacobi", 1: "jacobi",
                           0: "none"}[int(pc.value)]}
