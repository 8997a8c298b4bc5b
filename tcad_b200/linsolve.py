"""linsolve drop-in on the GPU (pytcad/linsolve.py).

``LinearSolveError`` is the reference's error class contract
(pytcad/linsolve.py:344-351): raised on singular or non-finite input and on
iterative non-convergence; a failed solve never returns a half-solved state.
"""


class LinearSolveError(RuntimeError):
    """Singular / non-finite input or iterative non-convergence."""
