"""ORACLE -- test infrastructure only, never shipped or measured.

CPU restatement (numpy + scipy) of PyTCAD's structured drift-diffusion
solve: the scaled device set-up, the Scharfetter-Gummel box-integration
residual/Jacobian (Device2D 5-point, Device3D 7-point), the symmetric
Dirichlet elimination, the damped Newton loops with a sparse direct solve,
and the terminal-current extraction.  Each function cites the reference
file:line it restates (paths relative to the reference's ``pytcad/``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline legs may import this package, and only as the checker.  The
product (``tcad_b200``) never imports it.

Parity is pinned: ``tests/golden/make_golden.py`` runs the reference itself
(importable in the build container) and commits its outputs as fixtures;
``tests/test_oracle_golden.py`` holds this restatement to them.
"""
from .dd_oracle import (  # noqa: F401
    SILICON_PARAMS, OracleModels, OracleDevice, bernoulli, dbernoulli,
    recombination, ohmic_values, control_volume_widths, eliminate_csr,
    build_block_jacobi, solve_linear_iterative,
)
