"""ctypes binding of the C ABI in include/tcad_b200.h.

The library is the in-tree ``tcad_b200/libtcad_b200.so`` built by
``tcad_b200/build.py`` (sm_100a).  There is no CPU fallback: importing the
solve path without the library, or without a CUDA device, raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtcad_b200.so")
# A different build of the same library (same ABI) can be selected with
# TCAD_B200_LIB, e.g. to compare compile options of the kernels.
LIB_PATH = os.environ.get("TCAD_B200_LIB", LIB_PATH)

TCAD_OK = 0
TCAD_ERR_ARG = 1
TCAD_ERR_SINGULAR = 2
TCAD_ERR_NONFINITE = 3
TCAD_ERR_NOCONV = 4
TCAD_ERR_CUDA = 5
TCAD_ERR_BREAKDOWN = 6
STATUS_NAMES = {0: "ok", 1: "bad argument", 2: "singular node block",
                3: "non-finite values", 4: "not converged", 5: "CUDA error",
                6: "Krylov breakdown", -1: "idle"}

NE = {2: 29, 3: 39}
FLAT_NODES = 512
TILE_X, TILE_Y, TILE_Z_MAX = 32, 8, 16
NPAR = 8
MODE_RAW, MODE_ELIMINATE, MODE_UNSTAMPED = 0, 1, 2
BC_CONTACT, BC_GATE = 1, 2

_p = ctypes.c_void_p


class TcadPack(ctypes.Structure):
    """Mirror of tcad_pack_t (include/tcad_b200.h)."""
    _fields_ = [
        ("dim", ctypes.c_int32), ("n_inst", ctypes.c_int32),
        ("n_nodes", ctypes.c_int64), ("n_flat", ctypes.c_int64),
        ("n_tiles", ctypes.c_int64), ("tile_z", ctypes.c_int32),
        ("flat_nodes", ctypes.c_int32), ("asm_stage", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("shape", _p), ("node_off", _p), ("flat_off", _p), ("flat_inst", _p),
        ("axis_off", _p), ("tile", _p), ("par", _p),
        ("h", _p * 3), ("dv", _p * 3),
        ("C", _p), ("nie", _p), ("nie_s", _p), ("tau_n", _p), ("tau_p", _p),
        ("an", _p * 3), ("ap", _p * 3), ("dl", _p * 3),
        ("bcflag", _p), ("bc_psi0", _p), ("bc_n0", _p), ("bc_p0", _p),
        ("bc_psi0_eq", _p), ("gate_k", _p), ("gate_v", _p), ("gate_veq", _p),
        ("gate_b", _p),
    ]


class NewtonOpts(ctypes.Structure):
    _fields_ = [("max_iter", ctypes.c_int32), ("method", ctypes.c_int32),
                ("krylov_maxiter", ctypes.c_int32), ("restart", ctypes.c_int32),
                ("tol_update", ctypes.c_double), ("max_dpsi", ctypes.c_double),
                ("rtol", ctypes.c_double), ("dens_floor", ctypes.c_double),
                ("verbose", ctypes.c_int32), ("polish", ctypes.c_int32),
                ("eta_max", ctypes.c_double), ("forcing", ctypes.c_int32),
                ("precision", ctypes.c_int32),
                ("density_scaling", ctypes.c_int32), ("precond", ctypes.c_int32),
                ("eta_min", ctypes.c_double), ("scale_floor", ctypes.c_double),
                ("polish_eta", ctypes.c_double), ("polish_scale_floor", ctypes.c_double),
                ("dt", ctypes.c_double), ("theta", ctypes.c_double),
                ("n_old", _p), ("p_old", _p), ("fn_old", _p), ("fp_old", _p),
                ("red_black", ctypes.c_int32), ("reserved_opts", ctypes.c_int32)]


class NewtonResult(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int32), ("converged", ctypes.c_int32),
                ("krylov_iters", ctypes.c_int32), ("status", ctypes.c_int32),
                ("err", ctypes.c_double), ("relres", ctypes.c_double),
                ("fp64_from", ctypes.c_int32), ("polish_iters", ctypes.c_int32)]


# name -> (restype, argtypes)
_SIGS = {
    "tcad_pack_sizeof": (ctypes.c_size_t, []),
    "tcad_version": (ctypes.c_char_p, []),
    "tcad_launch_count": (ctypes.c_uint64, []),
    "tcad_sg_assemble": (ctypes.c_int, [_p, _p, _p, _p, _p, _p, ctypes.c_int, _p]),
    "tcad_contact_current": (ctypes.c_int, [_p, _p, _p, _p, _p, ctypes.c_int64, _p,
                                            ctypes.c_int64, _p, _p]),
    "tcad_edge_currents": (ctypes.c_int, [_p, ctypes.c_int, _p, _p, _p, _p, _p, _p]),
    "tcad_poisson_assemble": (ctypes.c_int, [_p, _p, _p, _p, ctypes.c_int, _p]),
    "tcad_eval_bernoulli": (ctypes.c_int, [_p, ctypes.c_int64, _p, _p]),
    "tcad_eval_recombination": (ctypes.c_int, [_p, _p, _p, _p, _p, ctypes.c_int64, _p, _p,
                                               _p]),
    "tcad_block_workspace_bytes": (ctypes.c_size_t, [_p, ctypes.c_int, ctypes.c_int]),
    "tcad_set_krylov_fused": (ctypes.c_int, [ctypes.c_int]),
    "tcad_set_krylov_fused_test": (ctypes.c_int, [ctypes.c_int]),
    "tcad_krylov_fused_gave_up": (ctypes.c_uint64, []),
    "tcad_state_extrapolate": (ctypes.c_int, [_p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "tcad_block_jacobi_setup": (ctypes.c_int, [_p, _p, _p, _p, _p]),
    "tcad_block_jacobi_setup_rel": (ctypes.c_int, [_p, _p, _p, _p, _p, _p, ctypes.c_double,
                                                   _p]),
    "tcad_block_spmv": (ctypes.c_int, [_p, _p, _p, _p, _p]),
    "tcad_block_ilu_bytes": (ctypes.c_size_t, [_p]),
    "tcad_block_ilu_setup": (ctypes.c_int, [_p, _p, _p, _p, _p]),
    "tcad_block_ilu_apply": (ctypes.c_int, [_p, _p, _p, _p, _p, _p]),
    "tcad_block_krylov": (ctypes.c_int, [_p, _p, _p, _p, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_int, _p, ctypes.c_size_t,
                                         _p, _p, _p, _p]),
    "tcad_newton_update": (ctypes.c_int, [_p, _p, _p, _p, _p, ctypes.c_double,
                                          ctypes.c_double, _p, _p, _p, _p]),
    "tcad_newton_solve": (ctypes.c_int, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p,
                                         ctypes.c_size_t, _p, _p]),
    "tcad_equilibrium_solve": (ctypes.c_int, [_p, _p, _p, _p, _p, _p, _p, _p, _p,
                                              ctypes.c_size_t, _p, _p]),
    "tcad_set_contacts": (ctypes.c_int, [_p, _p, ctypes.c_int64, _p, _p, _p, _p, _p,
                                         _p, _p, _p, _p]),
    "tcad_stamp_contacts": (ctypes.c_int, [_p, _p, ctypes.c_int64, _p, _p, _p, _p]),
    "tcad_block_krylov_noalloc": (ctypes.c_int, [_p, _p, _p, _p, ctypes.c_double,
                                                 ctypes.c_int, _p, _p, _p, _p]),
    "tcad_csr_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int64, ctypes.c_int, ctypes.c_int]),
    "tcad_csr_krylov": (ctypes.c_int, [ctypes.c_int64, _p, _p, _p, _p, _p, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int, ctypes.c_int, _p, ctypes.c_size_t,
                                       _p, _p, _p, _p]),
}

_lib = None


def exported_names():
    return sorted(_SIGS)


def load(require_gpu=True):
    """Load the library (once).  Raises ImportError when it is not built --
    the product has no CPU path to fall back to."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"tcad_b200: CUDA library not built ({LIB_PATH} missing); run "
            "`python -c 'import __graft_entry__ as g; g.build()'` or "
            "`python tcad_b200/build.py`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.tcad_pack_sizeof() != ctypes.sizeof(TcadPack):
        raise ImportError("tcad_b200: tcad_pack_t ABI mismatch between the "
                          "library and the Python binding")
    _lib = lib
    return lib


def check(rc, what):
    """Map a TCAD status onto the reference's exception classes
    (core/bindings/module.cpp:100-127 does the same for the C++ core)."""
    if rc == TCAD_OK:
        return
    from .linsolve import LinearSolveError
    msg = f"{what}: {STATUS_NAMES.get(rc, rc)}"
    if rc == TCAD_ERR_ARG:
        raise ValueError(msg)
    if rc == TCAD_ERR_CUDA:
        raise RuntimeError(msg)
    raise LinearSolveError(msg)


def ptr(t):
    """Raw device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_ptr():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
