"""ctypes mirror of ``include/bosss_b200.h`` and the loader of the in-tree library.

The library is the product: there is no Python or CPU fallback. If
``libbosss_b200.so`` is missing, :func:`lib` raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# BOSSS_B200_LIB selects another build of the library (e.g. a tuning variant)
LIB_PATH = os.environ.get("BOSSS_B200_LIB") or os.path.join(HERE, "libbosss_b200.so")

MAX_VARS = 8
MAX_COMPONENTS = 32
MAX_PARAMS = 24

# status codes
OK = 0
ERR_BAD_ARG = -1
ERR_UNSUPPORTED_COMPONENT = -2
ERR_CUDA = -3
ERR_TIMEOUT = -4
ERR_NAN = -5
ERR_NO_DEVICE = -6
ERR_OUT_OF_MEMORY = -7

# component types
COMP_SCALAR_TRANSPORT_FLUX = 1
COMP_SIP_LAPLACE = 2
COMP_CONSTANT_SOURCE = 3
COMP_HLLC_DENSITY_FLUX = 10
COMP_HLLC_MOMENTUM_FLUX = 11
COMP_HLLC_ENERGY_FLUX = 12
COMP_CNS_SIPG_DENSITY_FLUX = 20
COMP_CNS_SIPG_MOMENTUM_FLUX = 21
COMP_CNS_SIPG_ENERGY_FLUX = 22

# quadrature-order kinds
QUAD_FIXED = 0
QUAD_LINEAR = 1
QUAD_NONLINEAR = 2
QUAD_MAXDEG_TIMES_TWO = 3
QUAD_SUM_OF_MAX_DEGREES = 4

CELLS_GENERATOR = 0
CELLS_GLOBALID = 1

# cudaStreamLegacy: the legacy default stream (a NULL stream argument selects the
# handle's own stream)
CUDA_STREAM_LEGACY = 1

MODE_RESIDUAL = 0
MODE_JVP = 1
MODE_VJP = 2

KERNEL_AUTO = 0
KERNEL_GENERIC = 1
KERNEL_SLAB = 2
KERNEL_FACES = 3

PRECISION_FP64 = 0
PRECISION_SPLIT_FP32 = 1


class Component(ctypes.Structure):
    _fields_ = [
        ("type", ctypes.c_int32),
        ("codomain", ctypes.c_int32),
        ("n_args", ctypes.c_int32),
        ("args", ctypes.c_int32 * MAX_VARS),
        ("params", ctypes.c_double * MAX_PARAMS),
    ]


class OpDesc(ctypes.Structure):
    _fields_ = [
        ("n_domain", ctypes.c_int32),
        ("n_codomain", ctypes.c_int32),
        ("domain_degree", ctypes.c_int32 * MAX_VARS),
        ("codomain_degree", ctypes.c_int32 * MAX_VARS),
        ("quad_kind", ctypes.c_int32),
        ("quad_param", ctypes.c_int32),
        ("n_components", ctypes.c_int32),
        ("components", Component * MAX_COMPONENTS),
    ]


class GridDesc(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32),
        ("n", ctypes.c_int32 * 3),
        ("lo", ctypes.c_double * 3),
        ("hi", ctypes.c_double * 3),
        ("periodic", ctypes.c_int32 * 3),
        ("cell_order", ctypes.c_int32),
        ("global_n", ctypes.c_int32 * 3),
        ("global_offset", ctypes.c_int32 * 3),
        ("global_periodic", ctypes.c_int32 * 3),
    ]


class SolverOpts(ctypes.Structure):
    _fields_ = [
        ("rtol", ctypes.c_double),
        ("atol", ctypes.c_double),
        ("max_outer", ctypes.c_int32),
        ("restart", ctypes.c_int32),
        ("max_krylov", ctypes.c_int32),
        ("precond", ctypes.c_int32),
        ("inner_rtol", ctypes.c_double),
        ("precond_update", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 7),
    ]


class SolverReport(ctypes.Structure):
    _fields_ = [
        ("outer_iters", ctypes.c_int32),
        ("krylov_iters", ctypes.c_int32),
        ("converged", ctypes.c_int32),
        ("reserved0", ctypes.c_int32),
        ("residual0", ctypes.c_double),
        ("residual", ctypes.c_double),
        ("reserved", ctypes.c_double * 6),
    ]


class LevelSetDesc(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("params", ctypes.c_double * 8)]


class XdgOpts(ctypes.Structure):
    _fields_ = [("cut_nodes_1d", ctypes.c_int32), ("fallback_nodes_1d", ctypes.c_int32),
                ("moment_degree", ctypes.c_int32), ("subdivision", ctypes.c_int32), ("rule", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 7)]


BOUNDARY_PRESCRIBED, BOUNDARY_OUTLET, BOUNDARY_SLIP_WALL = 0, 1, 2
XDG_RULE_MOMENT_FITTING = 0
XDG_RULE_SAYE = 1


LEVELSET_SPHERE = 1


class Options(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("check_nan", ctypes.c_int32),
        ("kernel", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 8),
    ]


_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
_I64 = ctypes.POINTER(ctypes.c_int64)
_I32 = ctypes.POINTER(ctypes.c_int32)

# name -> (restype, argtypes); every symbol declared in include/bosss_b200.h
SIGNATURES = {
    "bosss_b200_version": (ctypes.c_int, [_I32, _I32, _I32]),
    "bosss_b200_last_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
    "bosss_b200_device_count": (ctypes.c_int, [_I32]),
    "bosss_b200_create": (ctypes.c_int, [ctypes.POINTER(OpDesc), ctypes.POINTER(GridDesc),
                                         ctypes.POINTER(Options), ctypes.POINTER(_P)]),
    "bosss_b200_destroy": (ctypes.c_int, [_P]),
    "bosss_b200_get_sizes": (ctypes.c_int, [_P, _I64, _I64, _I32]),
    "bosss_b200_kernel_info": (ctypes.c_int, [_P, ctypes.c_int32, _I32, _I32]),
    "bosss_b200_set_boundary_kinds": (ctypes.c_int, [_P, _P]),
    "bosss_b200_saye_rule": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P, _P, ctypes.c_int32, _I64, _P, _P]),
    "bosss_b200_batch_solve": (ctypes.c_int, [_P, ctypes.c_int32, _P, _P, _P, _P, ctypes.POINTER(SolverOpts), _P]),
    "bosss_b200_pmg_create": (ctypes.c_int, [_P, _P, ctypes.POINTER(ctypes.c_void_p)]),
    "bosss_b200_pmg_apply_device": (ctypes.c_int, [_P, _P, _P, _P]),
    "bosss_b200_pmg_info": (ctypes.c_int, [_P, _I32, _I32, _I64, _I32]),
    "bosss_b200_pmg_destroy": (ctypes.c_int, [_P]),
    "bosss_b200_evaluate": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, _P, _P, ctypes.c_double]),
    "bosss_b200_evaluate_device": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, _P, _P,
                                                  ctypes.c_double, _P]),
    "bosss_b200_jvp": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_double]),
    "bosss_b200_vjp": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_double]),
    "bosss_b200_jvp_device": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_double, _P]),
    "bosss_b200_vjp_device": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_double, _P]),
    "bosss_b200_synchronize": (ctypes.c_int, [_P]),
    "bosss_b200_bsr_create": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                             _P, _P, _P, ctypes.c_int32, ctypes.POINTER(_P)]),
    "bosss_b200_bsr_destroy": (ctypes.c_int, [_P]),
    "bosss_b200_bsr_spmv": (ctypes.c_int, [_P, ctypes.c_double, _P, ctypes.c_double, _P]),
    "bosss_b200_bsr_spmv_device": (ctypes.c_int, [_P, ctypes.c_double, _P, ctypes.c_double, _P, _P]),
    "bosss_b200_bsr_get": (ctypes.c_int, [_P, _I64, _I64, _I32, _I32, _I64, _P, _P, _P]),
    "bosss_b200_compute_jacobian": (ctypes.c_int, [_P, _P, ctypes.c_double, ctypes.POINTER(_P)]),
    "bosss_b200_newton_solve": (ctypes.c_int, [_P, _P, ctypes.c_double, ctypes.POINTER(SolverOpts),
                                               ctypes.POINTER(SolverReport)]),
    "bosss_b200_bsr_solve": (ctypes.c_int, [_P, _P, _P, ctypes.POINTER(SolverOpts), ctypes.POINTER(SolverReport)]),
    "bosss_b200_batch_create": (ctypes.c_int, [ctypes.c_int32, _P, _P, ctypes.POINTER(Options), ctypes.POINTER(_P)]),
    "bosss_b200_batch_destroy": (ctypes.c_int, [_P]),
    "bosss_b200_batch_get_sizes": (ctypes.c_int, [_P, _P, _P]),
    "bosss_b200_batch_evaluate": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_double, ctypes.c_double, _P, _P, _P,
                                                 ctypes.c_double]),
    "bosss_b200_batch_evaluate_device": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_double, ctypes.c_double, _P, _P,
                                                        _P, ctypes.c_double, _P]),
    "bosss_b200_batch_capture": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_double]),
    "bosss_b200_batch_replay": (ctypes.c_int, [_P, _P]),
    "bosss_b200_batch_autotune": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_char_p]),
    "bosss_b200_batch_tiles": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, _I32, _I32]),
    "bosss_b200_xdg_create": (ctypes.c_int, [_P, _P, _P, ctypes.POINTER(LevelSetDesc), ctypes.POINTER(XdgOpts),
                                             ctypes.POINTER(Options), ctypes.POINTER(_P)]),
    "bosss_b200_xdg_destroy": (ctypes.c_int, [_P]),
    "bosss_b200_xdg_info": (ctypes.c_int, [_P, ctypes.c_int32, _I64, _I64, _I64, _I32, _I32, _I32, _D]),
    "bosss_b200_xdg_get_rules": (ctypes.c_int, [_P, ctypes.c_int32, _P, _P, _P, _P, _P, _P, _P]),
    "bosss_b200_xdg_get_moments": (ctypes.c_int, [_P, ctypes.c_int32, _P]),
    "bosss_b200_xdg_get_length_scales": (ctypes.c_int, [_P, ctypes.c_int32, _P]),
    "bosss_b200_boundary_nodes": (ctypes.c_int, [_P, _I64, _P]),
    "bosss_b200_set_boundary_state": (ctypes.c_int, [_P, _P]),
    "bosss_b200_xdg_set_length_scales": (ctypes.c_int, [_P, ctypes.c_int32, _P]),
    "bosss_b200_xdg_evaluate": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_double, ctypes.c_double, _P, _P,
                                               ctypes.c_double]),
    "bosss_b200_xdg_evaluate_device": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_double, ctypes.c_double, _P, _P,
                                                      ctypes.c_double, _P]),
    "bosss_b200_xdg_interface_setup": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                      ctypes.c_int32, ctypes.c_int32]),
    "bosss_b200_xdg_interface_get_rules": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "bosss_b200_xdg_interface_evaluate": (ctypes.c_int, [_P, ctypes.c_double, _P, _P, _P, _P]),
    "bosss_b200_xdg_interface_evaluate_device": (ctypes.c_int, [_P, ctypes.c_double, _P, _P, _P, _P, _P]),
    "bosss_b200_batch_evaluate_noalloc": (ctypes.c_int, [ctypes.c_int32, _P, ctypes.c_int32, ctypes.c_double,
                                                         ctypes.c_double, _P, _P, _P, ctypes.c_double, _P]),
    "bosss_b200_residual_vjp": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, _P, _P, _P, _P,
                                               ctypes.c_double]),
    "bosss_b200_apply_device": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_double, ctypes.c_double, _P, _P, _P,
                                               ctypes.c_double, ctypes.c_int64, ctypes.c_int64, _P]),
    "bosss_b200_rk_work_size": (ctypes.c_int, [_P, ctypes.c_int32, _I64]),
    "bosss_b200_rk_steps_device": (ctypes.c_int, [_P, ctypes.c_int32, _P, _P, _P, ctypes.c_double, ctypes.c_int32,
                                                  ctypes.c_double, _P, _P, ctypes.c_int32, _P]),
    "bosss_b200_rk_steps": (ctypes.c_int, [_P, ctypes.c_int32, _P, _P, _P, ctypes.c_double, ctypes.c_int32,
                                           ctypes.c_double, _P]),
}

_lib = None


class BosssError(RuntimeError):
    """Raised for a non-zero status of a C-ABI call; ``code`` is the status."""

    def __init__(self, code, msg):
        super().__init__("bosss_b200 error %d: %s" % (code, msg))
        self.code = code


def lib():
    """Load ``libbosss_b200.so`` (built in-tree); raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libbosss_b200.so is not built (run python -m bosss_b200.build); "
                               "there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error():
    buf = ctypes.create_string_buffer(1024)
    lib().bosss_b200_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc):
    if rc != OK:
        raise BosssError(rc, last_error())
    return rc


def ptr(a):
    """Raw data pointer of a numpy array or a torch tensor (host or device)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)
