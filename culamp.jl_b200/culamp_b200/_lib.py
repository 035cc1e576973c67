"""ctypes binding of libculamp_b200.so (declared in include/culamp.h).

The library is built in-tree by culamp.jl_b200/build.py. Loading it needs no
GPU (settings parsing works on any host); every compute entry point needs a
CUDA device and raises CulampError when it fails -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT_DIR = os.path.dirname(PKG_DIR)
LIB_PATH = os.path.join(ROOT_DIR, "libculamp_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(ROOT_DIR), "include", "culamp.h")

OK = 0
ERR_INVALID_ARG = 1
ERR_CUDA = 2
ERR_ALLOC = 3
ERR_UNSUPPORTED = 4
ERR_IO = 5
ERR_DEVICE_TIMEOUT = 6

FLAG_TRUE_PINF = 1
FLAG_CHECK_ALWAYS = 2
FLAG_MARGINAL_ONLY = 4
FLAG_FORM_PLAIN = 8
FLAG_NO_GRAPH = 16
FLAG_FEAT_X6 = 32
FLAG_FEAT_FP64 = 64
FLAG_FORM_FP32 = 128
FLAG_LADDER = 256
FLAG_FORM_FP64 = 512
FLAG_NO_PERSIST = 1024


class CulampError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"culamp status {status}: {message}")
        self.status = status


class CArgs(C.Structure):
    _fields_ = [("eta_p", C.c_double), ("eta_mu", C.c_double), ("tau_p", C.c_double),
                ("tau_mu", C.c_double), ("alpha", C.c_double), ("B", C.c_double),
                ("epsilon", C.c_double), ("anneal_mult", C.c_double),
                ("itermax", C.c_int64), ("inner_iter", C.c_int64), ("tmax", C.c_double),
                ("verbose", C.c_int32), ("_pad", C.c_int32)]


class CLogRow(C.Structure):
    _fields_ = [("time_s", C.c_double), ("iter", C.c_double), ("infeas", C.c_double),
                ("ot_objective", C.c_double), ("primal", C.c_double), ("dual", C.c_double)]


class CStats(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("num_iter", C.c_int64), ("residual", C.c_double),
                ("objective", C.c_double), ("winf", C.c_double), ("eta_t", C.c_double),
                ("s_t", C.c_double), ("elapsed_ms", C.c_double), ("log_rows", C.c_int64),
                ("stopped", C.c_int32), ("status", C.c_int32)]


class CInstance(C.Structure):
    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("r", C.c_void_p), ("c", C.c_void_p),
                ("phi", C.c_void_p), ("psi", C.c_void_p), ("n", C.c_int64), ("m", C.c_int64),
                ("d", C.c_int32), ("reserved", C.c_int32)]


class CBatchStats(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("num_iter", C.c_int64), ("residual", C.c_double),
                ("objective", C.c_double), ("winf", C.c_double), ("stopped", C.c_int32),
                ("status", C.c_int32)]


class CBatchInfo(C.Structure):
    _fields_ = [("elapsed_ms", C.c_double), ("tune_ms", C.c_double),
                ("target_ctas_per_sm", C.c_int32), ("feat_tiles_per_unit", C.c_int32),
                ("unroll", C.c_int32), ("launches_per_iteration", C.c_int32),
                ("phases", C.c_int32), ("reserved", C.c_int32)]


_VP = C.c_void_p
_D = C.c_double
_I64 = C.c_int64
_I32 = C.c_int32
_U32 = C.c_uint32

# name -> (restype, argtypes); must match include/culamp.h
SIGNATURES = {
    "culamp_version": (C.c_int, []),
    "culamp_create": (C.c_int, [C.POINTER(_VP), C.c_int]),
    "culamp_destroy": (C.c_int, [_VP]),
    "culamp_status_string": (C.c_char_p, [C.c_int]),
    "culamp_last_error": (C.c_char_p, [_VP]),
    "culamp_args_default": (C.c_int, [C.POINTER(CArgs)]),
    "culamp_args_from_json": (C.c_int, [C.c_char_p, C.POINTER(CArgs)]),
    "culamp_args_from_json_string": (C.c_int, [C.c_char_p, C.POINTER(CArgs)]),
    "culamp_max_cost": (C.c_int, [_VP, _VP, _VP, _I64, _I64, _I32, _D, _VP, C.POINTER(_D), _VP]),
    "culamp_lse_rows_sk": (C.c_int, [_VP, _VP, _VP, _VP, _I64, _I64, _I32, _VP, _VP, _D, _D, _D, _VP]),
    "culamp_lse_rows_sk_form": (C.c_int, [_VP, _VP, _VP, _VP, _I64, _I64, _I32, _VP, _VP, _D, _D, _D,
                                          C.c_uint32, _VP]),
    "culamp_residual_sk": (C.c_int, [_VP, _VP, _VP, _VP, _VP, _I64, _I64, _I32, _VP, _VP, _VP,
                                     _D, _D, _D, _VP]),
    "culamp_lse_rows_spp": (C.c_int, [_VP, _VP, _VP, _VP, _I64, _I64, _I32, _VP, _D, _D, _D, _D, _VP]),
    "culamp_col_residual_spp": (C.c_int, [_VP, _VP, _VP, _VP, _VP, _I64, _I64, _I32, _VP, _VP, _VP,
                                          _D, _D, _D, _D, _VP]),
    "culamp_min_reduce": (C.c_int, [_VP, _VP, _VP, _VP, _I64, _I64, _I32, _VP, _D, _D, _VP]),
    "culamp_theta_update": (C.c_int, [_VP, _VP, _VP, _VP, _VP, _VP, _D, _I32, _D, _D, _D, _I64, _VP]),
    "culamp_barycentric_sk": (C.c_int, [_VP, _VP, _VP, _VP, _I64, _I64, _I32, _VP, _VP, _D, _D, _D, _VP]),
    "culamp_sinkhorn": (C.c_int, [_VP, _VP, _VP, _I64, _I64, _I32, _VP, _VP, C.POINTER(CArgs), _I64,
                                  _D, _VP, _VP, _U32, _VP, _VP, C.POINTER(CStats),
                                  C.POINTER(CLogRow), _I64, _VP]),
    "culamp_lamp": (C.c_int, [_VP, _VP, _VP, _I64, _I64, _I32, _VP, _VP, C.POINTER(CArgs), _I64, _D,
                              _U32, _VP, _VP, _VP, _VP, C.POINTER(CStats), C.POINTER(CLogRow), _I64,
                              _VP]),
    "culamp_annealed_sinkhorn": (C.c_int, [_VP, _VP, _VP, _I64, _I64, _I32, _VP, _VP,
                                           C.POINTER(CArgs), _I64, _D, _U32, _VP, _VP,
                                           C.POINTER(CStats), C.POINTER(CLogRow), _I64, _VP]),
    "culamp_symmetric_sinkhorn": (C.c_int, [_VP, _VP, _I64, _I32, _VP, C.POINTER(CArgs), _I64, _D, _VP,
                                            _U32, _VP, C.POINTER(CStats), C.POINTER(CLogRow), _I64, _VP]),
    "culamp_sinkhorn_host": (C.c_int, [_VP, _VP, _VP, _I64, _I64, _I32, _VP, _VP, C.POINTER(CArgs),
                                       _I64, _D, _VP, _VP, _U32, _VP, _VP, C.POINTER(CStats),
                                       C.POINTER(CLogRow), _I64]),
    "culamp_lamp_host": (C.c_int, [_VP, _VP, _VP, _I64, _I64, _I32, _VP, _VP, C.POINTER(CArgs), _I64,
                                   _D, _U32, _VP, _VP, _VP, _VP, C.POINTER(CStats),
                                   C.POINTER(CLogRow), _I64]),
    "culamp_probe_pipes": (C.c_int, [_VP, C.POINTER(_D), _VP]),
    "culamp_probe_wait": (C.c_int, [_VP, C.c_uint64, _VP]),
    "culamp_probe_grid_wait": (C.c_int, [_VP, C.c_uint64, _VP]),
    "culamp_adjoint_sk": (C.c_int, [_VP, _VP, _VP, _VP, _VP, _I64, _I64, _I32, _VP, _VP, _D, _D, _D,
                                    _VP]),
    "culamp_lse_rows_sk_noalloc": (C.c_int, [_VP, _VP, _VP, _I64, _I64, _I32, _VP, _VP, _D, _D, _D,
                                             _VP]),
    "culamp_lse_combine": (C.c_int, [_VP, _VP, _VP, _I32, _I64, _VP]),
    "culamp_batched_sinkhorn": (C.c_int, [_VP, C.POINTER(CInstance), _I32, C.POINTER(CArgs), _I64, _D,
                                          _U32, C.POINTER(CBatchStats), C.POINTER(CBatchInfo), _VP]),
    "culamp_marginal_error_fp64": (C.c_int, [_VP, _VP, _VP, _I64, _I64, _I32, _VP, _VP, _VP, _VP,
                                             _D, _D, _D, C.POINTER(_D), C.POINTER(_D), _VP]),
    "culamp_sinkhorn_dense": (C.c_int, [_VP, _VP, _I64, _I64, _VP, _VP, C.POINTER(CArgs), _I64, _VP,
                                        _VP, _VP, _VP, _VP, C.POINTER(CStats), C.POINTER(CLogRow),
                                        _I64, _VP]),
    "culamp_lamp_dense": (C.c_int, [_VP, _VP, _I64, _I64, _VP, _VP, C.POINTER(CArgs), _I64, _VP, _VP,
                                    _VP, _VP, C.POINTER(CStats), C.POINTER(CLogRow), _I64, _VP]),
}

_lib = None


def load(build_if_missing: bool = True):
    """Load the in-tree library (building it first if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH) and build_if_missing:
        import importlib.util
        spec = importlib.util.spec_from_file_location("_culamp_build", os.path.join(ROOT_DIR, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    if not os.path.exists(LIB_PATH):
        raise CulampError(ERR_UNSUPPORTED, f"libculamp_b200.so not found at {LIB_PATH}; "
                          "run culamp.jl_b200/build.py")
    lib = C.CDLL(LIB_PATH)
    for name, (res, argt) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = argt
    _lib = lib
    return lib


def status_string(code: int) -> str:
    return load().culamp_status_string(code).decode()
