"""culamp_b200 -- Python host API of libculamp_b200 (B200 / sm_100a).

A drop-in for CuLAMP.jl's kernelized entropic-OT path: the `sinkhorn`, `lamp`
and `annealed_sinkhorn` `--kernel` solvers and their pass-level kernels, with
the reference's function names, EOTArgs settings and file formats. All compute
runs in libculamp_b200.so (hand-written CUDA for sm_100a); there is no CPU path.
"""
from ._lib import (CulampError, FLAG_CHECK_ALWAYS, FLAG_FEAT_FP64, FLAG_FEAT_X6, FLAG_FORM_FP32,
                   FLAG_FORM_FP64, FLAG_FORM_PLAIN, FLAG_LADDER, FLAG_MARGINAL_ONLY, FLAG_NO_GRAPH,
                   FLAG_NO_PERSIST, FLAG_TRUE_PINF,
                   LIB_PATH, load)
from .args import EOTArgs, args_from_json_string, default_args, read_args_json
from .solvers import (BatchResult, Handle, SolveResult, annealed_sinkhorn_euclidean, barycentric_map,
                      extragradient_color_transfer, extragradient_euclidean, get_handle,
                      lamp_barycentric_maps, marginal_error_fp64, sinkhorn_color_transfer,
                      sinkhorn_euclidean, solve_annealed_sinkhorn, solve_batched_sinkhorn, solve_lamp,
                      solve_sinkhorn, solve_symmetric_sinkhorn)
from . import kernels

__all__ = [
    "BatchResult", "CulampError", "EOTArgs", "Handle", "SolveResult", "LIB_PATH", "load",
    "FLAG_CHECK_ALWAYS", "FLAG_FEAT_FP64", "FLAG_FEAT_X6", "FLAG_FORM_FP32", "FLAG_FORM_FP64",
    "FLAG_FORM_PLAIN", "FLAG_LADDER", "FLAG_MARGINAL_ONLY", "FLAG_NO_GRAPH", "FLAG_NO_PERSIST",
    "FLAG_TRUE_PINF",
    "args_from_json_string", "default_args", "read_args_json",
    "annealed_sinkhorn_euclidean", "barycentric_map", "extragradient_color_transfer",
    "extragradient_euclidean", "get_handle", "lamp_barycentric_maps", "marginal_error_fp64",
    "sinkhorn_color_transfer", "sinkhorn_euclidean", "solve_annealed_sinkhorn", "solve_lamp",
    "solve_batched_sinkhorn", "solve_sinkhorn", "solve_symmetric_sinkhorn", "kernels",
]
