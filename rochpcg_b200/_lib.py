"""ctypes binding of libhpcgb200.so (the C ABI of include/hpcg_b200.h)."""
from __future__ import annotations

import ctypes
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libhpcgb200.so")

_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_ll = ctypes.c_longlong
_sz = ctypes.c_size_t
_cp = ctypes.c_char_p

# name -> (restype, argtypes)
SIGNATURES = {
    "hpcgb200_last_error": (_cp, []),
    "hpcgb200_version": (_cp, []),
    "hpcgb200_init": (_i, [_i]),
    "hpcgb200_reduction_workspace_bytes": (_sz, []),
    "hpcgb200_rand_sequence": (_i, [ctypes.c_uint, _i, _vp]),
    "hpcgb200_generate_problem": (_i, [_i, _i, _i, _ll, _ll, _ll, _ll, _ll, _ll, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                       _vp]),
    "hpcgb200_f2c_operator": (_i, [_i, _i, _i, _vp, _vp, _vp]),
    "hpcgb200_coloring_workspace_bytes": (_sz, [_i]),
    "hpcgb200_jpl_coloring": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "hpcgb200_build_ell": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_extract_diagonal": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_permute_vector": (_i, [_i, _vp, _vp, _vp, _vp]),
    "hpcgb200_unpermute_vector": (_i, [_i, _vp, _vp, _vp, _vp]),
    "hpcgb200_copy_diagonal": (_i, [_i, _vp, _vp, _vp, _vp]),
    "hpcgb200_replace_diagonal": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_testcg_scale": (_i, [_i, _vp, _vp, _vp, _vp]),
    "hpcgb200_transfer_indices": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_spmv": (_i, [_i, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_symgs": (_i, [_i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_symgs_zero": (_i, [_i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_restrict_fused": (_i, [_i, _vp, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_restrict": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_prolong": (_i, [_i, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_dot": (_i, [_i, _vp, _vp, _vp, _vp, _sz, _vp]),
    "hpcgb200_dot_noalloc": (_i, [_ll, _vp, _vp, _vp, _vp]),
    "hpcgb200_selftest_grid_barrier": (_i, [_i, _vp, _vp, _vp]),
    "hpcgb200_waxpby": (_i, [_i, _d, _vp, _d, _vp, _vp, _vp]),
    "hpcgb200_waxpby_dot": (_i, [_i, _d, _vp, _vp, _vp, _vp, _sz, _vp]),
    "hpcgb200_residual_inf": (_i, [_i, _vp, _vp, _vp, _vp, _sz, _vp]),
    "hpcgb200_conv_weight_tile_bytes": (_sz, []),
    "hpcgb200_conv_prepare_weights": (_i, [_vp, _vp, _i, _vp]),
    "hpcgb200_conv16": (_i, [_i, _i, _i, _i, _vp, _vp, _i, _vp, _vp, _vp, _vp]),
    "hpcgb200_conv_wgrad_partial_bytes": (_sz, [_i, _i, _i, _i]),
    "hpcgb200_conv16_wgrad": (_i, [_i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_smoother_create": (_i, [_vp]),
    "hpcgb200_smoother_destroy": (_i, [_vp]),
    "hpcgb200_smoother_set_weights": (_i, [_vp, _vp]),
    "hpcgb200_smoother_get_weights": (_i, [_vp, _vp]),
    "hpcgb200_smoother_init_jacobi": (_i, [_vp, ctypes.c_float, ctypes.c_float, ctypes.c_ulonglong, _i]),
    "hpcgb200_smoother_forward": (_i, [_vp, _i, _i, _i, _i, _vp, _vp, _vp]),
    "hpcgb200_smoother_configure": (_i, [_vp, _i]),
    "hpcgb200_smoother_loss_grad": (_i, [_vp, _i, _i, _i, _i, _vp, _vp, _vp, ctypes.c_float, _i, _vp, _vp, _vp]),
    "hpcgb200_sample_norms": (_i, [_i, _i, _i, _i, _vp, _i, _vp, _vp]),
    "hpcgb200_smoother_adam_step": (_i, [_vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, _vp]),
    "hpcgb200_smoother_train": (_i, [_vp, _vp, _i, _i, ctypes.c_float, ctypes.c_float, _i, ctypes.c_ulonglong,
                                     _vp, _vp]),
    "hpcgb200_make_training_pairs": (_i, [_i, _i, ctypes.c_ulonglong, _i, _vp, _vp, _vp, _d]),
    "hpcgb200_normal_rhs": (_i, [_ll, ctypes.c_ulonglong, _vp, _vp]),
    "hpcgb200_problem_set_smoother": (_i, [_vp, _vp, _i, _i]),
    "hpcgb200_problem_last_fallback": (_i, [_vp, _vp]),
    "hpcgb200_problem_create": (_i, [_i, _i, _i, _i, _vp]),
    "hpcgb200_problem_create_ex": (_i, [_i, _i, _i, _i, _i, _vp]),
    "hpcgb200_problem_destroy": (_i, [_vp]),
    "hpcgb200_problem_info": (_i, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_problem_setup_times": (_i, [_vp, _vp, _vp]),
    "hpcgb200_problem_stream": (_i, [_vp, _vp]),
    "hpcgb200_problem_stencil_ok": (_i, [_vp, _i, _vp]),
    "hpcgb200_problem_copy_field": (_i, [_vp, _i, _cp, _vp, _sz]),
    "hpcgb200_problem_field_bytes": (_i, [_vp, _i, _cp, _vp]),
    "hpcgb200_problem_device_field": (_i, [_vp, _i, _cp, _vp]),
    "hpcgb200_problem_set_rhs": (_i, [_vp, _vp]),
    "hpcgb200_problem_get_x": (_i, [_vp, _vp]),
    "hpcgb200_problem_cg": (_i, [_vp, _i, _i, _d, _i, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_problem_solve_host": (_i, [_vp, _i, _vp, _vp, _i, _d, _vp, _vp, _vp, _vp]),
    "hpcgb200_problem_true_residual": (_i, [_vp, _vp]),
    "hpcgb200_problem_cg_ref": (_i, [_vp, _i, _d, _i, _vp, _vp, _vp, _vp]),
    "hpcgb200_problem_set_fallback": (_i, [_vp, _d, _i, _i, _d]),
    "hpcgb200_problem_mg_ref": (_i, [_vp, _vp, _vp]),
    "hpcgb200_ref_spmv": (_i, [_i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_ref_symgs": (_i, [_i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_benchmark_run": (_i, [_vp, _vp]),
    "hpcgb200_benchmark_report": (_i, [_vp, _vp, _sz, _vp]),
    "hpcgb200_problem_kernels_per_iteration": (_i, [_vp, _i, _i, _vp]),
    "hpcgb200_problem_test_cg": (_i, [_vp, _i, _vp, _vp, _vp]),
    "hpcgb200_problem_test_symmetry": (_i, [_vp, _i, _vp, _vp, _vp]),
    "hpcgb200_problem_spmv": (_i, [_vp, _i, _vp, _vp]),
    "hpcgb200_problem_spmv_stencil": (_i, [_vp, _i, _vp, _vp]),
    "hpcgb200_problem_spmv_mixed": (_i, [_vp, _i, _vp, _vp]),
    "hpcgb200_problem_symgs": (_i, [_vp, _i, _vp, _vp]),
    "hpcgb200_problem_symgs_zero": (_i, [_vp, _i, _vp, _vp]),
    "hpcgb200_problem_mg": (_i, [_vp, _i, _vp, _vp]),
    "hpcgb200_problem_restrict": (_i, [_vp, _i, _vp, _vp, _vp]),
    "hpcgb200_problem_prolong": (_i, [_vp, _i, _vp, _vp]),
    "hpcgb200_problem_time_op": (_i, [_vp, _cp, _i, _vp]),
    # domain decomposition
    "hpcgb200_dist_shape": (_i, [_i, _vp, _vp, _vp]),
    "hpcgb200_geometry": (_i, [_i] * 11 + [_vp]),
    "hpcgb200_halo_plan_create": (_i, [_i, _i, _i, _i, _i, _i, _i, _i, _vp]),
    "hpcgb200_halo_plan_info": (_i, [_vp, _vp]),
    "hpcgb200_halo_plan_copy": (_i, [_vp, _cp, _vp, _sz]),
    "hpcgb200_halo_plan_destroy": (_i, [_vp]),
    "hpcgb200_dist_create": (_i, [_i, _i, _i, _i, _i, _i, _i, _i, _i, _vp]),
    "hpcgb200_dist_destroy": (_i, [_vp]),
    "hpcgb200_dist_info": (_i, [_vp, _i, _vp, _vp]),
    "hpcgb200_dist_copy_field": (_i, [_vp, _i, _cp, _vp, _sz]),
    "hpcgb200_dist_set_rhs": (_i, [_vp, _vp]),
    "hpcgb200_dist_get_x": (_i, [_vp, _vp]),
    "hpcgb200_dist_nccl_available": (_i, []),
    "hpcgb200_dist_nccl_id": (_i, [_vp, _sz]),
    "hpcgb200_dist_attach_nccl": (_i, [_vp, _vp, _sz]),
    "hpcgb200_dist_group_spmv": (_i, [_vp, _i, _i, _vp, _vp]),
    "hpcgb200_dist_group_symgs": (_i, [_vp, _i, _i, _vp, _vp]),
    "hpcgb200_dist_group_restrict": (_i, [_vp, _i, _i, _vp, _vp, _vp]),
    "hpcgb200_dist_group_mg": (_i, [_vp, _i, _vp, _vp]),
    "hpcgb200_dist_group_cg": (_i, [_vp, _i, _i, _d, _i, _vp, _vp, _vp, _vp, _vp]),
    "hpcgb200_dist_cg": (_i, [_vp, _i, _d, _i, _vp, _vp, _vp, _vp, _vp]),
}

_lib = None


class HpcgError(RuntimeError):
    def __init__(self, lib, code: int):
        msg = lib.hpcgb200_last_error().decode(errors="replace") if lib is not None else ""
        super().__init__(f"libhpcgb200 error {code}: {msg}")
        self.code = code


def check(lib, rc: int):
    if rc != 0:
        raise HpcgError(lib, rc)


def load(path: str | None = None):
    """Load the CUDA library; raises when it has not been built (there is no
    CPU implementation to fall back to)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(f"{p} is missing: build it with `python -m rochpcg_b200.build` "
                          "(the solver runs only on the CUDA path)")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib
