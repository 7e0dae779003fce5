"""ctypes binding of libmsbg_cuda.so (the C ABI declared in include/msbg_cuda.h).

The library is built in-tree (msbg-rs_b200/_build/libmsbg_cuda.so) by
`make -C msbg-rs_b200/csrc`.  Loading fails loudly when it is missing: there is
no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libmsbg_cuda.so")

MSBG_OK = 0
MSBG_ERR_ARG = 1
MSBG_ERR_OOM = 2
MSBG_ERR_TIMEOUT = 3
MSBG_ERR_CUDA = 4
MSBG_ERR_STATE = 5
MSBG_ERR_NUMERIC = 6

MSBG_F32, MSBG_U16, MSBG_BF16, MSBG_U8, MSBG_F16 = 0, 1, 2, 3, 4
MSBG_LAPLACIAN, MSBG_MEAN_CURVATURE, MSBG_BILAPLACIAN = 0, 1, 2
MSBG_CLAMP, MSBG_NEUMANN, MSBG_DIRICHLET = 0, 1, 2


class MsbgError(RuntimeError):
    """A non-zero status returned by the C ABI."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


_P = C.c_void_p
_U64 = C.c_uint64
_SZ = C.c_size_t
_I = C.c_int
_F = C.c_float
_U64P = C.POINTER(C.c_uint64)
_SZP = C.POINTER(C.c_size_t)

# name -> argtypes (every function returns int status)
SIGNATURES = {
    "msbg_ctx_create": [_I, C.POINTER(_P)],
    "msbg_ctx_destroy": [_P],
    "msbg_ctx_synchronize": [_P],
    "msbg_ctx_stream": [_P, C.POINTER(_P)],
    "msbg_ctx_kernel_launches": [_P, _U64P],
    "msbg_ctx_scratch_bytes": [_P, _U64P],
    "msbg_ctx_set_timing": [_P, _I],
    "msbg_ctx_timing_report": [_P, _I, _P, _SZ, _SZP],
    "msbg_grid_create": [_P, _U64, _U64, _U64, _I, _I, _F, _F, C.POINTER(_P)],
    "msbg_grid_destroy": [_P],
    "msbg_grid_dims": [_P, _U64P],
    "msbg_grid_ensure_blocks": [_P, _P, _SZ],
    "msbg_grid_ensure_blocks_device": [_P, _P, _SZ, _P],
    "msbg_grid_set_full_blocks": [_P, _P, _SZ],
    "msbg_grid_set_empty_blocks": [_P, _P, _SZ],
    "msbg_grid_set_values": [_P, _F, _F],
    "msbg_grid_write_blocks": [_P, _P, _SZ, _P],
    "msbg_grid_write_blocks_device": [_P, _P, _SZ, _P],
    "msbg_grid_read_blocks": [_P, _P, _SZ, _P],
    "msbg_grid_read_blocks_device": [_P, _P, _SZ, _P],
    "msbg_grid_fill_blocks": [_P, _P, _SZ, _F],
    "msbg_grid_value_block_ids": [_P, _P, _SZ, _SZP],
    "msbg_grid_payload": [_P, C.POINTER(_P), _U64P],
    "msbg_grid_slots": [_P, _P, _SZ, _P],
    "msbg_halo_gather": [_P, _P, _SZ, _I, _I, _I, _P],
    "msbg_halo_gather_device": [_P, _P, _SZ, _I, _I, _I, _P],
    "msbg_sweep": [_P, _P, _SZ, _I, _F, _I, _I],
    "msbg_sweep_stochastic": [_P, _P, _SZ, _I, _F, _I, _I, C.c_uint32, _I, _P],
    "msbg_sweep_multires": [_P, _P, _P, _P, _SZ, _I, _F, _I, _I],
    "msbg_morton3": [_P, _P, _SZ, _P],
    "msbg_sort_block_list_morton": [_P, _P, _SZ, _U64, _U64, _P, _SZ, _I],
    "msbg_morton_sort": [_P, _P, _SZ, _P, _P],
    "msbg_morton_sort_device": [_P, _P, _SZ, _P, _P],
    "msbg_morton_sort_noalloc_device": [_P, _P, _SZ, _P, _P],
    "msbg_test_sort_lookback_timeout": [_P, _U64],
    "msbg_permute_device": [_P, _P, _SZ, _I, _P, _P],
    "msbg_bucket_indices": [_P, _P, _SZ, _P, _P, _P, _SZP],
    "msbg_bucket_indices_device": [_P, _P, _SZ, _P, _P, _P, _SZP],
    "msbg_mac_create": [_P, _U64, _U64, _U64, _I, C.POINTER(_P)],
    "msbg_mac_destroy": [_P],
    "msbg_mac_channel": [_P, _I, C.POINTER(_P)],
    "msbg_mac_zero_blocks": [_P, _P, _SZ],
    "msbg_p2g": [_P, _P, _P, _P, _SZ, _F, _SZP],
    "msbg_p2g_device": [_P, _P, _P, _P, _SZ, _F, _SZP],
    "msbg_p2g_sorted_device": [_P, _P, _P, _P, _P, _SZ, _F, _SZP],
    "msbg_p2g_permuted_device": [_P, _P, _P, _P, _P, _P, _SZ, _F, _SZP],
    "msbg_mac_active_blocks": [_P, _P, _SZ, _SZP],
    "msbg_mac_normalize_velocity": [_P, _P, _SZ],
    "msbg_mac_divergence": [_P, _P, _P, _SZ],
    "msbg_g2p": [_P, _P, _SZ, _I, _P],
    "msbg_g2p_device": [_P, _P, _SZ, _I, _P],
    "msbg_g2p_blend_device": [_P, _P, _P, _P, _SZ, _F, _P],
    "msbg_g2p_flip_device": [_P, _P, _SZ, _I, _P, _P, _F, _P],
    "msbg_sample_linear": [_P, _P, _SZ, _I, _I, _P],
    "msbg_sample_ext": [_P, _P, _SZ, _I, _I, _I, _P],
    "msbg_sample_ext_device": [_P, _P, _SZ, _I, _I, _I, _P],
    "msbg_downsample_avg": [_P, _P],
    "msbg_regularize_refinement_map": [_P, _P, _U64, _U64, _U64, _I],
    "msbg_regularize_refinement_map_device": [_P, _P, _U64, _U64, _U64, _I],
    "msbg_block_topology": [_P, _P, _U64, _U64, _U64, _I, _P, _P, _P, _P, _U64P],
    "msbg_blockmap_create": [_P, _U64, C.POINTER(_P)],
    "msbg_blockmap_destroy": [_P],
    "msbg_blockmap_len": [_P, _U64P, _U64P],
    "msbg_blockmap_insert_device": [_P, _P, _P, _SZ],
    "msbg_blockmap_update_add_device": [_P, _P, _SZ],
    "msbg_blockmap_get_device": [_P, _P, _SZ, C.c_uint32, _P],
    "msbg_blockmap_remove_device": [_P, _P, _SZ],
    "msbg_blockmap_sorted_pairs_device": [_P, _P, _P, _SZ, _SZP],
    "msbg_surface_splat_device": [_P, _P, _SZ, _F, _F, _P, _SZ, _SZP],
    "msbg_surface_finalize": [_P, _P, _SZ, _F, _F],
    "msbg_reconstruct_and_smooth": [_P, _P, _SZ, _F, _F, _I, _F, _P, _SZ, _SZP],
    "msbg_place_instances": [_P, _P, _SZ, _P, _F, _U64, _U64, _U64, _F, _SZ, _P, _SZ, _SZP],
    "msbg_flip_create": [_P, _P, _P, _SZ, C.POINTER(_P)],
    "msbg_flip_destroy": [_P],
    "msbg_flip_step": [_P, _P, _P, _P, _SZ, _F, _I, _F, _I, _F, _P],
    "msbg_conv3_forward_device": [_P, _P, C.c_int64, _I, _I, _I, _P, _P, _P, _I, _I, _P],
    "msbg_conv3_wgrad_device": [_P, _P, C.c_int64, _I, _I, _I, _P, _P, _P],
    "msbg_unet_create": [_P, _U64, _U64, _U64, _P, _SZ, _U64, C.POINTER(_P)],
    "msbg_unet_destroy": [_P],
    "msbg_unet_num_params": [_P, _SZP],
    "msbg_unet_layers": [_P, _P, _SZ, _SZP],
    "msbg_unet_get_params": [_P, _P],
    "msbg_unet_set_params": [_P, _P],
    "msbg_unet_get_grads": [_P, _P],
    "msbg_unet_set_output_scale": [_P, _F],
    "msbg_unet_apply_device": [_P, _P, _P],
    "msbg_unet_forward_raw_device": [_P, _P, _P],
    "msbg_unet_train_step_device": [_P, _P, _P, _F, _I, C.POINTER(C.c_double)],
    "msbg_poisson_create": [_P, _U64, _U64, _U64, _I, _P, _SZ, C.POINTER(_P)],
    "msbg_poisson_destroy": [_P],
    "msbg_poisson_levels": [_P, _P, _SZ, _SZP],
    "msbg_poisson_set_smoother": [_P, _I, _I, _F],
    "msbg_poisson_matvec_device": [_P, _P, _P],
    "msbg_poisson_jacobi_device": [_P, _P, _P, _F, _I],
    "msbg_poisson_residual_device": [_P, _P, _P, _P, C.POINTER(C.c_double)],
    "msbg_poisson_vcycle_device": [_P, _P, _P],
    "msbg_poisson_dot_device": [_P, _P, _P, C.POINTER(C.c_double)],
    "msbg_poisson_solve_device": [_P, _I, _P, _P, C.c_double, _I, C.POINTER(_I), C.POINTER(C.c_double), _P],
    "msbg_poisson_solve": [_P, _I, _P, _P, C.c_double, _I, C.POINTER(_I), C.POINTER(C.c_double), _P],
    "msbg_poisson_set_preconditioner": [_P, _P],
    "msbg_poisson_set_network_lead": [_P, _I],
    "msbg_poisson_autotune": [_P, _P, _SZ, _SZP],
    "msbg_poisson_set_tuning": [_P, _P, _SZ],
    "msbg_batch_create": [_P, _I, _P, _P, _P, _P, _I, C.POINTER(_P)],
    "msbg_batch_destroy": [_P],
    "msbg_batch_groups": [_P, C.POINTER(_I)],
    "msbg_batch_problem": [_P, _I, C.POINTER(_I), _U64P, _U64P],
    "msbg_batch_buffers": [_P, _I, C.POINTER(_P), C.POINTER(_P), _U64P, C.POINTER(_I)],
    "msbg_batch_set_rhs": [_P, _I, _P],
    "msbg_batch_get_solution": [_P, _I, _P],
    "msbg_batch_tuning": [_P, _I, _P, _P, _SZ, _SZP],
    "msbg_batch_solve": [_P, C.c_double, _I, _I, _I, _P, _P, C.POINTER(_I)],
    "msbg_poisson_solve_f64_device": [_P, _I, _P, _P, C.c_double, _I, C.POINTER(_I), C.POINTER(C.c_double), _P],
    "msbg_poisson_solve_stats": [_P, _P],
    "msbg_poisson_rhs_device": [_P, _U64, _I, _P],
    "msbg_poisson_train_preconditioner": [_P, _I, _I, _I, _I, _F, _I, _U64, _P, C.c_int64, C.POINTER(C.c_int64)],
    "msbg_poisson_eval_preconditioner": [_P, _I, _I, _U64, _P],
}

_lib = None


def lib() -> C.CDLL:
    """Loads the C-ABI library (once).  Raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libmsbg_cuda.so not found at {LIB_PATH}; build it with `make -C msbg-rs_b200/csrc`"
            )
        h = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(h, name)
            f.argtypes = args
            f.restype = C.c_int
        h.msbg_status_string.argtypes = [C.c_int]
        h.msbg_status_string.restype = C.c_char_p
        h.msbg_last_error.argtypes = []
        h.msbg_last_error.restype = C.c_char_p
        _lib = h
    return _lib


def check(status: int) -> None:
    if status != MSBG_OK:
        h = lib()
        msg = h.msbg_last_error().decode() or h.msbg_status_string(status).decode()
        raise MsbgError(status, msg)


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))


def ptr(a) -> C.c_void_p:
    """Pointer to a contiguous numpy array's data (or a torch tensor's)."""
    if a is None:
        return C.c_void_p(0)
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the C ABI must be C-contiguous"
    return C.c_void_p(a.ctypes.data)
