"""Loader for the in-tree CUDA library libtsvdx4_cuda.so (C ABI in
include/tsvdx4_cuda.h). There is no CPU fallback: if the library is missing
this module raises, and every model call needs a visible sm_100 device."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from .abi import TsvdConfig, TsvdDatasetView, TsvdGpuOptions

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "_lib", "libtsvdx4_cuda.so")
CSRC = os.path.join(PKG, "csrc")

# Every symbol include/tsvdx4_cuda.h declares.
EXPORTED = [
    "tsvd_create", "tsvd_destroy", "tsvd_n_epochs", "tsvd_fit_epoch", "tsvd_predict_batch",
    "tsvd_predict_batch_device", "tsvd_n_subscores", "tsvd_subscore_name", "tsvd_predict_subscores_batch",
    "tsvd_gen_preds", "tsvd_calc_rmse", "tsvd_param_nbytes", "tsvd_get_param", "tsvd_set_param",
    "tsvd_rebuild_ycache", "tsvd_set_user_order", "tsvd_get_user_order", "tsvd_set_stream", "tsvd_synchronize",
    "tsvd_set_profiling", "tsvd_kernel_stats", "tsvd_reset_kernel_stats", "tsvd_launch_count", "tsvd_last_error",
    "tsvd_last_global_error", "tsvd_abi_version", "tsvd_user_order_for_seed", "tsvd_normal_stream",
    "tsvd_calc_rmse_device_noalloc",
    "tsvd_group_create", "tsvd_group_destroy", "tsvd_group_size", "tsvd_group_model", "tsvd_group_fit_epoch",
    "tsvd_group_set_graphs", "tsvd_group_last_epoch_ms", "tsvd_group_autotune", "tsvd_group_last_error",
    "tsvd_encoder_create", "tsvd_encoder_destroy", "tsvd_encoder_train_epoch", "tsvd_encoder_loss_grad",
    "tsvd_encoder_forward", "tsvd_encoder_apply", "tsvd_encoder_get", "tsvd_encoder_set",
    "tsvd_encoder_target_stats", "tsvd_encoder_last_error", "tsvd_foldin", "tsvd_reset_users",
    "tsvd_shard_user_block", "tsvd_shard_apply", "tsvd_shard_item_block", "tsvd_copy_rows", "tsvd_user_day_range",
    "tsvd_row_width",
]

_lib = None


def build(jobs: int = 8) -> str:
    """Compile the CUDA sources for sm_100a with nvcc (no GPU needed)."""
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", CSRC], check=True)
    return LIB_PATH


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA library not built: {LIB_PATH} is missing (run netflix_prize_b200.native.build())")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    L.tsvd_create.argtypes = [C.POINTER(TsvdConfig), C.POINTER(TsvdGpuOptions), C.POINTER(TsvdDatasetView),
                              C.POINTER(TsvdDatasetView), C.POINTER(P)]
    L.tsvd_destroy.argtypes = [P]
    L.tsvd_destroy.restype = None
    L.tsvd_n_epochs.argtypes = [P, C.POINTER(C.c_uint64)]
    L.tsvd_fit_epoch.argtypes = [P, C.c_uint64]
    L.tsvd_predict_batch.argtypes = [P, P, P, P, C.c_uint64, P]
    L.tsvd_predict_batch_device.argtypes = [P, P, P, P, C.c_uint64, P]
    L.tsvd_n_subscores.argtypes = [P, C.POINTER(C.c_uint64)]
    L.tsvd_subscore_name.argtypes = [P, C.c_uint64]
    L.tsvd_subscore_name.restype = C.c_char_p
    L.tsvd_predict_subscores_batch.argtypes = [P, P, P, P, C.c_uint64, P]
    L.tsvd_gen_preds.argtypes = [P, C.POINTER(TsvdDatasetView), P]
    L.tsvd_calc_rmse.argtypes = [P, C.POINTER(TsvdDatasetView), C.POINTER(C.c_double)]
    L.tsvd_param_nbytes.argtypes = [P, C.c_char_p, C.POINTER(C.c_uint64)]
    L.tsvd_get_param.argtypes = [P, C.c_char_p, P, C.c_uint64]
    L.tsvd_set_param.argtypes = [P, C.c_char_p, P, C.c_uint64]
    L.tsvd_rebuild_ycache.argtypes = [P]
    L.tsvd_set_user_order.argtypes = [P, C.c_uint64, P, C.c_uint64]
    L.tsvd_get_user_order.argtypes = [P, C.c_uint64, P, C.c_uint64]
    L.tsvd_set_stream.argtypes = [P, P]
    L.tsvd_synchronize.argtypes = [P]
    L.tsvd_set_profiling.argtypes = [P, C.c_int32]
    L.tsvd_kernel_stats.argtypes = [P, C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_double)]
    L.tsvd_reset_kernel_stats.argtypes = [P]
    L.tsvd_launch_count.argtypes = [P, C.POINTER(C.c_uint64)]
    L.tsvd_last_error.argtypes = [P]
    L.tsvd_last_error.restype = C.c_char_p
    L.tsvd_last_global_error.argtypes = []
    L.tsvd_last_global_error.restype = C.c_char_p
    L.tsvd_abi_version.argtypes = []
    L.tsvd_user_order_for_seed.argtypes = [C.c_uint64, C.c_int32, C.c_uint64, C.c_uint64, P]
    L.tsvd_normal_stream.argtypes = [C.c_uint64, C.c_float, C.c_uint64, P]
    L.tsvd_calc_rmse_device_noalloc.argtypes = [P, P, P, P, P, P, C.c_uint64, P]
    L.tsvd_group_create.argtypes = [P, C.c_uint32, C.POINTER(TsvdGpuOptions), C.POINTER(TsvdDatasetView),
                                    C.POINTER(TsvdDatasetView), C.POINTER(P)]
    L.tsvd_group_destroy.argtypes = [P]
    L.tsvd_group_destroy.restype = None
    L.tsvd_group_size.argtypes = [P, C.POINTER(C.c_uint32)]
    L.tsvd_group_model.argtypes = [P, C.c_uint32, C.POINTER(P)]
    L.tsvd_group_fit_epoch.argtypes = [P, C.c_uint64]
    L.tsvd_group_set_graphs.argtypes = [P, C.c_int32]
    L.tsvd_group_last_epoch_ms.argtypes = [P, C.POINTER(C.c_double)]
    L.tsvd_group_autotune.argtypes = [P, C.c_uint32, P]
    L.tsvd_group_last_error.argtypes = [P]
    L.tsvd_group_last_error.restype = C.c_char_p
    L.tsvd_shard_user_block.argtypes = [P, C.c_uint64, C.c_uint32, C.c_uint32, P, P, P]
    L.tsvd_shard_apply.argtypes = [P, P, P, P]
    L.tsvd_shard_item_block.argtypes = [P, C.c_uint32, C.c_uint32]
    L.tsvd_copy_rows.argtypes = [P, C.c_char_p, C.c_uint64, C.c_uint64, P, C.c_int32]
    L.tsvd_user_day_range.argtypes = [P, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.tsvd_row_width.argtypes = [P, C.POINTER(C.c_uint32)]
    _lib = L
    return L


class TsvdError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"tsvd status {status}: {msg}")
        self.status = status
