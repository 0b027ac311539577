"""ctypes mirrors of the C ABI structs in include/tsvdx4_cuda.h.

`TsvdConfig` is TxConfig (src/tx.rs:128-204) field for field; `TsvdDatasetView`
borrows the arrays of a Dataset (src/lib.rs:227-242) or of a MaskedDataset
(src/lib.rs:421-455, ratings and residuals NULL).
"""
from __future__ import annotations

import ctypes as C

TSVD_OK = 0
TSVD_ERR_INVALID = 1
TSVD_ERR_UNSUPPORTED = 2
TSVD_ERR_CUDA = 3
TSVD_ERR_NO_DEVICE = 4
TSVD_ERR_OOM = 5
TSVD_ERR_TIMEOUT = 6

SCHED_STRATIFIED = 0
SCHED_HOGWILD = 1
SCHED_SEQUENTIAL = 2
PREC_FP32 = 0
PREC_BF16_READ = 1
PREC_BF16_READ_ALL = 2


class TsvdOrdinalConfig(C.Structure):
    _fields_ = [
        ("th_init", C.c_float * 4),
        ("th_gap", C.c_float),
        ("lr_t", C.c_float),
        ("reg_t", C.c_float),
    ]


_F = C.c_float
_U64 = C.c_uint64
_I32 = C.c_int32

CONFIG_FIELDS = [
    ("n_feat", _U64), ("n_epochs", _U64), ("seed", _U64), ("shuffle_users", _I32),
    ("n_time_bins", _U64), ("beta", _F), ("n_freq_bins", _U64),
    ("lr_u", _F), ("lr_ud", _F), ("lr_u2", _F), ("lr_ub", _F), ("lr_ubd", _F),
    ("lr_i", _F), ("lr_ib", _F), ("lr_y", _F), ("lr_yb", _F), ("lr_yd", _F),
    ("lr_tu", _F), ("lr_ti", _F), ("lr_ta", _F), ("lr_ibf", _F), ("lr_iqf", _F), ("lr_cu", _F),
    ("reg_iqf", _F), ("reg_cu", _F), ("reg_u", _F), ("reg_u2", _F), ("reg_ud", _F),
    ("reg_i", _F), ("reg_y", _F), ("reg_yd", _F),
    ("sigma_iqf", _F), ("sigma_u", _F), ("sigma_i", _F), ("sigma_y", _F), ("sigma_yd", _F),
    ("reset_u_epoch", _U64),
    ("max_neighbors", _U64),
    ("lr_w", _F), ("lr_c", _F), ("reg_w", _F), ("reg_c", _F),
    ("lr_w_day", _F), ("lr_c_day", _F), ("reg_w_day", _F), ("reg_c_day", _F),
    ("w_bias", _F), ("w_factor", _F), ("w_nbr", _F),
    ("sum_err_bug", _I32), ("lambda1", _F), ("lambda2", _F),
    ("has_ordinal_head", _I32), ("ordinal_head", TsvdOrdinalConfig),
    ("save_ifeat", _I32), ("low_memory", _I32), ("full_su", _I32),
]


class TsvdConfig(C.Structure):
    _fields_ = CONFIG_FIELDS


class TsvdDatasetView(C.Structure):
    _fields_ = [
        ("user_idxs", C.POINTER(C.c_int32)),
        ("user_cnts", C.POINTER(C.c_int32)),
        ("item_idxs", C.POINTER(C.c_int32)),
        ("item_cnts", C.POINTER(C.c_int32)),
        ("raw_ratings", C.POINTER(C.c_int8)),
        ("residuals", C.POINTER(C.c_float)),
        ("dates", C.POINTER(C.c_int16)),
        ("is_test", C.POINTER(C.c_int8)),
        ("n_users", C.c_uint64),
        ("n_items", C.c_uint64),
        ("n_ratings", C.c_uint64),
    ]


class TsvdGpuOptions(C.Structure):
    _fields_ = [
        ("schedule", C.c_int32),
        ("precision", C.c_int32),
        ("nsvd_norm_exp", C.c_float),
        ("device", C.c_int32),
        ("warps_per_block", C.c_int32),
        ("heavy_item_ratings", C.c_int32),
        ("seq_epochs", C.c_int32 * 5),
        ("reserved", C.c_int32 * 2),
    ]


def ptr(arr, ctype):
    """Pointer to a contiguous numpy array (None -> NULL)."""
    if arr is None:
        return C.cast(None, C.POINTER(ctype))
    assert arr.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return arr.ctypes.data_as(C.POINTER(ctype))
