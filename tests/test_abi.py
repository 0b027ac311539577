"""The C ABI library loads on a CPU-only host and exports every symbol that
include/tsvdx4_cuda.h declares; struct layouts agree with the header."""
import ctypes as C
import os
import re

import numpy as np

from netflix_prize_b200 import native
from netflix_prize_b200.abi import TsvdConfig, TsvdDatasetView, TsvdGpuOptions
from netflix_prize_b200.config import TxConfig

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "tsvdx4_cuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tsvd_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = native.load()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), f"missing export {n}"
    assert set(names) == set(native.EXPORTED)


def test_abi_version():
    assert native.load().tsvd_abi_version() == 2


def test_struct_sizes_match_c_layout():
    # computed with the host compiler from the header itself
    import subprocess, tempfile
    code = ('#include "tsvdx4_cuda.h"\n#include <stdio.h>\n#include <stddef.h>\nint main(){printf("%zu %zu %zu %zu %zu\\n",'
            'sizeof(tsvd_config), sizeof(tsvd_dataset_view), sizeof(tsvd_gpu_options),'
            'offsetof(tsvd_config, ordinal_head), offsetof(tsvd_config, full_su));return 0;}')
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(code)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert int(out[0]) == C.sizeof(TsvdConfig)
    assert int(out[1]) == C.sizeof(TsvdDatasetView)
    assert int(out[2]) == C.sizeof(TsvdGpuOptions)
    assert int(out[3]) == TsvdConfig.ordinal_head.offset
    assert int(out[4]) == TsvdConfig.full_su.offset


def test_config_packs_every_field():
    c = TxConfig(n_feat=77, seed=9, lr_iqf=1.5e-6, full_su=False).to_c()
    assert c.n_feat == 77 and c.seed == 9 and abs(c.lr_iqf - 1.5e-6) < 1e-12 and c.full_su == 0


def test_null_arguments_are_rejected_without_touching_a_device():
    L = native.load()
    h = C.c_void_p()
    assert L.tsvd_create(None, None, None, None, C.byref(h)) == 1
    assert L.tsvd_fit_epoch(None, 1) == 1
    assert L.tsvd_predict_batch(None, None, None, None, 0, None) == 1


def test_gpu_options_are_validated_before_any_device_call():
    """Bad options fail at create with TSVD_ERR_INVALID and a message, on a
    host without a GPU as on one with it."""
    L = native.load()
    cfg = TxConfig(n_feat=16).to_c()
    tv, pv = TsvdDatasetView(), TsvdDatasetView()
    for field, value, text in (("schedule", 7, "schedule"), ("precision", 9, "precision"),
                               ("heavy_item_ratings", -1, "heavy_item_ratings")):
        opts = TsvdGpuOptions()
        opts.nsvd_norm_exp = 1.0
        setattr(opts, field, value)
        h = C.c_void_p()
        rc = L.tsvd_create(C.byref(cfg), C.byref(opts), C.byref(tv), C.byref(pv), C.byref(h))
        assert rc == 1, field
        assert text in L.tsvd_last_global_error().decode()
        assert not h.value


def test_heavy_item_threshold_has_its_header_offset():
    import subprocess, tempfile
    code = ('#include "tsvdx4_cuda.h"\n#include <stdio.h>\n#include <stddef.h>\n'
            'int main(){printf("%zu\\n", offsetof(tsvd_gpu_options, heavy_item_ratings));return 0;}')
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(code)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert int(out[0]) == TsvdGpuOptions.heavy_item_ratings.offset
