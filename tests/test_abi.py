"""The C-ABI library loads without a GPU and exports every function that
include/msbg_cuda.h declares; argument validation runs on the host."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "msbg_cuda.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(msbg_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["msbg_ctx_create", "msbg_grid_create", "msbg_sweep", "msbg_halo_gather", "msbg_morton_sort",
                 "msbg_bucket_indices", "msbg_p2g", "msbg_g2p", "msbg_downsample_avg"]:
        assert must in names


def test_library_exports_every_declared_symbol(msbg):
    h = msbg._lib.lib()
    missing = [n for n in declared_functions() if not hasattr(h, n)]
    assert not missing, missing
    # The Python binding covers every declared entry point too.
    extra = set(declared_functions()) - set(msbg._lib.SIGNATURES) - {"msbg_status_string", "msbg_last_error"}
    assert not extra, extra


def test_status_strings(msbg):
    h = msbg._lib.lib()
    assert h.msbg_status_string(0) == b"ok"
    assert h.msbg_status_string(1) == b"invalid argument"


def test_null_arguments_rejected_without_gpu(msbg):
    h = msbg._lib.lib()
    assert h.msbg_ctx_create(0, None) == msbg._lib.MSBG_ERR_ARG
    assert h.msbg_grid_create(None, 16, 16, 16, 16, 0, 0.0, 1.0, None) == msbg._lib.MSBG_ERR_ARG
    assert h.msbg_sweep(None, None, 0, 0, 0.0, 1, 0) == msbg._lib.MSBG_ERR_ARG
    assert b"null" in h.msbg_last_error()
