"""The C-ABI library builds, loads and exports every entry point that
include/genomics_b200.h declares.  CPU only: no call here needs a GPU."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "genomics_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gb2_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("gb2_create", "gb2_destroy", "gb2_batch_upload", "gb2_batch_free",
                 "gb2_sw_banded", "gb2_sw_banded_host", "gb2_sw_pair", "gb2_wfa_affine",
                 "gb2_wfa_affine_host", "gb2_wfa_pair", "gb2_strerror", "gb2_version"):
        assert must in names


def test_library_exports_every_declared_symbol(built_lib):
    out = subprocess.check_output(["nm", "-D", "--defined-only", built_lib], text=True)
    exported = set(re.findall(r"\bT (gb2_[a-z0-9_]+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing


def test_library_loads_and_binding_covers_header(built_lib):
    from genomics_b200 import _lib
    L = _lib.lib()
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(declared_functions()) == bound
    for name in bound:
        assert hasattr(L, name)
    assert L.gb2_version() == 100
    assert L.gb2_strerror(0) == b"ok"
    assert L.gb2_strerror(-1) == b"invalid argument"
    assert L.gb2_strerror(-5) == b"input outside the exact integer range"


def test_flag_and_status_constants_match_header():
    """The Python binding's flag bits and status codes are the header's."""
    from genomics_b200 import _lib
    text = open(HEADER).read()
    defines = {name: int(val, 0) for name, val in
               re.findall(r"#define (GB2_(?:FLAG_[A-Z0-9_]+|E[A-Z]+|OK))\s+\(?(-?(?:0x)?[0-9a-fA-F]+)",
                          text)}
    flags = {k: v for k, v in defines.items() if k.startswith("GB2_FLAG_")}
    assert "GB2_FLAG_PACKED" in flags and len(flags) >= 8
    for name, val in flags.items():
        assert getattr(_lib, name[len("GB2_"):]) == val, name
    assert len(set(flags.values())) == len(flags)  # no two flags share a bit
    for name, val in defines.items():
        if not name.startswith("GB2_FLAG_"):
            assert getattr(_lib, name) == val, name


def test_struct_layouts_match_header(built_lib):
    from genomics_b200 import _lib
    assert ctypes.sizeof(_lib.SwCfg) == 20
    assert ctypes.sizeof(_lib.SwResult) == 12
    assert ctypes.sizeof(_lib.WfaCfg) == 16


def test_null_arguments_rejected_without_gpu(built_lib):
    from genomics_b200 import _lib
    L = _lib.lib()
    assert L.gb2_create(0, None) == _lib.GB2_EINVAL
    assert L.gb2_destroy(None) == _lib.GB2_EINVAL
    assert L.gb2_sync(None) == _lib.GB2_EINVAL
    assert L.gb2_sw_pair(None, None, 0, None, 0, None, None) == _lib.GB2_EINVAL
    assert L.gb2_batch_info(None, None, None) == _lib.GB2_EINVAL
    res = _lib.TuneResult()
    assert L.gb2_autotune(None, _lib.GB2_TUNE_SW, None, None, None, None, 1, 1,
                          ctypes.byref(res)) == _lib.GB2_EINVAL
    v = ctypes.c_int()
    assert L.gb2_tune_set(None, _lib.GB2_TUNE_SW, 32, 1) == _lib.GB2_EINVAL
    assert L.gb2_tune_get(None, _lib.GB2_TUNE_WFA, 0, ctypes.byref(v)) == _lib.GB2_EINVAL


def test_tune_result_layout(built_lib):
    """gb2_tune_result: 4 int32, then GB2_TUNE_MAX int32 variants and floats."""
    from genomics_b200 import _lib
    assert ctypes.sizeof(_lib.TuneResult) == 4 * 4 + _lib.GB2_TUNE_MAX * 8


def test_sources_compile_for_sm100a():
    """The CUDA sources target sm_100a only (no other arch in the build)."""
    from genomics_b200 import _build
    flags = " ".join(_build.NVCC_FLAGS)
    assert "arch=compute_100a,code=sm_100a" in flags
    assert "sm_90" not in flags and "sm_80" not in flags
