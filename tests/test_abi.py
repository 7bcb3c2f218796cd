"""The C-ABI library loads without a GPU and exports every entry point that
include/relight_b200.h declares (no compute calls are made here)."""
import ctypes as C
import os
import re

from relight_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "relight_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rl_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for must in ("rl_scene_create", "rl_trace_segments", "rl_bake_direct", "rl_bake_ao", "rl_emit_photons",
                 "rl_photonmap_gather", "rl_bake_indirect", "rl_ff_pairwise", "rl_ff_hemisphere",
                 "rl_radiosity_solve", "rl_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_abi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert sorted(_abi.SIGNATURES) == declared_functions()
    _abi.load()


def test_version_and_error_text_without_gpu():
    lib = _abi.load()
    assert b"sm_100a" in lib.rl_version()
    buf = C.create_string_buffer(64)
    assert lib.rl_last_error(buf, 64) >= 0


def test_tune_parameters_are_checked_without_gpu():
    """rl_tune_set keeps each parameter within its documented range and
    changes nothing on a refusal."""
    lib = _abi.load()
    v = C.c_int()
    assert lib.rl_tune_get(_abi.TUNE_KNN_CELL, C.byref(v)) == 0 and v.value == 80
    for bad in (7, 257, 0, -1):
        assert lib.rl_tune_set(_abi.TUNE_KNN_CELL, bad) != 0
    assert lib.rl_tune_get(_abi.TUNE_KNN_CELL, C.byref(v)) == 0 and v.value == 80
    assert lib.rl_tune_set(_abi.TUNE_KNN_CELL, 48) == 0
    assert lib.rl_tune_get(_abi.TUNE_KNN_CELL, C.byref(v)) == 0 and v.value == 48
    assert lib.rl_tune_set(_abi.TUNE_KNN_CELL, 80) == 0
    assert lib.rl_tune_get(_abi.TUNE_AO_SPLIT, C.byref(v)) == 0 and v.value == 0
    for bad in (3, 16, -1):
        assert lib.rl_tune_set(_abi.TUNE_AO_SPLIT, bad) != 0
    assert lib.rl_tune_get(_abi.TUNE_FG_POOL, C.byref(v)) == 0 and v.value == 0
    for bad in (2, -1):
        assert lib.rl_tune_set(_abi.TUNE_FG_POOL, bad) != 0
    assert lib.rl_tune_get(_abi.TUNE_FG_CHUNK, C.byref(v)) == 0 and v.value == 32
    for bad in (7, 257, 0):
        assert lib.rl_tune_set(_abi.TUNE_FG_CHUNK, bad) != 0
    assert lib.rl_tune_get(_abi.TUNE_FG_CHUNK, C.byref(v)) == 0 and v.value == 32
    assert lib.rl_tune_get(_abi.TUNE_FG_CHUNK + 1, C.byref(v)) != 0
    assert lib.rl_tune_set(_abi.TUNE_BVH_WIDTH, 3) != 0
