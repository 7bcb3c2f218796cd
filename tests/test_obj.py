"""OBJ ingest: rl_obj_load / Mesh.create_from_file against the reference's
own MeshLoader (Mesh::createFromFile, scene/MeshLoader.cpp:44-226).

The synthetic files of make_golden.obj_texts() cover submeshes, quads,
shared and -0.0 / 0.0 corners, uv clamping, octal / hex / signed indices,
CRLF endings, a missing final newline and position-only faces; their
reference outputs are committed in golden/obj.npz.  Where the reference
build is present, the reference's own sample meshes are compared live.
All comparisons are bit for bit.  Host-only: no GPU involved.
"""
import ctypes as C
import glob
import os
import sys

import numpy as np
import pytest

import oracle_bind as ob
from relight_b200 import _abi
from relight_b200.api import Mesh

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_golden import obj_texts  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "obj.npz"))
_REF_ROOT = ob.reference_root()
REF_DATA = os.path.join(_REF_ROOT, "data") if _REF_ROOT else None


def _load(path):
    L = _abi.lib()
    h = C.c_void_p()
    _abi.check(L.rl_obj_load(str(path).encode(), C.byref(h)))
    nv, ni, ns = C.c_int32(), C.c_int32(), C.c_int32()
    _abi.check(L.rl_obj_mesh_counts(h, C.byref(nv), C.byref(ni), C.byref(ns)))
    out = {"pos": np.zeros((nv.value, 3), np.float32), "nrm": np.zeros((nv.value, 3), np.float32),
           "uv1": np.zeros((nv.value, 2), np.float32), "idx": np.zeros(ni.value, np.int32)}
    p = lambda a: C.c_void_p(a.ctypes.data)
    _abi.check(L.rl_obj_mesh_arrays(h, p(out["pos"]), p(out["nrm"]), p(out["uv1"]), p(out["idx"])))
    L.rl_obj_mesh_destroy(h)
    out["submeshes"] = ns.value
    return out


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


# Files whose faces the reference reads outside its arrays (undefined): the
# uv-only "f a/b" form is parsed as "a/b/c", leaving later corners at index -1.
REF_UNDEFINED = {"object_uv.obj"}


@pytest.mark.parametrize("name", sorted(obj_texts()))
def test_obj_matches_golden(name, tmp_path):
    text = obj_texts()[name]
    path = tmp_path / f"{name}.obj"
    path.write_bytes(text.encode())
    got = _load(path)
    # without "vt" lines the reference leaves uv uninitialised; here it is 0
    has_uv = any(l.startswith("vt") for l in text.splitlines())
    for k in ("pos", "nrm", "uv1") if has_uv else ("pos", "nrm"):
        assert np.array_equal(_bits(got[k]), _bits(GOLD[f"{name}_{k}"])), k
    if not has_uv:
        assert not got["uv1"].any()
    assert np.array_equal(got["idx"], GOLD[f"{name}_idx"])
    assert not GOLD[f"{name}_uv0"].any()  # the diffuse layer stays 0


def test_obj_submeshes_and_mesh_api(tmp_path):
    path = tmp_path / "objects.obj"
    path.write_bytes(obj_texts()["objects"].encode())
    assert _load(path)["submeshes"] == 2
    m = Mesh.create_from_file(str(path))
    assert m.vertex_count() == GOLD["objects_pos"].shape[0]
    assert np.array_equal(np.asarray(m.indices).reshape(-1), GOLD["objects_idx"])
    assert np.array_equal(_bits(m.uv1), _bits(GOLD["objects_uv1"]))
    assert Mesh.create_from_file(str(tmp_path / "missing.obj")) is None


def test_obj_undefined_inputs_are_errors(tmp_path):
    """Face indices the reference would read out of bounds are refused."""
    bad = {"zero": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 0 1 2\n",
           "past_end": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 9\n",
           "normals_only_form": "v 0 0 0\nv 1 0 0\nv 0 1 0\nvn 0 0 1\nf 1//1 2//1 3//1\n"}
    for name, text in bad.items():
        path = tmp_path / f"{name}.obj"
        path.write_bytes(text.encode())
        h = C.c_void_p()
        rc = _abi.lib().rl_obj_load(str(path).encode(), C.byref(h))
        assert rc == _abi.RL_INVALID_CALL and not h.value, name
        assert "out of range" in _abi.last_error()


@pytest.mark.skipif(not (os.path.exists(ob.REF_LIB) and REF_DATA and os.path.isdir(REF_DATA)),
                    reason="reference build or its sample meshes absent")
def test_obj_matches_reference_sample_meshes():
    L = ob.ref_lib()
    files = sorted(glob.glob(os.path.join(REF_DATA, "*.obj")))
    assert files
    for path in files:
        if os.path.basename(path) in REF_UNDEFINED:
            with pytest.raises(_abi.RelightCudaError, match="out of range"):
                _load(path)
            continue
        ni = C.c_int()
        nv = L.ref_load_obj(path.encode(), C.byref(ni))
        want = {"pos": np.zeros((nv, 3), np.float32), "nrm": np.zeros((nv, 3), np.float32),
                "uv1": np.zeros((nv, 2), np.float32), "idx": np.zeros(ni.value, np.int32)}
        L.ref_obj_arrays(ob.ptr(want["pos"]), ob.ptr(want["nrm"]), None, ob.ptr(want["uv1"]), ob.ptr(want["idx"]))
        got = _load(path)
        for k in ("pos", "nrm", "uv1"):
            assert np.array_equal(_bits(got[k]), _bits(want[k])), (path, k)
        assert np.array_equal(got["idx"], want["idx"]), path


def test_cpp_mesh_create_from_file(tmp_path):
    """A C++ program on the drop-in API loads the same mesh."""
    import subprocess
    from relight_b200 import build
    exe = build.build_cpp_example(str(tmp_path), "load_obj")
    obj = tmp_path / "objects.obj"
    obj.write_bytes(obj_texts()["objects"].encode())
    out = tmp_path / "mesh.bin"
    subprocess.run([exe, str(obj), str(out)], check=True, timeout=60)
    raw = out.read_bytes()
    nv, ni = np.frombuffer(raw[:8], np.int32)
    v = np.frombuffer(raw[8:8 + 32 * nv], np.float32).reshape(nv, 8)
    idx = np.frombuffer(raw[8 + 32 * nv:], np.int32)
    assert np.array_equal(_bits(v[:, 0:3]), _bits(GOLD["objects_pos"]))
    assert np.array_equal(_bits(v[:, 3:6]), _bits(GOLD["objects_nrm"]))
    assert np.array_equal(_bits(v[:, 6:8]), _bits(GOLD["objects_uv1"]))
    assert np.array_equal(idx, GOLD["objects_idx"]) and ni == idx.size
