"""ctypes binding of the C ABI (include/relight_b200.h) in librelight_b200.so.

The library is built in-tree by relight_b200/build.py.  There is no CPU
fallback: if the shared library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librelight_b200.so")

RL_OK, RL_INVALID_CALL, RL_NOT_IMPLEMENTED, RL_OUT_OF_MEMORY, RL_CUDA_ERROR, RL_CAPACITY = range(6)
HIT_POINT, HIT_UV, HIT_COLOR, HIT_NORMAL, HIT_USE_ALPHA = 1, 2, 4, 8, 16
HIT_ALL = 15
TUNE_FG_REFILL, TUNE_FG_BLOCK, TUNE_AO_REFILL, TUNE_AO_BLOCK, TUNE_BVH_WIDTH, TUNE_SPECULATIVE = 0, 1, 2, 3, 4, 5
TUNE_KNN_CELL = 6
TUNE_AO_SPLIT = 7
TUNE_FG_POOL, TUNE_FG_CHUNK = 8, 9
SOLVE_NOALLOC_MAX_PATCHES = 65536


class SceneDesc(C.Structure):
    """rl_scene_desc."""
    _fields_ = [
        ("nverts", C.c_int32),
        ("pos", C.c_void_p), ("nrm", C.c_void_p), ("uv0", C.c_void_p), ("uv1", C.c_void_p), ("vmat", C.c_void_p),
        ("ntris", C.c_int32), ("tris", C.c_void_p),
        ("nmeshes", C.c_int32), ("mesh_first_tri", C.c_void_p), ("mesh_lightmap", C.c_void_p),
        ("mesh_photonmap", C.c_void_p),
        ("nmats", C.c_int32), ("mat_rgb", C.c_void_p), ("mat_tex", C.c_void_p),
        ("ntex", C.c_int32), ("tex_dims", C.c_void_p), ("tex_offset", C.c_void_p), ("tex_pixels", C.c_void_p),
        ("bounds_lo", C.c_float * 3), ("bounds_hi", C.c_float * 3),
    ]


class Iterator(C.Structure):
    """rl_iterator: kind 0 LumelBakeIterator(first, step), kind 1
    FaceBakeIterator(first, step) over one scene mesh."""
    _fields_ = [("kind", C.c_int32), ("first", C.c_int32), ("step", C.c_int32), ("mesh", C.c_int32)]


class BatchJob(C.Structure):
    """rl_batch_job."""
    _fields_ = [("kind", C.c_int32), ("scene", C.c_void_p), ("lightmap", C.c_void_p), ("photonmaps", C.c_void_p),
                ("nmaps", C.c_int32), ("lights", C.c_void_p), ("nlights", C.c_int32),
                ("light_vertices", C.c_void_p), ("nlight_vertices", C.c_int32), ("samples", C.c_int32),
                ("occluded_fraction", C.c_float), ("max_distance", C.c_float), ("exponent", C.c_float),
                ("sky", C.c_float * 3), ("ambient", C.c_float * 3), ("seed", C.c_uint64),
                ("iterator", Iterator), ("begin", C.c_int64), ("end", C.c_int64)]


def _ptr(a):
    """A c_void_p to `a`'s data that holds a reference to `a` (numpy's
    data_as), so the array outlives the pointer."""
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def make_scene_desc(flat):
    """Build an rl_scene_desc over a FlatScene's arrays.  Returns (desc, keep)
    where `keep` holds the contiguous arrays the pointers refer to."""
    keep = {}

    def c(name, dtype):
        a = np.ascontiguousarray(getattr(flat, name), dtype=dtype)
        keep[name] = a
        return a

    pos = c("pos", np.float32); nrm = c("nrm", np.float32); uv0 = c("uv0", np.float32); uv1 = c("uv1", np.float32)
    vmat = c("vmat", np.int32); tris = c("tris", np.int32); first = c("mesh_first_tri", np.int32)
    lmap = c("mesh_lightmap", np.int32); pmap = c("mesh_photonmap", np.int32)
    mat_rgb = c("mat_rgb", np.float32); mat_tex = c("mat_tex", np.int32)
    tex_dims = c("tex_dims", np.int32); tex_off = c("tex_offset", np.int64); tex_px = c("tex_pixels", np.uint8)
    d = SceneDesc()
    d.nverts = pos.shape[0]
    d.pos, d.nrm, d.uv0, d.uv1, d.vmat = _ptr(pos), _ptr(nrm), _ptr(uv0), _ptr(uv1), _ptr(vmat)
    d.ntris = tris.shape[0]
    d.tris = _ptr(tris)
    d.nmeshes = first.shape[0] - 1
    d.mesh_first_tri, d.mesh_lightmap, d.mesh_photonmap = _ptr(first), _ptr(lmap), _ptr(pmap)
    d.nmats = mat_rgb.shape[0]
    d.mat_rgb, d.mat_tex = _ptr(mat_rgb), _ptr(mat_tex)
    d.ntex = tex_dims.shape[0]
    d.tex_dims, d.tex_offset, d.tex_pixels = _ptr(tex_dims), _ptr(tex_off), _ptr(tex_px)
    for k in range(3):
        d.bounds_lo[k] = float(flat.bounds_lo[k])
        d.bounds_hi[k] = float(flat.bounds_hi[k])
    return d, keep


_P = C.c_void_p
_I = C.c_int
_I64 = C.c_int64
_U64 = C.c_uint64
_F = C.c_float

# name -> (restype, argtypes): every symbol include/relight_b200.h declares
SIGNATURES = {
    "rl_last_error": (_I, [C.c_char_p, C.c_size_t]),
    "rl_version": (C.c_char_p, []),
    "rl_scene_create": (_I, [_P, _I, _P, _P]),
    "rl_scene_destroy": (_I, [_P]),
    "rl_scene_bvh_stats": (_I, [_P, _P, _P, _P, _P]),
    "rl_scene_status": (_I, [_P, _I, _P, _P]),
    "rl_intersect_rays": (_I, [_P, C.c_int64, _P, _I, _P, _P, _P]),
    "rl_intersect_rays_host": (_I, [_P, C.c_int64, _P, _I, _P, _P]),
    "rl_trace_segments": (_I, [_P, _I64, _P, _I, _P, _P, _P, _P, _P, _P, _P, _P]),
    "rl_map_create": (_I, [_I, _I, _I, _P]),
    "rl_map_destroy": (_I, [_P]),
    "rl_map_add_mesh": (_I, [_P, _P, _I, _P]),
    "rl_map_download": (_I, [_P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "rl_map_upload": (_I, [_P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "rl_map_clear": (_I, [_P, _I, _I, _P]),
    "rl_map_device_arrays": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "rl_map_valid_count": (_I, [_P, _P]),
    "rl_bake_direct": (_I, [_P, _P, _P, _I, _P, _I, _P, _P]),
    "rl_bake_ao": (_I, [_P, _P, _I, _F, _F, _F, _U64, _P, _P]),
    "rl_emit_photons": (_I, [_P, _P, _I, _P, _I, _I, _I, _F, _F, _U64, _P, _P]),
    "rl_emit_photons_range": (_I, [_P, _P, _I, _P, _I, _I, _I, _F, _F, _U64, _I64, _I64, _P, _P]),
    "rl_photon_count": (_I, [_P, _I, _I, _P]),
    "rl_photonmap_gather": (_I, [_P, _I, _P]),
    "rl_bake_indirect": (_I, [_P, _P, _P, _I, _I, _F, _P, _P, _U64, _P, _P]),
    "rl_ff_pairwise": (_I, [_P, _I, _P, _P, _F, _P, _P, _P, _I64, _P, _P]),
    "rl_ff_hemisphere": (_I, [_P, _I, _P, _P, _I, _F, _U64, _P, _I, _P, _P, _P, _I64, _P, _P, _P, _I64, _P, _P]),
    "rl_ff_hemisphere_device": (_I, [_P, _I, _P, _P, _I, _F, _U64, _P, _I, _P, _P, _P, _I64, _P, _P, _P, _I64, _P, _P]),
    "rl_radiosity_solve": (_I, [_I, _P, _P, _P, _P, _P, _I, _P, _P]),
    "rl_radiosity_solve_noalloc": (_I, [_I, _P, _P, _P, _P, _P, _I, _P, _P]),
    "rl_radiosity_step": (_I, [_I, _I, _P, _P, _P, _P, _P, _P, _P, _P]),
    "rl_obj_load": (_I, [C.c_char_p, _P]),
    "rl_obj_mesh_counts": (_I, [_P, _P, _P, _P]),
    "rl_obj_mesh_arrays": (_I, [_P, _P, _P, _P, _P]),
    "rl_obj_mesh_destroy": (_I, [_P]),
    "rl_dn_conv3x3": (_I, [_P, _I, _P, _I, _I, _I, _I, _P, _I, _P, _I, _F, _P, _I, _I, _I, _P, _P, _I, _I, _I,
                           _P, _P, _P]),
    "rl_dn_conv3x3_wgrad": (_I, [_P, _I, _I, _P, _I, _I, _I, _I, _I, _P, _I, _I, _P, _P]),
    "rl_denoiser_create": (_I, [_U64, _P]),
    "rl_denoiser_destroy": (_I, [_P]),
    "rl_denoiser_param_count": (_I, [_P, _P]),
    "rl_denoiser_get_params": (_I, [_P, _P]),
    "rl_denoiser_set_params": (_I, [_P, _P]),
    "rl_denoiser_get_grads": (_I, [_P, _P]),
    "rl_denoiser_features": (_I, [_P, _P, _P, _P]),
    "rl_denoiser_targets": (_I, [_P, _P, _P]),
    "rl_denoiser_train_step": (_I, [_P, _P, _P, _I, _I, _F, _P, _P]),
    "rl_denoiser_apply": (_I, [_P, _P, _P, _P, _P]),
    "rl_denoiser_forward": (_I, [_P, _P, _I, _I, _I, _P, _P]),
    "rl_denoiser_status": (_I, [_P, _P]),
    "rl_denoiser_reserve": (_I, [_P, _I, _I, _I, _I]),
    "rl_photons_create": (_I, [_I64, _P]),
    "rl_photons_destroy": (_I, [_P]),
    "rl_photons_count": (_I, [_P, _P]),
    "rl_photons_download": (_I, [_P, _P, _P, _P]),
    "rl_photons_upload": (_I, [_P, _I64, _P, _P, _P]),
    "rl_emit_photons_records": (_I, [_P, _P, _I, _P, _I, _I, _I, _F, _F, _U64, _P, _P, _P]),
    "rl_photonmap_gather_knn": (_I, [_P, _I, _P, _I, _F, _P]),
    "rl_batch_create": (_I, [_P, _I, _P]),
    "rl_batch_update": (_I, [_P, _P, _I, _P]),
    "rl_map_bytes": (_I, [_I, _I, _P]),
    "rl_map_expand": (_I, [_P, _P]),
    "rl_map_blur": (_I, [_P, _P]),
    "rl_map_encode": (_I, [_P, _I, _P, _P]),
    "rl_map_save": (_I, [_P, C.c_char_p, _I, _P]),
    "rl_pool_trim": (_I, [_I64]),
    "rl_pool_bytes": (_I, [_P, _P]),
    "rl_map_download_async": (_I, [_P, _P, _P]),
    "rl_map_create_async": (_I, [_I, _I, _I, _P, _P]),
    "rl_map_destroy_async": (_I, [_P, _P]),
    "rl_batch_launch": (_I, [_P, _P]),
    "rl_batch_capture": (_I, [_P, _P]),
    "rl_batch_replay": (_I, [_P, _P]),
    "rl_batch_work_items": (_I, [_P, _P]),
    "rl_batch_destroy": (_I, [_P]),
    "rl_measure_read_bandwidth": (_I, [C.c_size_t, _I, _P]),
    "rl_measure_l1_read_bandwidth": (_I, [C.c_size_t, _I, _P]),
    "rl_tune_set": (_I, [_I, _I]),
    "rl_tune_get": (_I, [_I, _P]),
}


class RelightCudaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"relight_b200 error {code}: {msg}")
        self.code = code


def load(path: str = LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m relight_b200.build` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = load()
    return _lib


def last_error() -> str:
    """rl_last_error: the message of this thread's last failed call."""
    buf = C.create_string_buffer(1024)
    lib().rl_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc):
    if rc != RL_OK:
        raise RelightCudaError(rc, last_error())
    return rc
