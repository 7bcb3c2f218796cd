"""ctypes bindings of the oracle (oracle/liboracle.so, the C restatement) and
of the reference baker compiled from its own sources
(oracle/_ref/librelight_ref.so).  Test infrastructure: the checkers of the
CUDA library, and the CPU baseline that bench.py times beside it — never the
thing the GPU arm measures.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from relight_b200 import _abi
from relight_b200.api import FlatScene, Scene

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(ORACLE_DIR)
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle.so")
REF_LIB = os.environ.get("RELIGHT_REF_LIB") or os.path.join(ORACLE_DIR, "_ref", "librelight_ref.so")
REF_FAST_LIB = os.path.join(ORACLE_DIR, "_ref", "librelight_ref_fast.so")
# the reference over the GPU Embree backend (embree2_gpu.cpp): same sources,
# its Embree calls answered by relight_b200/librelight_b200.so
REF_GPU_LIB = os.path.join(ORACLE_DIR, "_ref", "librelight_ref_gpu.so")

_P = C.c_void_p


def build_oracle():
    if not os.path.exists(ORACLE_LIB):
        subprocess.run(["make", "-C", ORACLE_DIR, "liboracle.so"], check=True, capture_output=True)


def reference_available():
    return os.path.exists(REF_LIB)


def reference_root():
    """The reference checkout the oracle/_ref build was compiled from, as
    recorded by oracle/Makefile, or None where it is not present."""
    p = os.path.join(ORACLE_DIR, "_ref", "reference_root.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        root = f.read().strip()
    return root if os.path.isdir(root) else None


class Lumels(C.Structure):
    """rl_lumels (oracle/rl_oracle.h)."""
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("flags", _P), ("face", _P), ("position", _P),
                ("normal", _P), ("color", _P), ("photons", _P), ("gathered", _P), ("mesh", _P)]


# ------------------------------------------------------------ post-process

RAW_HDR, TGA_DOUBLE_LDR, TGA_RGBM = 0, 1, 2   # relight::StorageFormat (Relight.h:89-93)


def expand(lm: LumelMap):
    """Lightmap::expand in place (oro_expand)."""
    s = lm.struct()
    oracle_lib().oro_expand(C.byref(s))


def blur(lm: LumelMap):
    """Lightmap::blur in place (oro_blur)."""
    s = lm.struct()
    oracle_lib().oro_blur(C.byref(s))


def to_double_ldr(lm: LumelMap) -> np.ndarray:
    out = np.zeros(lm.width * lm.height * 3, np.uint8)
    s = lm.struct()
    oracle_lib().oro_to_double_ldr(C.byref(s), ptr(out))
    return out


def to_rgbm(lm: LumelMap) -> np.ndarray:
    """The RGBM buffer with the bytes the reference never writes left 0."""
    out = np.zeros(lm.width * lm.height * 4, np.uint8)
    s = lm.struct()
    oracle_lib().oro_to_rgbm(C.byref(s), ptr(out))
    return out


def rgbm_written_mask(width: int, height: int) -> np.ndarray:
    """Bytes of the RGBM buffer that Lightmap::toRgbmLdr writes: 3w + 1 of
    every 4w-byte row (Lightmap.cpp:288-308)."""
    m = np.zeros((height, width * 4), bool)
    m[:, :3 * width + 1] = True
    return m.reshape(-1)


def save_bytes(lm: LumelMap, fmt: int) -> bytes:
    """The file Lightmap::save (Lightmap.cpp:223-283) writes, as bytes."""
    w, h = lm.width, lm.height
    if fmt == RAW_HDR:
        return np.array([w, h], np.int32).tobytes() + np.ascontiguousarray(lm.color, np.float32).tobytes()
    ch = 3 if fmt == TGA_DOUBLE_LDR else 4
    px = (to_double_ldr(lm) if fmt == TGA_DOUBLE_LDR else to_rgbm(lm)).reshape(-1, ch)
    head = bytes([0, 0, 2, 0, 0, 0, 0, 0, 0, 0, 0, 0]) + bytes([w % 256, w // 256, h % 256, h // 256, ch * 8, 0])
    order = [2, 1, 0] + ([3] if ch == 4 else [])
    return head + np.ascontiguousarray(px[:, order]).tobytes()


def tga_written_mask(width: int, height: int, fmt: int) -> np.ndarray:
    """Bytes of a saved file that the reference determines (RGBM leaves
    some pixel bytes uninitialised)."""
    if fmt != TGA_RGBM:
        n = 8 + width * height * 12 if fmt == RAW_HDR else 18 + width * height * 3
        return np.ones(n, bool)
    px = rgbm_written_mask(width, height).reshape(-1, 4)[:, [2, 1, 0, 3]].reshape(-1)
    return np.concatenate([np.ones(18, bool), px])


class Iterator(C.Structure):
    """rl_iterator (oracle/rl_oracle.h)."""
    _fields_ = [("kind", C.c_int32), ("first", C.c_int32), ("step", C.c_int32), ("mesh", C.c_int32)]


def iterator(first=0, step=1, mesh=None):
    """LumelBakeIterator(first, step) if mesh is None, else FaceBakeIterator."""
    return C.byref(Iterator(0 if mesh is None else 1, first, step, -1 if mesh is None else mesh))


class LumelMap:
    """Numpy-backed lumel arrays (Lightmap.h:35-55) for the oracle."""

    FIELDS = ("flags", "face", "position", "normal", "color", "photons", "gathered", "mesh")

    def __init__(self, width, height):
        n = width * height
        self.width, self.height = width, height
        self.flags = np.zeros(n, np.int32)
        self.face = np.full(n, 0xFFFF, np.int32)
        self.position = np.zeros((n, 3), np.float32)
        self.normal = np.zeros((n, 3), np.float32)
        self.color = np.zeros((n, 3), np.float32)
        self.photons = np.zeros(n, np.int32)
        self.gathered = np.zeros((n, 3), np.float32)
        self.mesh = np.full(n, -1, np.int32)

    def struct(self):
        s = Lumels()
        s.width, s.height = self.width, self.height
        for f in self.FIELDS:
            setattr(s, f, getattr(self, f).ctypes.data)
        return s

    def copy(self):
        m = LumelMap(self.width, self.height)
        for f in self.FIELDS:
            setattr(m, f, getattr(self, f).copy())
        return m

    def as_dict(self):
        return {f: getattr(self, f) for f in self.FIELDS}


def _load_oracle():
    build_oracle()
    lib = C.CDLL(ORACLE_LIB)
    sig = {
        "oro_create": (_P, [_P]),
        "oro_destroy": (None, [_P]),
        "oro_philox4x32_10": (None, [_P, _P, _P]),
        "oro_init_lumels": (None, [_P, C.c_int, _P]),
        "oro_trace_segments": (None, [_P, C.c_int, _P, C.c_int, _P, _P, _P, _P, _P, _P, _P]),
        "oro_bake_direct": (None, [_P, _P, C.c_int, _P, _P, _P]),
        "oro_bake_ao": (None, [_P, _P, C.c_int, C.c_float, C.c_float, C.c_float, C.c_uint64, _P]),
        "oro_emit_photons": (C.c_longlong, [_P, _P, C.c_int, _P, C.c_int, C.c_int, C.c_float, C.c_float,
                                            C.c_uint64]),
        "oro_emit_photons_range": (C.c_longlong, [_P, _P, C.c_int, _P, C.c_int, C.c_int, C.c_float, C.c_float,
                                                  C.c_uint64, C.c_longlong, C.c_longlong]),
        "oro_photonmap_gather": (None, [_P, C.c_int]),
        "oro_bake_indirect": (None, [_P, _P, _P, C.c_int, C.c_float, _P, _P, C.c_uint64, _P]),
        "oro_ff_pairwise": (C.c_longlong, [_P, C.c_int, _P, _P, C.c_float, _P, _P, _P]),
        "oro_ff_hemisphere": (C.c_longlong, [_P, C.c_int, _P, _P, C.c_int, C.c_float, C.c_uint64, _P, _P, _P, _P,
                                             _P, _P, _P]),
        "oro_jacobi_f64": (None, [C.c_int, _P, _P, _P, _P, _P, C.c_int, _P]),
        "oro_jacobi_f32": (None, [C.c_int, _P, _P, _P, _P, _P, C.c_int, _P]),
        "oro_ao_expect_f64": (None, [_P, _P, C.c_int, _P, C.c_int, C.c_float, C.c_float, C.c_uint64, _P]),
        "oro_fg_expect_f64": (None, [_P, _P, _P, C.c_int, _P, C.c_int, C.c_float, _P, _P, C.c_uint64, _P]),
        "oro_expand": (None, [_P]),
        "oro_blur": (None, [_P]),
        "oro_to_double_ldr": (None, [_P, _P]),
        "oro_to_rgbm": (None, [_P, _P]),
        "oro_f2u8": (C.c_uint8, [C.c_float]),
        "oro_last_stats": (None, [_P, _P]),
        "oro_trace_stats": (None, [_P, C.c_int, _P, C.c_int, _P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_oracle = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        _oracle = _load_oracle()
    return _oracle


def ptr(a):
    """A c_void_p to `a`'s data that keeps `a` alive as long as the pointer
    (numpy's data_as holds a reference), so temporaries survive the call."""
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def philox(ctr, key):
    c = np.asarray(ctr, np.uint32)
    k = np.asarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    oracle_lib().oro_philox4x32_10(ptr(c), ptr(k), ptr(out))
    return out


class Oracle:
    """The C restatement over one flat scene."""

    def __init__(self, flat: FlatScene):
        self.flat = flat
        self.desc, self.keep = _abi.make_scene_desc(flat)
        self.lib = oracle_lib()
        self.ctx = self.lib.oro_create(C.byref(self.desc))

    def __del__(self):
        try:
            self.lib.oro_destroy(self.ctx)
        except Exception:
            pass

    def maps(self, kind="lightmap"):
        """Fresh lumel maps with every mesh rasterised, in add order."""
        maps = self.flat.lightmaps if kind == "lightmap" else self.flat.photonmaps
        out = []
        scene_meshes = self._scene_meshes
        for m in maps:
            lm = LumelMap(m.width, m.height)
            for mesh in m.meshes:
                self.init_lumels(scene_meshes.index(mesh), lm)
            out.append(lm)
        return out

    _scene_meshes = None

    def bind_scene(self, scene: Scene):
        self._scene_meshes = scene.meshes
        return self

    def init_lumels(self, mesh, lm: LumelMap):
        s = lm.struct()
        self.lib.oro_init_lumels(C.byref(self.desc), mesh, C.byref(s))

    def trace_segments(self, seg, flags):
        seg = np.ascontiguousarray(seg, np.float32)
        n = seg.shape[0]
        out = dict(hit=np.zeros(n, np.int32), point=np.zeros((n, 3), np.float32),
                   normal=np.zeros((n, 3), np.float32), rgba=np.zeros((n, 4), np.float32),
                   uv=np.zeros((n, 2), np.float32), mesh=np.zeros(n, np.int32), face=np.zeros(n, np.int32))
        self.lib.oro_trace_segments(self.ctx, n, ptr(seg), flags, ptr(out["hit"]), ptr(out["point"]),
                                    ptr(out["normal"]), ptr(out["rgba"]), ptr(out["uv"]), ptr(out["mesh"]),
                                    ptr(out["face"]))
        return out

    def bake_direct(self, lm: LumelMap, first=0, step=1, mesh=None):
        f = self.flat
        s = lm.struct()
        self.lib.oro_bake_direct(self.ctx, ptr(f.lights), len(f.lights), ptr(f.light_vertices), C.byref(s),
                                 iterator(first, step, mesh))

    def bake_ao(self, lm: LumelMap, samples, fraction, maxd, exponent, seed, first=0, step=1, mesh=None):
        s = lm.struct()
        self.lib.oro_bake_ao(self.ctx, C.byref(s), samples, fraction, maxd, exponent, seed,
                             iterator(first, step, mesh))

    def emit_photons(self, pms, passes, depth, threshold, maxd, seed):
        arr = (Lumels * max(len(pms), 1))(*[p.struct() for p in pms])
        f = self.flat
        return self.lib.oro_emit_photons(self.ctx, ptr(f.lights), len(f.lights), arr, passes, depth, threshold, maxd,
                                         seed)

    def emit_photons_range(self, pms, passes, depth, threshold, maxd, seed, first, count):
        arr = (Lumels * max(len(pms), 1))(*[p.struct() for p in pms])
        f = self.flat
        return self.lib.oro_emit_photons_range(self.ctx, ptr(f.lights), len(f.lights), arr, passes, depth, threshold,
                                               maxd, seed, first, count)

    def gather(self, pm: LumelMap, radius):
        s = pm.struct()
        self.lib.oro_photonmap_gather(C.byref(s), radius)

    def bake_indirect(self, lm: LumelMap, pms, samples, maxd, sky, ambient, seed, first=0, step=1, mesh=None):
        arr = (Lumels * max(len(pms), 1))(*[p.struct() for p in pms])
        s = lm.struct()
        sky = np.asarray(sky, np.float32); amb = np.asarray(ambient, np.float32)
        self.lib.oro_bake_indirect(self.ctx, C.byref(s), arr, samples, maxd, ptr(sky), ptr(amb), seed,
                                   iterator(first, step, mesh))

    def ff_pairwise(self, pos, nrm, threshold):
        pos = np.ascontiguousarray(pos, np.float32); nrm = np.ascontiguousarray(nrm, np.float32)
        n = pos.shape[0]
        nnz = self.lib.oro_ff_pairwise(self.ctx, n, ptr(pos), ptr(nrm), threshold, None, None, None)
        row = np.zeros(n + 1, np.int64); cols = np.zeros(max(nnz, 1), np.int32); vals = np.zeros(max(nnz, 1), np.float32)
        self.lib.oro_ff_pairwise(self.ctx, n, ptr(pos), ptr(nrm), threshold, ptr(row), ptr(cols), ptr(vals))
        return row, cols[:nnz], vals[:nnz]

    def ff_hemisphere(self, pos, nrm, rays, maxd, seed, mesh_map, map_dims, map_base, patch_of_texel):
        pos = np.ascontiguousarray(pos, np.float32); nrm = np.ascontiguousarray(nrm, np.float32)
        mesh_map = np.ascontiguousarray(mesh_map, np.int32); map_dims = np.ascontiguousarray(map_dims, np.int32)
        map_base = np.ascontiguousarray(map_base, np.int64); pot = np.ascontiguousarray(patch_of_texel, np.int32)
        n = pos.shape[0]
        nnz = self.lib.oro_ff_hemisphere(self.ctx, n, ptr(pos), ptr(nrm), rays, maxd, seed, ptr(mesh_map),
                                         ptr(map_dims), ptr(map_base), ptr(pot), None, None, None)
        row = np.zeros(n + 1, np.int64); cols = np.zeros(max(nnz, 1), np.int32); vals = np.zeros(max(nnz, 1), np.float32)
        self.lib.oro_ff_hemisphere(self.ctx, n, ptr(pos), ptr(nrm), rays, maxd, seed, ptr(mesh_map), ptr(map_dims),
                                   ptr(map_base), ptr(pot), ptr(row), ptr(cols), ptr(vals))
        return row, cols[:nnz], vals[:nnz]

    def ao_expect(self, lm, texels, samples, fraction, maxd, seed):
        texels = np.ascontiguousarray(texels, np.int32)
        out = np.zeros(len(texels), np.float64)
        s = lm.struct()
        self.lib.oro_ao_expect_f64(self.ctx, C.byref(s), len(texels), ptr(texels), samples, fraction, maxd, seed,
                                   ptr(out))
        return out

    def fg_expect(self, lm, pms, texels, samples, maxd, sky, ambient, seed):
        texels = np.ascontiguousarray(texels, np.int32)
        out = np.zeros((len(texels), 3), np.float64)
        arr = (Lumels * max(len(pms), 1))(*[p.struct() for p in pms])
        s = lm.struct()
        sky = np.asarray(sky, np.float32); amb = np.asarray(ambient, np.float32)
        self.lib.oro_fg_expect_f64(self.ctx, C.byref(s), arr, len(texels), ptr(texels), samples, maxd, ptr(sky),
                                   ptr(amb), seed, ptr(out))
        return out

    def last_stats(self):
        out = np.zeros(3, np.uint64)
        self.lib.oro_last_stats(self.ctx, ptr(out))
        return out

    def trace_stats(self, seg, any_hit=False):
        seg = np.ascontiguousarray(seg, np.float32)
        out = np.zeros(3, np.uint64)
        self.lib.oro_trace_stats(self.ctx, seg.shape[0], ptr(seg), int(any_hit), ptr(out))
        return out


def jacobi_f64(row, cols, vals, E, rho, iters):
    lib = oracle_lib()
    n = len(row) - 1
    B = np.zeros((n, 3), np.float64)
    lib.oro_jacobi_f64(n, ptr(np.ascontiguousarray(row, np.int64)), ptr(np.ascontiguousarray(cols, np.int32)),
                       ptr(np.ascontiguousarray(vals, np.float32)), ptr(np.ascontiguousarray(E, np.float32)),
                       ptr(np.ascontiguousarray(rho, np.float32)), iters, ptr(B))
    return B


def jacobi_f32(row, cols, vals, E, rho, iters):
    lib = oracle_lib()
    n = len(row) - 1
    B = np.zeros((n, 3), np.float32)
    lib.oro_jacobi_f32(n, ptr(np.ascontiguousarray(row, np.int64)), ptr(np.ascontiguousarray(cols, np.int32)),
                       ptr(np.ascontiguousarray(vals, np.float32)), ptr(np.ascontiguousarray(E, np.float32)),
                       ptr(np.ascontiguousarray(rho, np.float32)), iters, ptr(B))
    return B


# ------------------------------------------------------------- reference

def _load_ref(path):
    lib = C.CDLL(path)
    I, F = C.c_int, C.c_float
    sig = {
        "ref_create": (_P, []), "ref_destroy": (None, [_P]), "ref_set_rand": (None, [I, C.c_uint]),
        "ref_add_material": (I, [_P, F, F, F, I, I, I, _P]),
        "ref_add_mesh": (I, [_P, I, _P, _P, _P, _P, _P, I, _P]),
        "ref_add_mesh_transformed": (I, [_P, I, _P, _P, _P, _P, _P, I, _P, _P]),
        "ref_mesh_vertices": (None, [_P, I, _P, _P]),
        "ref_add_point_light": (I, [_P, _P, F, _P, F, I]),
        "ref_add_spot_light": (I, [_P, _P, _P, F, F, _P, F, I]),
        "ref_add_directional_light": (I, [_P, _P, _P, F, I]),
        "ref_add_area_light": (I, [_P, I, _P, _P, I, _P, _P, _P, F, I]),
        "ref_light_set_attenuation": (None, [_P, I, F, F, F, F]),
        "ref_light_clear_emitter": (None, [_P, I]),
        "ref_light_vertices": (I, [_P, I, _P]),
        "ref_create_map": (I, [_P, I, I, I]),
        "ref_map_add_mesh": (I, [_P, I, I]),
        "ref_scene_end": (I, [_P]),
        "ref_scene_bounds": (None, [_P, _P, _P]),
        "ref_map_lumels": (None, [_P, I, _P, _P, _P, _P, _P, _P, _P]),
        "ref_map_set_colors": (None, [_P, I, _P]),
        "ref_map_set_photons": (None, [_P, I, _P, _P]),
        "ref_map_set_flags": (None, [_P, I, _P]),
        "ref_load_obj": (I, [C.c_char_p, _P]),
        "ref_obj_arrays": (None, [_P, _P, _P, _P, _P]),
        "ref_map_expand": (None, [_P, I]),
        "ref_map_blur": (None, [_P, I]),
        "ref_map_save": (I, [_P, I, C.c_char_p, I]),
        "ref_bake_direct": (I, [_P, I, I, I, I]),
        "ref_bake_ao": (I, [_P, I, I, F, F, F, I, I, I]),
        "ref_emit_photons": (I, [_P, I, I, F, F, I]),
        "ref_photonmap_gather": (None, [_P, I, I]),
        "ref_bake_indirect": (I, [_P, I, I, F, I, _P, _P, I, I, I]),
        "ref_bake_full": (I, [_P, I, I, I, F, F, F, I, F, I, _P, _P]),
        "ref_bake_sampled": (I, [_P, I, I, I, I, I, F, F, F, I, F, I, _P, _P]),
        "ref_radiosity_build": (I, [_P, F, I, _P]),
        "ref_radiosity_get": (None, [_P, _P, _P, _P, _P, _P]),
        "ref_trace_segments": (None, [_P, I, _P, I, _P, _P, _P, _P, _P, _P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_refs = {}


def ref_lib(fast=False):
    """fast: False = the parity build, True = the timed build, "gpu" = the
    parity build over the GPU Embree backend."""
    path = REF_GPU_LIB if fast == "gpu" else REF_FAST_LIB if fast else REF_LIB
    if path not in _refs:
        _refs[path] = _load_ref(path)
    return _refs[path]


class RefScene:
    """The reference baker driven through its own API with the same inputs
    as a relight_b200 Scene: source meshes, the same light factory calls, the
    same map/mesh registration order.  `radiancemaps` lists maps to create
    as Radiancemaps instead of Lightmaps."""

    def __init__(self, scene: Scene, fast=False, radiancemaps=()):
        self.lib = ref_lib(fast)
        L = self.lib
        self.h = L.ref_create()
        self.scene = scene
        self._keep = []
        mats = {}
        self.mesh_index = {}
        for i, inst in enumerate(scene.meshes):
            src, transform, material = inst.source
            if material is not None:
                raise NotImplementedError("the reference driver adds meshes without a material override")
            vmat = np.full(src.vertex_count(), -1, np.int32)
            for v, m in enumerate(src.materials):
                if m is None:
                    continue
                if id(m) not in mats:
                    if m.texture is not None:
                        t = m.texture
                        px = np.ascontiguousarray(t.pixels)
                        self._keep.append(px)
                        mats[id(m)] = L.ref_add_material(self.h, *[float(x) for x in m.color], t.width, t.height,
                                                         t.channels, ptr(px))
                    else:
                        mats[id(m)] = L.ref_add_material(self.h, *[float(x) for x in m.color], 0, 0, 0, None)
                vmat[v] = mats[id(m)]
            arrs = [np.ascontiguousarray(a, np.float32) for a in (src.positions, src.normals, src.uv0, src.uv1)]
            idx = np.ascontiguousarray(src.indices, np.int32)
            self._keep += arrs + [idx, vmat]
            if transform is None:
                k = L.ref_add_mesh(self.h, src.vertex_count(), *[ptr(a) for a in arrs], ptr(vmat), idx.size, ptr(idx))
            else:
                mat = np.ascontiguousarray(np.asarray(transform, np.float32).reshape(16))
                self._keep.append(mat)
                k = L.ref_add_mesh_transformed(self.h, src.vertex_count(), *[ptr(a) for a in arrs], ptr(vmat),
                                               idx.size, ptr(idx), ptr(mat))
            self.mesh_index[id(inst)] = k
        f3 = lambda v: (C.c_float * 3)(*[float(x) for x in np.asarray(v).reshape(3)])
        for li, l in enumerate(scene.lights):
            name, args = l.factory
            if name == "point":
                p, radius, color, inten, sh = args
                k = L.ref_add_point_light(self.h, f3(p), float(radius), f3(color), float(inten), int(sh))
            elif name == "spot":
                p, d, cut, radius, color, inten, sh = args
                k = L.ref_add_spot_light(self.h, f3(p), f3(d), float(cut), float(radius), f3(color), float(inten),
                                         int(sh))
            elif name == "directional":
                d, color, inten, sh = args
                k = L.ref_add_directional_light(self.h, f3(d), f3(color), float(inten), int(sh))
            else:
                mesh, p, color, inten, sh = args
                pos = np.ascontiguousarray(mesh.positions, np.float32)
                nrm = np.ascontiguousarray(mesh.normals, np.float32)
                idx = np.ascontiguousarray(mesh.indices, np.int32)
                self._keep += [pos, nrm, idx]
                k = L.ref_add_area_light(self.h, mesh.vertex_count(), ptr(pos), ptr(nrm), idx.size, ptr(idx), f3(p),
                                         f3(color), float(inten), int(sh))
            a = l.attenuation
            if l.attenuation_overridden and a is not None:
                L.ref_light_set_attenuation(self.h, k, a.radius, a.constant, a.linear, a.quadratic)
            if l.emitter == 0:
                L.ref_light_clear_emitter(self.h, k)
        self.maps = {}
        flat = scene.flat
        for kind, maps in ((0, flat.lightmaps), (1, flat.photonmaps)):
            for m in maps:
                mk = 2 if m in radiancemaps else kind
                k = L.ref_create_map(self.h, mk, m.width, m.height)
                self.maps[id(m)] = k
                for mesh in m.meshes:
                    L.ref_map_add_mesh(self.h, k, self.mesh_index[id(mesh)])
        L.ref_scene_end(self.h)

    def mesh(self, inst):
        return self.mesh_index[id(inst)]

    def lumels(self, m) -> LumelMap:
        k = self.maps[id(m)]
        out = LumelMap(m.width, m.height)
        self.lib.ref_map_lumels(self.h, k, ptr(out.flags), ptr(out.face), ptr(out.position), ptr(out.normal),
                                ptr(out.color), ptr(out.photons), ptr(out.gathered))
        return out

    def post_map(self, width, height, flags, color) -> int:
        """A fresh Lightmap of the reference with the given lumel flags and
        colours (for expand / blur / save)."""
        k = self.lib.ref_create_map(self.h, 0, width, height)
        self.set_map(k, flags, color)
        return k

    def set_map(self, k, flags, color):
        flags = np.ascontiguousarray(flags, np.int32)
        color = np.ascontiguousarray(color, np.float32)
        self.lib.ref_map_set_flags(self.h, k, ptr(flags))
        self.lib.ref_map_set_colors(self.h, k, ptr(color))

    def map_colors(self, k, width, height):
        out = np.zeros((width * height, 3), np.float32)
        self.lib.ref_map_lumels(self.h, k, None, None, None, None, ptr(out), None, None)
        return out

    def mesh_vertices(self, inst):
        n = inst.vertex_count()
        pos = np.zeros((n, 3), np.float32); nrm = np.zeros((n, 3), np.float32)
        self.lib.ref_mesh_vertices(self.h, self.mesh(inst), ptr(pos), ptr(nrm))
        return pos, nrm

    def light_vertices(self, li):
        n = self.lib.ref_light_vertices(self.h, li, None)
        out = np.zeros((max(n, 1), 3), np.float32)
        self.lib.ref_light_vertices(self.h, li, ptr(out))
        return out[:n]

    def trace_segments(self, seg, flags):
        seg = np.ascontiguousarray(seg, np.float32)
        n = seg.shape[0]
        out = dict(hit=np.zeros(n, np.int32), point=np.zeros((n, 3), np.float32),
                   normal=np.zeros((n, 3), np.float32), rgba=np.zeros((n, 4), np.float32),
                   uv=np.zeros((n, 2), np.float32), mesh=np.zeros(n, np.int32))
        self.lib.ref_trace_segments(self.h, n, ptr(seg), flags, ptr(out["hit"]), ptr(out["point"]),
                                    ptr(out["normal"]), ptr(out["rgba"]), ptr(out["uv"]), ptr(out["mesh"]))
        return out

    def radiosity(self, threshold=0.1, max_ff=0):
        nnz = C.c_longlong()
        n = self.lib.ref_radiosity_build(self.h, threshold, max_ff, C.byref(nnz))
        row = np.zeros(n + 1, np.int64); cols = np.zeros(max(nnz.value, 1), np.int32)
        vals = np.zeros(max(nnz.value, 1), np.float32)
        pos = np.zeros((n, 3), np.float32); nrm = np.zeros((n, 3), np.float32)
        self.lib.ref_radiosity_get(self.h, ptr(row), ptr(cols), ptr(vals), ptr(pos), ptr(nrm))
        return row, cols[:nnz.value], vals[:nnz.value], pos, nrm
