"""The baking front end: relight::Relight over the CUDA C ABI.

`Relight` mirrors Relight.h:155-189.  A scene's BVH and every lightmap /
photonmap live on the device once the first bake call sees the scene; the
bake calls enqueue kernels on `stream` (a cudaStream_t as an int, None = the
legacy default stream) and return at once, as the C ABI does.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _abi
from ._abi import check, lib
from .api import (AmbientOcclusionSettings, IndirectLightSettings, Lightmap, Mesh, Photonmap, RelightStatus, Scene)


@dataclass
class LumelBakeIterator:
    """bake::LumelBakeIterator (baker/Baker.h:138-148): lumels first, first+step, ...
    of the mesh's whole lightmap (whichever mesh rasterised them)."""
    first: int = 0
    step: int = 1


@dataclass
class FaceBakeIterator:
    """bake::FaceBakeIterator (baker/Baker.h:151-155): the lumels rasterised
    from the baked mesh's faces first, first+step, ..."""
    first: int = 0
    step: int = 1


@dataclass
class JobData:
    """Worker.h:35-42: what a worker is handed for one mesh."""
    worker: Optional["Worker"] = None
    job: Optional["Job"] = None
    relight: Optional["Relight"] = None
    scene: Optional[Scene] = None
    mesh: Optional[Mesh] = None
    iterator: object = None


class Job:
    """Worker.h:45-49: user code run for every (mesh, worker) pair."""

    def execute(self, data: JobData):
        raise NotImplementedError


class Worker:
    """Worker.h:72-84 (a Progress): runs a pushed job at once on the calling
    thread; subclasses may run jobs elsewhere."""

    def push(self, job: Job, data: JobData):
        data.worker = self
        job.execute(data)

    def wait(self):
        pass

    def notify(self, instance, step, step_count):
        pass


def _volume(mesh: Mesh):
    """Bounds::volume of the mesh's bounds, in float32 and the reference's
    operation order."""
    lo, hi = mesh.bounds()
    d = (np.asarray(hi, np.float32) - np.asarray(lo, np.float32)).astype(np.float32)
    return np.float32(np.float32(d[0] * d[1]) * d[2])


class FullBakeJob(Job):
    """Worker.h:52-69, Worker.cpp:43-83: for every scene mesh, largest bounding
    volume first (ties keep scene order), push `job` to every worker j with
    FaceBakeIterator(j, n) (LumelBakeIterator(j, n) when the mesh has fewer
    faces than workers), then wait for every worker."""

    def __init__(self, job: Job, workers):
        self.job, self.workers = job, list(workers)

    def execute(self, data: JobData):
        n = len(self.workers)
        meshes = sorted(data.scene.meshes, key=lambda m: -float(_volume(m)))
        for mesh in meshes:
            for j, w in enumerate(self.workers):
                it = FaceBakeIterator(j, n) if mesh.face_count() >= n else LumelBakeIterator(j, n)
                w.push(self.job, JobData(job=self.job, relight=data.relight, scene=data.scene, mesh=mesh,
                                         iterator=it))
            for w in self.workers:
                w.wait()


class DeviceScene:
    """An rl_scene: the flat scene uploaded and its BVH built (Scene::end)."""

    def __init__(self, flat, stream=None, builder: int = 0):
        self.flat = flat
        self.desc, self.keep = _abi.make_scene_desc(flat)
        self.handle = C.c_void_p()
        self.stream = stream
        check(lib().rl_scene_create(C.byref(self.desc), builder, stream, C.byref(self.handle)))

    def bvh_stats(self):
        nodes, leaves, depth, sah = C.c_int64(), C.c_int64(), C.c_int32(), C.c_double()
        check(lib().rl_scene_bvh_stats(self.handle, C.byref(nodes), C.byref(leaves), C.byref(depth), C.byref(sah)))
        return {"nodes": nodes.value, "leaves": leaves.value, "depth": depth.value, "sah": sah.value}

    def status(self, clear=False, stream=None):
        """The traversal status word after the queued work: bit 0 = a
        traversal stack overflowed (rl_scene_status)."""
        flags = C.c_int32()
        check(lib().rl_scene_status(self.handle, int(clear), C.byref(flags), stream or self.stream))
        return flags.value

    def close(self):
        if self.handle:
            check(lib().rl_scene_destroy(self.handle))
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceMap:
    """An rl_map: lumel arrays of one lightmap / photonmap on the device."""

    def __init__(self, kind: int, width: int, height: int, stream=None, stream_ordered: bool = False):
        """stream_ordered: one block from the stream-ordered allocator
        (rl_map_create_async on `stream`), released by close() in stream
        order as well; neither waits for the device."""
        self.kind, self.width, self.height = kind, width, height
        self.handle = C.c_void_p()
        self.stream_ordered = stream_ordered
        self.stream = stream
        if stream_ordered:
            check(lib().rl_map_create_async(kind, width, height, stream, C.byref(self.handle)))
        else:
            check(lib().rl_map_create(kind, width, height, C.byref(self.handle)))

    @staticmethod
    def nbytes(width: int, height: int) -> int:
        """Device bytes of a stream-ordered width x height map (rl_map_bytes)."""
        b = C.c_int64()
        check(lib().rl_map_bytes(width, height, C.byref(b)))
        return b.value

    def add_mesh(self, scene: DeviceScene, mesh_index: int, stream=None):
        check(lib().rl_map_add_mesh(self.handle, scene.handle, mesh_index, stream))

    def download(self, stream=None, fields=("flags", "face", "position", "normal", "color", "photons", "gathered")):
        n = self.width * self.height
        shapes = {"flags": (n,), "face": (n,), "photons": (n,), "position": (n, 3), "normal": (n, 3),
                  "color": (n, 3), "gathered": (n, 3)}
        out = {}
        args = []
        for f in ("flags", "face", "position", "normal", "color", "photons", "gathered"):
            if f in fields:
                dt = np.int32 if f in ("flags", "face", "photons") else np.float32
                out[f] = np.zeros(shapes[f], dt)
                args.append(C.c_void_p(out[f].ctypes.data))
            else:
                args.append(None)
        check(lib().rl_map_download(self.handle, *args, stream))
        return out

    def expand(self, stream=None):
        """Lightmap::expand on the device (rl_map_expand)."""
        check(lib().rl_map_expand(self.handle, stream))

    def blur(self, stream=None):
        """Lightmap::blur on the device (rl_map_blur)."""
        check(lib().rl_map_blur(self.handle, stream))

    def encode(self, fmt: int, stream=None) -> np.ndarray:
        """The reference's pixel buffer for a StorageFormat (0 RawHdr floats
        as bytes, 1 DoubleLdr, 2 RGBM), encoded on the device (rl_map_encode)."""
        n = self.width * self.height
        out = np.zeros(n * (12 if fmt == 0 else 3 if fmt == 1 else 4), np.uint8)
        check(lib().rl_map_encode(self.handle, int(fmt), C.c_void_p(out.ctypes.data), stream))
        return out

    def save(self, path: str, fmt: int, stream=None):
        """Lightmap::save: the reference's file, byte for byte (rl_map_save)."""
        check(lib().rl_map_save(self.handle, str(path).encode(), int(fmt), stream))

    def download_color_async(self, out_ptr: int, stream=None):
        """Copy the colours ([w*h][3] float32) to host memory at `out_ptr` in
        stream order, without waiting (rl_map_download_async)."""
        check(lib().rl_map_download_async(self.handle, C.c_void_p(out_ptr), stream))

    def upload(self, stream=None, **arrays):
        args = []
        for f in ("flags", "face", "position", "normal", "color", "photons", "gathered"):
            a = arrays.get(f)
            if a is not None:
                dt = np.int32 if f in ("flags", "face", "photons") else np.float32
                a = np.ascontiguousarray(a, dt)
                arrays[f] = a
                args.append(C.c_void_p(a.ctypes.data))
            else:
                args.append(None)
        check(lib().rl_map_upload(self.handle, *args, stream))

    def clear(self, colors=True, photons=False, stream=None):
        check(lib().rl_map_clear(self.handle, int(colors), int(photons), stream))

    def device_arrays(self):
        ptrs = [C.c_void_p() for _ in range(6)]
        check(lib().rl_map_device_arrays(self.handle, *[C.byref(p) for p in ptrs]))
        return dict(zip(("flags", "position", "normal", "color", "photons", "gathered"), [p.value for p in ptrs]))

    def valid_count(self):
        c = C.c_int64()
        check(lib().rl_map_valid_count(self.handle, C.byref(c)))
        return c.value

    def close(self, stream=None):
        if self.handle:
            if self.stream_ordered:
                check(lib().rl_map_destroy_async(self.handle, stream if stream is not None else self.stream))
            else:
                check(lib().rl_map_destroy(self.handle))
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PhotonRecords:
    """rl_photons: world-space photon deposits and their grid, for
    the k-nearest-neighbour estimate."""

    def __init__(self, capacity: int):
        self.capacity = capacity
        self.handle = C.c_void_p()
        check(lib().rl_photons_create(capacity, C.byref(self.handle)))

    def count(self) -> int:
        n = C.c_int64()
        check(lib().rl_photons_count(self.handle, C.byref(n)))
        return n.value

    def download(self):
        """(xyzrgb [n][6], photon [n], depth [n], slot [n]) in no particular order."""
        n = min(self.count(), self.capacity)
        xyz = np.zeros((n, 6), np.float32)
        ph = np.zeros(n, np.uint32)
        ds = np.zeros((n, 2), np.int32)
        check(lib().rl_photons_download(self.handle, C.c_void_p(xyz.ctypes.data), C.c_void_p(ph.ctypes.data),
                                        C.c_void_p(ds.ctypes.data)))
        return xyz, ph, ds[:, 0], ds[:, 1]

    def upload(self, xyzrgb, photon, depth, slot):
        """Replace the records (rl_photons_upload): xyzrgb [n][6], photon [n],
        depth [n], slot [n]."""
        xyz = np.ascontiguousarray(xyzrgb, np.float32).reshape(-1, 6)
        ph = np.ascontiguousarray(photon, np.uint32)
        ds = np.ascontiguousarray(np.stack([np.asarray(depth), np.asarray(slot)], 1), np.int32)
        check(lib().rl_photons_upload(self.handle, len(xyz), C.c_void_p(xyz.ctypes.data), C.c_void_p(ph.ctypes.data),
                                      C.c_void_p(ds.ctypes.data)))

    def gather_knn(self, photonmap, slot: int, k: int = 100, radius: float = 1.0, stream=None):
        """rl_photonmap_gather_knn on a DeviceMap (after its disc gather)."""
        check(lib().rl_photonmap_gather_knn(photonmap.handle, slot, self.handle, k, float(radius), stream))

    def close(self):
        if self.handle:
            check(lib().rl_photons_destroy(self.handle))
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _map_array(maps):
    arr = (C.c_void_p * max(len(maps), 1))()
    for i, m in enumerate(maps):
        arr[i] = m.handle.value
    return arr


class Relight:
    """relight::Relight (Relight.h:155-189)."""

    def __init__(self, stream=None, seed: int = 0x5EED, builder: int = 0):
        self.stream = stream
        self._seed = seed
        self._calls = 0
        self.builder = builder  # 0: binned SAH on the host, 1: LBVH on the device

    @staticmethod
    def create(stream=None):
        return Relight(stream)

    def create_scene(self) -> Scene:
        s = Scene()
        s.begin()
        return s

    def create_lightmap(self, width, height) -> Lightmap:
        return Lightmap(width, height)

    def create_photonmap(self, width, height) -> Photonmap:
        return Photonmap(width, height)

    # ------------------------------------------------------------ helpers
    def next_seed(self):
        """Each stochastic call draws from its own Philox key."""
        self._calls += 1
        return (self._seed * 0x9E3779B97F4A7C15 + self._calls) & 0xFFFFFFFFFFFFFFFF

    def device_scene(self, scene: Scene) -> DeviceScene:
        """Upload the scene and rasterise every map's lumels (Scene::end +
        Lightmap/Photonmap::addMesh, in the reference's addMesh order)."""
        if scene.flat is None:
            raise RuntimeError("Scene::end has not been called")
        if scene._device is None:
            ds = DeviceScene(scene.flat, self.stream, self.builder)
            for maps in (scene.flat.lightmaps, scene.flat.photonmaps):
                for m in maps:
                    if m._device is None:
                        m._device = DeviceMap(m.KIND, m.width, m.height)
                        for mesh in m.meshes:
                            m._device.add_mesh(ds, scene.meshes.index(mesh), self.stream)
            scene._device = ds
        return scene._device

    @staticmethod
    def _iter(scene, mesh, iterator):
        if iterator is None:
            return None
        if isinstance(iterator, LumelBakeIterator):
            return C.byref(_abi.Iterator(0, iterator.first, iterator.step, -1))
        if isinstance(iterator, FaceBakeIterator):
            return C.byref(_abi.Iterator(1, iterator.first, iterator.step, scene.meshes.index(mesh)))
        raise TypeError("iterator must be a LumelBakeIterator or a FaceBakeIterator")

    def _check_mesh(self, scene: Scene, mesh: Mesh):
        if mesh.face_count() == 0 or mesh.lightmap is None:
            return RelightStatus.RelightInvalidCall
        return RelightStatus.RelightSuccess

    # -------------------------------------------------------------- bakes
    def bake_direct_light(self, scene: Scene, mesh: Mesh, progress=None, iterator=None) -> RelightStatus:
        """Relight::bakeDirectLight (Relight.cpp:216-227)."""
        st = self._check_mesh(scene, mesh)
        if st:
            return st
        ds = self.device_scene(scene)
        it = self._iter(scene, mesh, iterator)
        f = scene.flat
        check(lib().rl_bake_direct(ds.handle, mesh.lightmap._device.handle, C.c_void_p(f.lights.ctypes.data),
                                   len(f.lights), C.c_void_p(f.light_vertices.ctypes.data),
                                   int(sum(int(l["vertex_count"]) for l in f.lights)), it, self.stream))
        return RelightStatus.RelightSuccess

    def bake_ambient_occlusion(self, scene: Scene, mesh: Mesh, progress, settings: AmbientOcclusionSettings,
                               iterator=None, seed: Optional[int] = None) -> RelightStatus:
        """Relight::bakeAmbientOcclusion (Relight.cpp:260-271)."""
        st = self._check_mesh(scene, mesh)
        if st:
            return st
        ds = self.device_scene(scene)
        it = self._iter(scene, mesh, iterator)
        seed = self.next_seed() if seed is None else seed
        check(lib().rl_bake_ao(ds.handle, mesh.lightmap._device.handle, settings.samples, settings.occluded_fraction,
                               settings.max_distance, settings.exponent, seed, it, self.stream))
        return RelightStatus.RelightSuccess

    def emit_photons(self, scene: Scene, settings: IndirectLightSettings, seed: Optional[int] = None,
                     knn: Optional[tuple] = None, records: Optional["PhotonRecords"] = None) -> RelightStatus:
        """Relight::emitPhotons (Relight.cpp:244-257): trace, then gather every
        photonmap.  knn = (k, radius): also keep the deposits in `records` and
        replace the estimate at valid lumels by the k nearest deposits'
        mean colour (rl_photonmap_gather_knn)."""
        ds = self.device_scene(scene)
        f = scene.flat
        maps = [m._device for m in f.photonmaps]
        seed = self.next_seed() if seed is None else seed
        args = (ds.handle, _map_array(maps), len(maps), C.c_void_p(f.lights.ctypes.data), len(f.lights),
                settings.photon_pass_count, settings.photon_bounce_count, settings.photon_energy_threshold,
                settings.photon_max_distance, seed)
        if knn is not None:
            if records is None:
                raise ValueError("knn needs a PhotonRecords buffer")
            check(lib().rl_emit_photons_records(*args, records.handle, None, self.stream))
        else:
            check(lib().rl_emit_photons(*args, None, self.stream))
        for slot, m in enumerate(maps):
            check(lib().rl_photonmap_gather(m.handle, settings.final_gather_radius, self.stream))
            if knn is not None:
                records.gather_knn(m, slot, knn[0], knn[1], self.stream)
        return RelightStatus.RelightSuccess

    def bake_indirect_light(self, scene: Scene, mesh: Mesh, progress, settings: IndirectLightSettings,
                            iterator=None, seed: Optional[int] = None) -> RelightStatus:
        """Relight::bakeIndirectLight (Relight.cpp:230-241)."""
        st = self._check_mesh(scene, mesh)
        if st:
            return st
        ds = self.device_scene(scene)
        it = self._iter(scene, mesh, iterator)
        maps = [m._device for m in scene.flat.photonmaps]
        sky = (C.c_float * 3)(*[float(x) for x in settings.sky_color])
        amb = (C.c_float * 3)(*[float(x) for x in settings.ambient_color])
        seed = self.next_seed() if seed is None else seed
        check(lib().rl_bake_indirect(ds.handle, mesh.lightmap._device.handle, _map_array(maps), len(maps),
                                     settings.final_gather_samples, settings.final_gather_distance, sky, amb, seed,
                                     it, self.stream))
        return RelightStatus.RelightSuccess


    def bake(self, scene: Scene, job: Job, root: Worker, workers) -> None:
        """Relight::bake (Relight.cpp:204-213): push a FullBakeJob over
        `workers` to `root`."""
        full = FullBakeJob(job, workers)
        root.push(full, JobData(job=full, relight=self, scene=scene))

    # ------------------------------------------- one bake over several GPUs
    # The engine interface of relight_b200.parallel: torch views of the
    # device accumulators, and the shard-sized calls of each pass.

    def torch_stream(self):
        """The torch stream the collectives must run on so they order with
        this object's kernels (None: torch's current stream)."""
        import torch
        return None if self.stream is None else torch.cuda.ExternalStream(int(self.stream))

    def color_tensor(self, lightmap: Lightmap):
        from .parallel import map_tensor
        return map_tensor(lightmap._device, "color")

    def photon_accumulators(self, scene: Scene):
        """Colour sums, then photon counts, of every photonmap (zero-copy)."""
        from .parallel import map_tensor
        self.device_scene(scene)
        maps = [m._device for m in scene.flat.photonmaps]
        return [map_tensor(m, "color") for m in maps] + [map_tensor(m, "photons") for m in maps]

    def photon_total(self, scene: Scene, settings: IndirectLightSettings) -> int:
        f = scene.flat
        total = C.c_int64()
        check(lib().rl_photon_count(C.c_void_p(f.lights.ctypes.data), len(f.lights), settings.photon_pass_count,
                                    C.byref(total)))
        return total.value

    def emit_photon_range(self, scene: Scene, settings: IndirectLightSettings, seed: int, first: int, count: int):
        """Photons [first, first + count) of the emission's global sequence
        (rl_emit_photons_range), deposited into every photonmap."""
        ds = self.device_scene(scene)
        f = scene.flat
        maps = [m._device for m in f.photonmaps]
        check(lib().rl_emit_photons_range(ds.handle, _map_array(maps), len(maps), C.c_void_p(f.lights.ctypes.data),
                                          len(f.lights), settings.photon_pass_count, settings.photon_bounce_count,
                                          settings.photon_energy_threshold, settings.photon_max_distance, seed,
                                          first, count, None, self.stream))

    def gather_photons(self, scene: Scene, settings: IndirectLightSettings):
        """Photonmap::gather on every photonmap (Relight.cpp:250-254)."""
        for m in scene.flat.photonmaps:
            check(lib().rl_photonmap_gather(m._device.handle, settings.final_gather_radius, self.stream))

    def radiosity_step(self, r0, r1, row, cols, vals, E, rho, B, B_next):
        """Rows [r0, r1) of one Jacobi step (rl_radiosity_step); torch
        tensors on the device, [n][3] iterates."""
        check(lib().rl_radiosity_step(int(r0), int(r1), C.c_void_p(row.data_ptr()), C.c_void_p(cols.data_ptr()),
                                      C.c_void_p(vals.data_ptr()), C.c_void_p(E.data_ptr()),
                                      C.c_void_p(rho.data_ptr()), C.c_void_p(B.data_ptr()),
                                      C.c_void_p(B_next.data_ptr()), self.stream))


def lumels(lightmap: Lightmap, stream=None):
    """Lightmap::lumels(): the map's lumel arrays copied to the host."""
    if lightmap._device is None:
        raise RuntimeError("the lightmap has not been baked yet")
    return lightmap._device.download(stream)


RAW_HDR, TGA_DOUBLE_LDR, TGA_RGBM = 0, 1, 2   # relight::StorageFormat (Relight.h:89-93)


def expand(lightmap: Lightmap, stream=None):
    """Lightmap::expand (Lightmap.cpp:167-193) on the baked lightmap."""
    lightmap._device.expand(stream)


def blur(lightmap: Lightmap, stream=None):
    """Lightmap::blur (Lightmap.cpp:196-220) on the baked lightmap."""
    lightmap._device.blur(stream)


def save(lightmap: Lightmap, path: str, fmt: int = RAW_HDR, stream=None):
    """Lightmap::save (Lightmap.cpp:223-283)."""
    lightmap._device.save(path, fmt, stream)


def to_hdr(lightmap: Lightmap, stream=None):
    """Lightmap::toHdr (Lightmap.cpp:332-349): float RGB, row-major."""
    c = lightmap._device.download(stream, fields=("color",))["color"]
    return c.reshape(lightmap.height, lightmap.width, 3)
