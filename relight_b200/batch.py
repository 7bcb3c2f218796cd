"""Many bake jobs in one launch: the rl_batch_* entry points.

A job is one single-job bake call (rl_bake_direct, rl_bake_ao or
rl_bake_indirect) on one lightmap; a batch runs any number of them, over any
scenes and lightmap sizes, as one persistent kernel per pass kind.  The
batch's lumels are bit-identical to the per-job calls made in the order
direct light, AO, final gather (the plain per-job loop, `run_per_job`).

The reference bakes jobs one after another on each worker thread
(Worker.cpp:43-83, Relight.cpp:132-163); it has no batch of its own.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _abi
from ._abi import check, lib
from .device import DeviceMap, DeviceScene, _map_array

DIRECT, AO, INDIRECT = 0, 1, 2


@dataclass
class BakeJob:
    """One pass over one lightmap.  `lights` / `light_vertices` are the flat
    scene's rl_light records (direct light); `photonmaps` the scene's
    photonmaps by slot (final gather)."""
    kind: int
    scene: DeviceScene
    lightmap: DeviceMap
    lights: Optional[np.ndarray] = None
    light_vertices: Optional[np.ndarray] = None
    photonmaps: Sequence[DeviceMap] = ()
    samples: int = 0
    occluded_fraction: float = 0.8
    max_distance: float = 0.0
    exponent: float = 1.0
    sky: Sequence[float] = (0.0, 0.0, 0.0)
    ambient: Sequence[float] = (0.0, 0.0, 0.0)
    seed: int = 0
    iterator: tuple = (0, 0, 1, -1)  # (kind, first, step, mesh): LumelBakeIterator(0, 1)
    begin: int = 0
    end: int = -1

    @staticmethod
    def direct(scene: DeviceScene, lightmap: DeviceMap, **kw) -> "BakeJob":
        f = scene.flat
        return BakeJob(DIRECT, scene, lightmap, lights=f.lights, light_vertices=f.light_vertices, **kw)

    @staticmethod
    def ambient_occlusion(scene: DeviceScene, lightmap: DeviceMap, settings, seed: int, **kw) -> "BakeJob":
        return BakeJob(AO, scene, lightmap, samples=settings.samples, occluded_fraction=settings.occluded_fraction,
                       max_distance=settings.max_distance, exponent=settings.exponent, seed=seed, **kw)

    @staticmethod
    def indirect(scene: DeviceScene, lightmap: DeviceMap, photonmaps: Sequence[DeviceMap], settings, seed: int,
                 **kw) -> "BakeJob":
        return BakeJob(INDIRECT, scene, lightmap, photonmaps=list(photonmaps), samples=settings.final_gather_samples,
                       max_distance=settings.final_gather_distance, sky=tuple(settings.sky_color),
                       ambient=tuple(settings.ambient_color), seed=seed, **kw)

    def nlight_vertices(self) -> int:
        if self.lights is None:
            return 0
        return int(sum(int(l["vertex_count"]) for l in self.lights))


def _job_array(jobs: Sequence[BakeJob]):
    """rl_batch_job records for `jobs` (and the ctypes objects they point into)."""
    keep: List[object] = []
    arr = (_abi.BatchJob * max(len(jobs), 1))()
    for q, j in enumerate(jobs):
        b = arr[q]
        b.kind = j.kind
        b.scene = j.scene.handle.value
        b.lightmap = j.lightmap.handle.value
        if j.photonmaps:
            maps = _map_array(j.photonmaps)
            keep.append(maps)
            b.photonmaps = C.cast(maps, C.c_void_p)
        b.nmaps = len(j.photonmaps)
        if j.lights is not None and len(j.lights):
            b.lights = j.lights.ctypes.data
            b.nlights = len(j.lights)
        if j.light_vertices is not None and len(j.light_vertices):
            b.light_vertices = j.light_vertices.ctypes.data
            b.nlight_vertices = j.nlight_vertices()
        b.samples = j.samples
        b.occluded_fraction = j.occluded_fraction
        b.max_distance = j.max_distance
        b.exponent = j.exponent
        b.sky = (C.c_float * 3)(*[float(x) for x in j.sky])
        b.ambient = (C.c_float * 3)(*[float(x) for x in j.ambient])
        b.seed = j.seed & 0xFFFFFFFFFFFFFFFF
        b.iterator = _abi.Iterator(*j.iterator)
        b.begin = j.begin
        b.end = j.end
    return arr, keep


class Batch:
    """An rl_batch: the job table on the device, launched or replayed as a
    captured CUDA graph."""

    def __init__(self, jobs: Sequence[BakeJob]):
        self.jobs = list(jobs)
        arr, keep = _job_array(self.jobs)
        self.handle = C.c_void_p()
        check(lib().rl_batch_create(arr, len(self.jobs), C.byref(self.handle)))

    def update(self, jobs: Sequence[BakeJob], stream=None):
        """Replace the job table in stream order (a captured graph stays valid)."""
        self.jobs = list(jobs)
        arr, keep = _job_array(self.jobs)
        check(lib().rl_batch_update(self.handle, arr, len(self.jobs), stream))

    def launch(self, stream=None):
        check(lib().rl_batch_launch(self.handle, stream))

    def capture(self, stream):
        """Capture one launch into a CUDA graph on `stream` (not the default stream)."""
        check(lib().rl_batch_capture(self.handle, stream))

    def replay(self, stream=None):
        check(lib().rl_batch_replay(self.handle, stream))

    @property
    def work_items(self) -> int:
        n = C.c_int64()
        check(lib().rl_batch_work_items(self.handle, C.byref(n)))
        return n.value

    def close(self):
        if self.handle:
            check(lib().rl_batch_destroy(self.handle))
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_per_job(jobs: Sequence[BakeJob], stream=None):
    """The plain per-job loop: one single-job call per job, in batch order
    (direct light, then AO, then final gather)."""
    for j in jobs:
        if j.begin != 0 or j.end != -1:
            raise ValueError("the single-job calls bake whole iterators: slices need a Batch")
    for kind in (DIRECT, AO, INDIRECT):
        for j in jobs:
            if j.kind != kind:
                continue
            it = C.byref(_abi.Iterator(*j.iterator))
            if kind == DIRECT:
                nl = 0 if j.lights is None else len(j.lights)
                check(lib().rl_bake_direct(j.scene.handle, j.lightmap.handle,
                                           None if not nl else C.c_void_p(j.lights.ctypes.data), nl,
                                           None if j.light_vertices is None or not len(j.light_vertices)
                                           else C.c_void_p(j.light_vertices.ctypes.data),
                                           j.nlight_vertices(), it, stream))
            elif kind == AO:
                check(lib().rl_bake_ao(j.scene.handle, j.lightmap.handle, j.samples, j.occluded_fraction,
                                       j.max_distance, j.exponent, j.seed, it, stream))
            else:
                sky = (C.c_float * 3)(*[float(x) for x in j.sky])
                amb = (C.c_float * 3)(*[float(x) for x in j.ambient])
                check(lib().rl_bake_indirect(j.scene.handle, j.lightmap.handle, _map_array(j.photonmaps),
                                             len(j.photonmaps), j.samples, j.max_distance, sky, amb, j.seed, it,
                                             stream))


@dataclass
class ResidentBatch:
    """A batch workload on the device: each scene's BVH and gathered
    photonmap, and each job's lightmap with its lumels rasterised."""
    scenes: List[DeviceScene]
    photonmaps: List[List[DeviceMap]]
    lightmaps: List[DeviceMap]
    jobs: List[BakeJob]
    texels: int = 0

    def clear(self, stream=None):
        for m in self.lightmaps:
            m.clear(colors=True, photons=False, stream=stream)


@dataclass
class ResidentScenes:
    """Scenes on the device: each one's BVH and its gathered photonmaps."""
    scenes: List[DeviceScene]
    photonmaps: List[List[DeviceMap]]
    workload: object

    def nbytes(self) -> int:
        """Device bytes held: BVH nodes and triangle records, the flat
        scene's arrays as uploaded, and the photonmaps."""
        total = 0
        for ds, pms in zip(self.scenes, self.photonmaps):
            st = ds.bvh_stats()
            f = ds.flat
            total += st["nodes"] * 64 + f.ntris * 48
            for name in ("pos", "nrm", "uv0", "uv1", "vmat", "tris", "mat_rgb", "tex_pixels"):
                a = getattr(f, name, None)
                if isinstance(a, np.ndarray):
                    total += a.nbytes
            total += sum(DeviceMap.nbytes(m.width, m.height) for m in pms)
        return total


def make_resident_scenes(workload, stream=None, builder: int = 0, photons: bool = True) -> ResidentScenes:
    """Build each scene's BVH (binned SAH on the host by default; 1 = the
    device LBVH), then emit and gather its photons."""
    from .device import Relight
    scenes, pmaps = [], []
    for k, wl in enumerate(workload.scenes):
        rl = Relight(stream, seed=0xBA7C + k, builder=builder)
        ds = rl.device_scene(wl.scene)
        if photons:
            rl.emit_photons(wl.scene, wl.settings)
        scenes.append(ds)
        pmaps.append([m._device for m in wl.scene.flat.photonmaps])
    return ResidentScenes(scenes, pmaps, workload)


def make_resident(workload, stream=None, builder: int = 0, passes=(DIRECT, AO, INDIRECT)) -> ResidentBatch:
    """Upload a scenes.BatchWorkload: make its scenes resident, rasterise
    each job's lightmap over all its scene's meshes, and make one BakeJob
    per pass per job."""
    rs = make_resident_scenes(workload, stream, builder, photons=INDIRECT in passes)
    scenes, pmaps = rs.scenes, rs.photonmaps
    lightmaps, jobs = [], []
    texels = 0
    for spec in workload.jobs:
        ds = scenes[spec.scene]
        wl = workload.scenes[spec.scene]
        lm = DeviceMap(0, spec.side, spec.side)
        for mi in range(len(wl.scene.flat.mesh_photonmap)):
            lm.add_mesh(ds, mi, stream)
        lightmaps.append(lm)
        texels += spec.side * spec.side
        if DIRECT in passes:
            jobs.append(BakeJob.direct(ds, lm))
        if AO in passes:
            jobs.append(BakeJob.ambient_occlusion(ds, lm, workload.ao, seed=spec.seed ^ 0xA0))
        if INDIRECT in passes:
            jobs.append(BakeJob.indirect(ds, lm, pmaps[spec.scene], wl.settings, seed=spec.seed ^ 0xF6))
    return ResidentBatch(scenes, pmaps, lightmaps, jobs, texels)
