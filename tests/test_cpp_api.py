"""The C++ drop-in (include/relight/Relight.h): tests/cpp/bake_room.cpp and
tests/cpp/bake_job.cpp, Relight-style C++ programs (the second bakes through
Relight::bake with base and thread workers, as Relight's demo does), build
against it, and on a GPU bake the same lumels as the same scene baked
through the Python front end."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from relight_b200 import build
from relight_b200.api import (AmbientOcclusionSettings, IndirectLightSettings, Light, LinearLightAttenuation,
                              Lightmap, Material, Mesh, Photonmap, Scene)

F32 = np.float32


@pytest.mark.parametrize("name", ["bake_room", "bake_job"])
def test_cpp_example_builds_against_the_cpp_api(name):
    with tempfile.TemporaryDirectory() as d:
        exe = build.build_cpp_example(d, name)
        assert os.path.exists(exe)


def test_full_bake_job_fan_out():
    """FullBakeJob (Worker.cpp:43-83) through the Python mirror, with a
    recording engine: meshes largest bounding volume first, every worker
    once per mesh with FaceBakeIterator(j, n), LumelBakeIterator(j, n) for
    meshes with fewer faces than workers, JobData filled in."""
    from relight_b200.device import FaceBakeIterator, Job, LumelBakeIterator, Relight, Worker
    scene, room, lm = _python_room()
    small = Mesh.create().add_faces([[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 0, 1]] * 3, None,
                                    [[0, 0], [1, 0], [0, 1]], [0, 1, 2])
    calls = []

    class Record(Job):
        def execute(self, data):
            calls.append((data.scene.meshes.index(data.mesh), type(data.iterator).__name__, data.iterator.first,
                          data.iterator.step, data.worker, data.relight))

    sc = Scene()
    sc.begin()
    for m in (scene.meshes[1].source[0], small, scene.meshes[0].source[0]):
        sc.add_mesh(m)
    sc.end()
    rl = Relight()
    workers = [Worker() for _ in range(3)]
    rl.bake(sc, Record(), Worker(), workers)
    # the room (1000 units^3) first, then the crate, then the flat triangle (volume 0, 1 face < 3 workers)
    assert [c[0] for c in calls] == [2] * 3 + [0] * 3 + [1] * 3
    assert [c[1] for c in calls] == ["FaceBakeIterator"] * 6 + ["LumelBakeIterator"] * 3
    assert [(c[2], c[3]) for c in calls] == [(j, 3) for j in range(3)] * 3
    assert [c[4] for c in calls] == workers * 3 and all(c[5] is rl for c in calls)


def _box(mesh, lo, hi, inward, cell, material):
    """tests/cpp/bake_room.cpp's box(): same vertices, normals, uvs, order."""
    lo, hi = np.asarray(lo, F32), np.asarray(hi, F32)
    pos, nrm, uv, idx = [], [], [], []
    for axis in range(3):
        i, j = (axis + 1) % 3, (axis + 2) % 3
        for side in (0, 1):
            c = hi[axis] if side else lo[axis]
            n = np.zeros(3, F32)
            n[axis] = (1.0 if side else -1.0) * (-1.0 if inward else 1.0)
            cx, cy = cell % 4, cell // 4
            cell += 1
            u0, v0 = F32((cx * 16 + 1) / 64.0), F32((cy * 16 + 1) / 64.0)
            u1, v1 = F32((cx * 16 + 15) / 64.0), F32((cy * 16 + 15) / 64.0)
            base = len(pos)
            for (a, b), t in zip(((0, 0), (1, 0), (1, 1), (0, 1)), ((u0, v0), (u1, v0), (u1, v1), (u0, v1))):
                p = np.zeros(3, F32)
                p[axis] = c
                p[i] = hi[i] if a else lo[i]
                p[j] = hi[j] if b else lo[j]
                pos.append(p); nrm.append(n); uv.append(t)
            idx += [base + k for k in (0, 1, 2, 0, 2, 3)]
    mesh.add_faces(np.array(pos), np.array(nrm), None, np.array(uv, F32), np.array(idx), material)


def _python_room():
    scene = Scene()
    scene.begin()
    room, crate = Mesh.create(), Mesh.create()
    _box(room, (0, 0, 0), (10, 10, 10), True, 0, Material((0.7, 0.7, 0.7)))
    _box(crate, (3, 0, 4), (6, 3, 6), False, 6, Material((0.8, 0.2, 0.2)))
    r, c = scene.add_mesh(room), scene.add_mesh(crate)
    lm, pm = Lightmap(64, 64), Photonmap(64, 64)
    lm.add_mesh(r); lm.add_mesh(c); pm.add_mesh(r); pm.add_mesh(c)
    scene.add_light(Light.create_point_light((5, 9, 5), 10.0, (1, 1, 1), 1.0))
    scene.add_light(Light.create_spot_light((2, 8, 2), (0.5, -0.7, 0.5), 0.9238795, 10.0, (1.0, 0.9, 0.7), 1.0))
    lmesh = Mesh.create().add_faces([[-0.5, 0, -0.5], [0.5, 0, -0.5], [0.5, 0, 0.5], [-0.5, 0, 0.5]],
                                    [[0, -1, 0]] * 4, None, [[0, 0], [1, 0], [1, 1], [0, 1]], [0, 1, 2, 0, 2, 3])
    area = Light.create_area_light(lmesh, (7, 9, 7), (0.8, 0.9, 1.0), 1.0)
    area.set_attenuation(LinearLightAttenuation(10.0))
    scene.add_light(area)
    scene.end()
    return scene, r, lm


def _load_map(path, n):
    raw = np.fromfile(path, dtype=np.uint8)
    return raw[:4 * n].view(np.int32), raw[4 * n:].view(np.float32).reshape(n, 3)


@pytest.mark.gpu
def test_cpp_relight_bake_matches_the_python_front_end(cuda):
    """tests/cpp/bake_job.cpp: Relight::bake with 3 base workers (direct +
    final gather per mesh and worker) against the Python mirror's
    Relight.bake; 4 thread workers (direct light) against the whole-map
    direct bake, bit for bit."""
    from relight_b200.device import Job, Relight, Worker, lumels
    with tempfile.TemporaryDirectory() as d:
        exe = build.build_cpp_example(d, "bake_job")
        out = os.path.join(d, "job")
        r = subprocess.run([exe, out], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        n = 64 * 64
        flags_w, col_w = _load_map(out + ".workers.bin", n)
        flags_t, col_t = _load_map(out + ".threads.bin", n)
    st = IndirectLightSettings(1, 1, 0.05, 20.0, 16, 20.0, 7, (0.2, 0.2, 0.3), (0, 0, 0))

    class Bake(Job):
        def __init__(self, both):
            self.both = both

        def execute(self, data):
            data.relight.bake_direct_light(data.scene, data.mesh, data.worker, data.iterator)
            if self.both:
                data.relight.bake_indirect_light(data.scene, data.mesh, data.worker, st, data.iterator)

    scene, room, lm = _python_room()
    rl = Relight(seed=0x5EED)
    rl.emit_photons(scene, st)
    rl.bake(scene, Bake(True), Worker(), [Worker() for _ in range(3)])
    g = lumels(lm)
    assert (g["flags"] & 1).sum() > 1000
    assert np.array_equal(flags_w, g["flags"])
    # photon deposits are atomic float sums: the final gather within their tolerance
    np.testing.assert_allclose(col_w, g["color"], rtol=1e-4, atol=1e-6)
    scene, room, lm = _python_room()
    rl = Relight(seed=0x5EED)
    rl.bake_direct_light(scene, room, None)  # LumelBakeIterator(0, 1): the whole shared map
    g = lumels(lm)
    assert np.array_equal(flags_t, g["flags"])
    assert np.array_equal(col_t.view(np.uint32), g["color"].view(np.uint32))


@pytest.mark.gpu
def test_cpp_program_bakes_what_the_python_front_end_bakes(cuda):
    from relight_b200.device import Relight, lumels
    with tempfile.TemporaryDirectory() as d:
        exe = build.build_cpp_example(d)
        out = os.path.join(d, "room")
        r = subprocess.run([exe, out], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        n = 64 * 64

        def load(path):
            raw = np.fromfile(path, dtype=np.uint8)
            return raw[:4 * n].view(np.int32), raw[4 * n:].view(np.float32).reshape(n, 3)

        cpp_flags, cpp_ao = load(out + ".direct_ao.bin")
        _, cpp_final = load(out + ".final.bin")
    scene, room, lm = _python_room()
    rl = Relight(seed=0x5EED)
    rl.bake_direct_light(scene, room, None)
    rl.bake_ambient_occlusion(scene, room, None, AmbientOcclusionSettings(16, 0.8, 2.0, 1.0))
    g = lumels(lm)
    assert (g["flags"] & 1).sum() > 1000
    assert np.array_equal(cpp_flags, g["flags"])
    assert np.array_equal(cpp_ao, g["color"])
    st = IndirectLightSettings(1, 1, 0.05, 20.0, 16, 20.0, 7, (0.2, 0.2, 0.3), (0, 0, 0))
    rl.emit_photons(scene, st)
    rl.bake_indirect_light(scene, room, None, st)
    g = lumels(lm)
    assert not np.array_equal(g["color"], cpp_ao)
    np.testing.assert_allclose(cpp_final, g["color"], rtol=1e-4, atol=1e-6)
