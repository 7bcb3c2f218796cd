"""Host logic of the Relight-API mirror (relight_b200/api.py): state machine,
error behaviour, presets and the float32 scene build, the last checked
against the reference baker where oracle/_ref exists."""
import math

import numpy as np
import pytest

from oracle_bind import RefScene, reference_available
from relight_b200 import scenes
from relight_b200.api import (AmbientOcclusionSettings, IndirectLightSettings, Light, Lightmap, Material, Mesh,
                              Photonmap, RelightStatus, Scene, Texture, TexturedMaterial, flatten)


def test_presets_match_reference():
    # Relight.cpp:43-120 and 123-172
    assert [(p.photon_pass_count, p.photon_bounce_count, p.final_gather_samples) for p in
            (IndirectLightSettings.draft(), IndirectLightSettings.fast(), IndirectLightSettings.best(),
             IndirectLightSettings.production())] == [(8, 1, 32), (16, 3, 64), (32, 3, 128), (64, 4, 1024)]
    for p in (IndirectLightSettings.draft(), IndirectLightSettings.production()):
        assert p.final_gather_radius == 7 and p.photon_energy_threshold == pytest.approx(0.05)
        assert p.photon_max_distance == 10.0 and p.final_gather_distance == 50.0
    assert [a.samples for a in (AmbientOcclusionSettings.draft(), AmbientOcclusionSettings.fast(),
                                AmbientOcclusionSettings.best(), AmbientOcclusionSettings.production())] == \
        [128, 256, 1024, 2048]
    a = AmbientOcclusionSettings.draft()
    assert (a.occluded_fraction, a.max_distance, a.exponent) == (pytest.approx(0.8), pytest.approx(0.6), 1.0)


def test_scene_state_machine():
    s = Scene()
    assert s.end() == RelightStatus.RelightInvalidCall
    assert s.begin() == RelightStatus.RelightSuccess
    assert s.begin() == RelightStatus.RelightInvalidCall
    m = Mesh.create().add_faces([[0, 0, 0], [1, 0, 0], [0, 1, 0]], None, None, [[0, 0], [1, 0], [0, 1]], [0, 1, 2])
    s.add_mesh(m)
    assert s.end() == RelightStatus.RelightSuccess
    assert s.end() == RelightStatus.RelightInvalidCall


def test_a_mesh_takes_one_lightmap_and_one_photonmap():
    m = Mesh.create()
    lm, lm2, pm = Lightmap(8, 8), Lightmap(8, 8), Photonmap(8, 8)
    assert lm.add_mesh(m) == RelightStatus.RelightSuccess
    assert lm2.add_mesh(m) == RelightStatus.RelightInvalidCall
    assert pm.add_mesh(m) == RelightStatus.RelightSuccess
    assert pm.add_mesh(m) == RelightStatus.RelightInvalidCall


def test_sixteen_bit_index_limit():
    m = Mesh.create()
    p = np.zeros((40000, 3), np.float32)
    m.add_faces(p, None, None, None, [0, 1, 2])
    with pytest.raises(ValueError):
        m.add_faces(p, None, None, None, [0, 1, 2])


def test_flatten_offsets_and_materials():
    red, blue = Material((1, 0, 0)), Material((0, 0, 1))
    tri = ([[0, 0, 0], [1, 0, 0], [0, 1, 0]], None, None, [[0, 0], [1, 0], [0, 1]], [0, 1, 2])
    a = Mesh.create().add_faces(*tri, red)
    b = Mesh.create().add_faces(*tri, blue).add_faces(*tri, red)
    s = Scene()
    s.begin()
    s.add_mesh(a)
    s.add_mesh(b)
    s.end()
    f = s.flat
    assert list(f.mesh_first_tri) == [0, 1, 3]
    assert f.tris.tolist() == [[0, 1, 2], [3, 4, 5], [6, 7, 8]]
    assert f.vmat.tolist() == [0, 0, 0, 1, 1, 1, 0, 0, 0]
    assert np.allclose(f.mat_rgb, [[1, 0, 0], [0, 0, 1]])


def test_directional_light_plane_and_area_light_centroids():
    d = Light.create_directional_light((0.3, -1.0, 0.2))
    assert np.array_equal(d.emitter_plane[:3], np.float32([0.3, -1.0, 0.2]))
    m = Mesh.create().add_faces([[0, 0, 0], [3, 0, 0], [0, 3, 0]], None, None, None, [0, 1, 2])
    a = Light.create_area_light(m, (0, 5, 0))
    assert np.allclose(a.vertices, [[1, 1, 0]])
    assert a.attenuation.radius == 0.0  # the light mesh is flat: bounds volume 0 (scene/Light.cpp:219)


def test_texture_rules():
    with pytest.raises(ValueError):
        Texture.create(2, 2, 3, np.zeros(5, np.uint8))
    with pytest.raises(ValueError):
        TexturedMaterial(None, (1, 1, 1))


@pytest.mark.skipif(not reference_available(), reason="reference build (oracle/_ref) not present")
def test_transformed_meshes_match_reference_bit_for_bit():
    rng = np.random.default_rng(4)
    c, s_ = math.cos(0.7), math.sin(0.7)
    # a rotation about y, a scale and a translation, row-vector convention (Types.h:1188-1196)
    M = np.array([[c * 1.5, 0, -s_ * 1.5, 0], [0, 0.8, 0, 0], [s_, 0, c, 0], [3.25, -1.5, 7.0, 1]], np.float32)
    src = Mesh.create()
    n = rng.normal(size=(30, 3)).astype(np.float32)
    n /= np.linalg.norm(n, axis=1, keepdims=True).astype(np.float32)
    src.add_faces(rng.uniform(-5, 5, (30, 3)), n, None, rng.random((30, 2)), np.arange(30))
    sc = Scene()
    sc.begin()
    inst = sc.add_mesh(src, M)
    lm = Lightmap(32, 32)
    lm.add_mesh(inst)
    sc.end()
    ref = RefScene(sc)
    p, q = ref.mesh_vertices(inst)
    assert np.array_equal(p, inst.positions)
    assert np.array_equal(q, inst.normals)


@pytest.mark.skipif(not reference_available(), reason="reference build (oracle/_ref) not present")
def test_scene_bounds_match_reference():
    w = scenes.terrain_scene(verts=32, n_boxes=20, size=64, tiles=2)
    ref = RefScene(w.scene)
    lo, hi = np.zeros(3, np.float32), np.zeros(3, np.float32)
    from oracle_bind import ptr
    ref.lib.ref_scene_bounds(ref.h, ptr(lo), ptr(hi))
    assert np.array_equal(lo, w.scene.flat.bounds_lo) and np.array_equal(hi, w.scene.flat.bounds_hi)
