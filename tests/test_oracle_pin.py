"""Pins the oracle (the C restatement in oracle/) before it is trusted:
  1. against the golden fixtures made by the reference baker compiled from
     its own sources (tests/golden/make_golden.py) — bit-exact;
  2. against the live reference build, where oracle/_ref/ exists — bit-exact
     for the deterministic passes, statistical for the Monte-Carlo passes
     (the reference draws from the C library's rand(), the oracle from
     Philox; both estimate the same expectation);
  3. Philox4x32-10 against the Random123 known-answer vectors.
CPU only.
"""
import os

import numpy as np
import pytest

from oracle_bind import LumelMap, Oracle, RefScene, philox, ptr, reference_available
from relight_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
needs_ref = pytest.mark.skipif(not reference_available(), reason="reference build (oracle/_ref) not present")


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


# ------------------------------------------------------------------ Philox

@pytest.mark.parametrize("ctr,key,expect", [
    ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
    ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
    ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
     [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
])
def test_philox_known_answers(ctr, key, expect):
    assert list(philox(ctr, key)) == expect


# ------------------------------------------------------- golden fixtures

def test_scene_build_matches_golden():
    g = golden("room64.npz")
    w = scenes.room_scene(size=64)
    assert np.array_equal(w.mesh.positions, g["mesh_pos"])
    assert np.array_equal(w.mesh.normals, g["mesh_nrm"])
    area = [l for l in w.scene.lights if l.vertices is not None][0]
    assert np.array_equal(area.vertices, g["light_vertices"])


def test_texel_init_and_direct_light_match_golden():
    g = golden("room64.npz")
    w = scenes.room_scene(size=64)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    lm = orc.maps()[0]
    for f in ("flags", "face", "position", "normal"):
        assert np.array_equal(getattr(lm, f), g[f]), f
    orc.bake_direct(lm)
    assert (g["color"].sum(1) > 0).sum() > 500
    assert np.array_equal(lm.color, g["color"])


def test_trace_segments_match_golden():
    g = golden("trace_room.npz")
    w = scenes.room_scene(size=64)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    r = orc.trace_segments(g["seg"], 15)
    assert np.array_equal(r["hit"], g["hit"])
    m = g["hit"] > 0
    for f in ("point", "normal", "rgba", "uv", "mesh"):
        assert np.array_equal(r[f][m], g[f][m]), f


# fields traceSegment fills for each flag set (rt/Embree.cpp:167-174)
_TRACE_FIELDS = {15: ("point", "normal", "rgba", "uv", "mesh"), 31: ("point", "normal", "rgba", "uv", "mesh")}


def test_textured_alpha_trace_and_direct_match_golden():
    """RGBA textures (Texture::colorAt: nearest texel, wrap, out-of-range
    colour) and the HitUseAlpha re-trace through cut-out texels
    (rt/Embree.cpp:157-165): traceSegment with and without HitUseAlpha, and
    direct light whose shadow rays pass through alpha <= 0.1."""
    from golden.make_golden import segments
    g = golden("textured_room48.npz")
    w = scenes.room_scene(size=48, textured=True)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    seg = segments(w.scene.flat, 6000, 13)
    assert np.array_equal(seg, g["seg"])
    for flags in (15, 31):
        r = orc.trace_segments(seg, flags)
        assert np.array_equal(r["hit"], g[f"hit_{flags}"])
        m = g[f"hit_{flags}"] > 0
        for f in _TRACE_FIELDS[flags]:
            assert np.array_equal(r[f][m], g[f"{f}_{flags}"][m]), (flags, f)
    # the alpha re-trace changed hundreds of results, and textures coloured them
    moved = (g["hit_15"] != g["hit_31"]) | np.any(g["point_15"] != g["point_31"], 1)
    assert moved.sum() > 100
    m = g["hit_15"] > 0
    assert len(np.unique(g["rgba_15"][m], axis=0)) > 50
    lm = orc.maps()[0]
    assert np.array_equal(lm.flags, g["flags"])
    orc.bake_direct(lm)
    assert (g["color"].sum(1) > 0).sum() > 300
    assert np.array_equal(lm.color, g["color"])


@needs_ref
def test_textured_alpha_matches_reference():
    """The same on a larger textured room, live against the reference."""
    from golden.make_golden import segments
    w = scenes.room_scene(size=96, textured=True, seed=4)
    ref = RefScene(w.scene)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    seg = segments(w.scene.flat, 20000, 3)
    for flags in (15, 31):
        r, o = ref.trace_segments(seg, flags), orc.trace_segments(seg, flags)
        assert np.array_equal(r["hit"], o["hit"])
        m = r["hit"] > 0
        for f in _TRACE_FIELDS[flags]:
            assert np.array_equal(r[f][m], o[f][m]), (flags, f)
    ref.lib.ref_bake_direct(ref.h, ref.mesh(w.mesh), 0, 0, 1)
    lm = orc.maps()[0]
    orc.bake_direct(lm)
    r = ref.lumels(w.lightmap)
    assert (r.color.sum(1) > 0).sum() > 1000
    assert np.array_equal(lm.color, r.color)


@pytest.mark.parametrize("W,H", [(48, 48), (56, 40), (40, 56)])
def test_photon_gather_matches_golden(W, H):
    from golden.make_golden import gather_inputs
    g = golden("gather.npz")[f"gathered_{W}x{H}"]
    color, photons = gather_inputs(W, H, W * 100 + H)
    pm = LumelMap(W, H)
    pm.color[:] = color
    pm.photons[:] = photons
    w = scenes.room_scene(size=16, n_boxes=0, area_light=False, spot_light=False)
    Oracle(w.scene.flat).gather(pm, 7)
    assert np.array_equal(pm.gathered, g)


def test_pairwise_form_factors_match_golden():
    g = golden("ff_room24.npz")
    w = scenes.radiosity_room(size=24)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    lm = orc.maps()[0]
    valid = np.nonzero(lm.flags & 1)[0]
    assert np.array_equal(lm.position[valid], g["pos"]) and np.array_equal(lm.normal[valid], g["nrm"])
    row, cols, vals = orc.ff_pairwise(g["pos"], g["nrm"], 0.1)
    assert np.array_equal(row, g["row"]) and np.array_equal(cols, g["cols"]) and np.array_equal(vals, g["vals"])
    # every row sums to one (refineFormFactors)
    sums = np.add.reduceat(vals.astype(np.float64), row[:-1][np.diff(row) > 0])
    np.testing.assert_allclose(sums, 1.0, rtol=1e-5)


# ------------------------------------------------------ live reference

@needs_ref
def test_terrain_build_and_texels_match_reference():
    w = scenes.terrain_scene(verts=48, n_boxes=50, size=128, tiles=2)
    ref = RefScene(w.scene)
    for m in w.meshes:
        p, n = ref.mesh_vertices(m)
        assert np.array_equal(p, m.positions) and np.array_equal(n, m.normals)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    for m, lm in zip(w.scene.flat.lightmaps + w.scene.flat.photonmaps, orc.maps() + orc.maps("photonmap")):
        r = ref.lumels(m)
        for f in ("flags", "face", "position", "normal"):
            assert np.array_equal(getattr(lm, f), getattr(r, f)), f


@needs_ref
def test_direct_light_matches_reference_with_directional_light():
    w = scenes.terrain_scene(verts=40, n_boxes=40, size=96, tiles=2)
    ref = RefScene(w.scene)
    ref.lib.ref_bake_direct(ref.h, ref.mesh(w.meshes[0]), 0, 0, 1)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    lm = orc.maps()[0]
    orc.bake_direct(lm)
    r = ref.lumels(w.lightmap)
    assert (r.color.sum(1) > 0).sum() > 1000
    assert np.array_equal(lm.color, r.color)


@needs_ref
def test_pairwise_form_factors_match_reference():
    w = scenes.radiosity_room(size=40)
    ref = RefScene(w.scene, radiancemaps=(w.radiancemap,))
    row, cols, vals, pos, nrm = ref.radiosity(0.1)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    r2, c2, v2 = orc.ff_pairwise(pos, nrm, 0.1)
    assert np.array_equal(row, r2) and np.array_equal(cols, c2) and np.array_equal(vals, v2)


def _rmse(a, b):
    return float(np.sqrt(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2)))


@needs_ref
def test_ambient_occlusion_statistics_match_reference():
    """Same expectation at equal sample count (64): over 4,096 seeded texels,
    the per-texel RMSE against an FP64 2,048-sample estimate is within 1.1x
    of the reference's, and neither is biased beyond 3 standard errors."""
    w = scenes.room_scene(size=128)
    ref = RefScene(w.scene)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    lm = orc.maps()[0]
    lm.color[:] = 1.0
    ref.lib.ref_map_set_colors(ref.h, ref.maps[id(w.lightmap)], ptr(np.ones_like(lm.color)))
    ref.lib.ref_set_rand(0, 17)
    ref.lib.ref_bake_ao(ref.h, ref.mesh(w.mesh), 64, 0.8, 2.0, 1.0, 0, 0, 1)
    orc.bake_ao(lm, 64, 0.8, 2.0, 1.0, 4242)
    r = ref.lumels(w.lightmap)
    valid = np.nonzero(lm.flags & 1)[0]
    tex = np.sort(np.random.default_rng(3).choice(valid, 4096, replace=False))
    ex = orc.ao_expect(lm, tex, 2048, 0.8, 2.0, 99)
    e_ref, e_or = r.color[tex, 0] - ex, lm.color[tex, 0] - ex
    assert _rmse(lm.color[tex, 0], ex) <= 1.1 * _rmse(r.color[tex, 0], ex)
    for e in (e_or, e_ref):
        assert abs(e.mean()) < 3 * e.std() / np.sqrt(len(tex)) + 1e-3


@needs_ref
def test_photon_pass_statistics_match_reference():
    """Photons: the deposit count and the gathered photonmap's mean colour
    agree with the reference within Monte-Carlo noise (2 passes)."""
    w = scenes.terrain_scene(verts=40, n_boxes=40, size=96, tiles=2, passes=2, bounces=3)
    st = w.settings
    ref = RefScene(w.scene)
    ref.lib.ref_set_rand(0, 3)
    ref.lib.ref_emit_photons(ref.h, st.photon_pass_count, st.photon_bounce_count, st.photon_energy_threshold,
                             st.photon_max_distance, st.final_gather_radius)
    r = ref.lumels(w.photonmap)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    pm = orc.maps("photonmap")[0]
    orc.emit_photons([pm], st.photon_pass_count, st.photon_bounce_count, st.photon_energy_threshold,
                     st.photon_max_distance, 11)
    orc.gather(pm, st.final_gather_radius)
    n_ref, n_or = r.photons.sum(), pm.photons.sum()
    assert abs(n_ref - n_or) < 5 * np.sqrt(n_ref) + 0.01 * n_ref
    c_ref, c_or = r.color.sum(0), pm.color.sum(0)
    np.testing.assert_allclose(c_or, c_ref, rtol=0.03)
    v = (pm.flags & 1) > 0
    np.testing.assert_allclose(pm.gathered[v].mean(0), r.gathered[v].mean(0), rtol=0.03)


@needs_ref
def test_final_gather_statistics_match_reference():
    """Final gather from the same (reference-gathered) photonmap at equal
    sample count (32): over 4,096 seeded texels, the per-texel RMSE against
    an FP64 2,048-sample estimate is within 1.1x of the reference's, and
    neither is biased beyond 3 standard errors (per channel)."""
    w = scenes.terrain_scene(verts=40, n_boxes=40, size=96, tiles=2, passes=1, bounces=2, fg_samples=32)
    st = w.settings
    ref = RefScene(w.scene)
    ref.lib.ref_set_rand(0, 5)
    ref.lib.ref_emit_photons(ref.h, st.photon_pass_count, st.photon_bounce_count, st.photon_energy_threshold,
                             st.photon_max_distance, st.final_gather_radius)
    rp = ref.lumels(w.photonmap)
    sky = np.asarray(st.sky_color, np.float32)
    amb = np.asarray(st.ambient_color, np.float32)
    ref.lib.ref_bake_indirect(ref.h, ref.mesh(w.meshes[0]), st.final_gather_samples, st.final_gather_distance,
                              st.final_gather_radius, ptr(sky), ptr(amb), 0, 0, 1)
    r = ref.lumels(w.lightmap)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    pm = orc.maps("photonmap")[0]
    pm.gathered[:] = rp.gathered
    lm = orc.maps()[0]
    orc.bake_indirect(lm, [pm], st.final_gather_samples, st.final_gather_distance, sky, amb, 77)
    valid = np.nonzero(lm.flags & 1)[0]
    tex = np.sort(np.random.default_rng(4).choice(valid, 4096, replace=False))
    ex = orc.fg_expect(lm, [pm], tex, 2048, st.final_gather_distance, sky, amb, 8)
    assert _rmse(lm.color[tex], ex) <= 1.1 * _rmse(r.color[tex], ex)
    for c in (lm.color[tex], r.color[tex]):
        e = c - ex
        assert (np.abs(e.mean(0)) < 3 * e.std(0) / np.sqrt(len(tex)) + 1e-3).all()


@needs_ref
def test_face_iterator_direct_light_matches_reference():
    """FaceBakeIterator over each mesh of a shared lightmap (the iterator
    Relight's FullBakeJob hands its workers, Worker.cpp:69-73)."""
    w = scenes.terrain_scene(verts=40, n_boxes=40, size=96, tiles=2)
    ref = RefScene(w.scene)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    lm = orc.maps()[0]
    for k, mesh in enumerate(w.meshes):
        ref.lib.ref_bake_direct(ref.h, ref.mesh(mesh), 1, k % 2, 2)
        orc.bake_direct(lm, k % 2, 2, mesh=w.scene.meshes.index(mesh))
    r = ref.lumels(w.lightmap)
    assert (r.color.sum(1) > 0).sum() > 500
    assert np.array_equal(lm.color, r.color)
