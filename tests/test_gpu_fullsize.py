"""Parity at the benchmarked sizes, through the production launch path.

  - the room workload as benchmarked: 256x256 lightmap, point + 45 degree
    spot + 16-sample area light, then AO with 64 rays of length 2 — the whole
    map bit for bit against the oracle;
  - the terrain workload as benchmarked: 256x256-vertex terrain + 2,000
    boxes (154,050 triangles), one 1024x1024 lightmap and photonmap,
    1,000,000 photons with 3 bounces, gather radius 7, final gather 256 rays
    per lumel.  Photon counts exact and colours within 1e-5 relative (atomic
    float adds); the gather within 1e-4; the final gather baked by the GPU over
    the whole map (8x8 lumel tiles, the default launch tuning, per-triangle
    shading records) from a photonmap pinned to
    the GPU's, and compared bit for bit with the oracle on every 997th lumel;
  - the scene's traversal status word stays 0 (no stack overflow) after
    every pass.
"""
import numpy as np
import pytest

from oracle_bind import Oracle
from relight_b200 import scenes

pytestmark = pytest.mark.gpu


def _lumels(m):
    from relight_b200.device import lumels
    return lumels(m)


def test_room_benchmark_bake_bit_exact(cuda):
    from relight_b200.device import Relight
    w = scenes.room_scene()  # 256^2, the benchmarked room
    assert w.lightmap.width == 256
    rl = Relight()
    rl.bake_direct_light(w.scene, w.mesh, None)
    g_direct = _lumels(w.lightmap)["color"].copy()
    rl.bake_ambient_occlusion(w.scene, w.mesh, None, w.ao, seed=1234)
    g = _lumels(w.lightmap)
    assert w.scene._device.status() == 0
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    lm = orc.maps()[0]
    assert np.array_equal(g["flags"], lm.flags)
    orc.bake_direct(lm)
    assert np.array_equal(g_direct.view(np.uint32), lm.color.view(np.uint32))
    orc.bake_ao(lm, w.ao.samples, w.ao.occluded_fraction, w.ao.max_distance, w.ao.exponent, 1234)
    valid = (lm.flags & 1) > 0
    assert valid.sum() > 40000
    assert np.array_equal(g["color"].view(np.uint32), lm.color.view(np.uint32))


@pytest.fixture(scope="module")
def terrain(cuda):
    """The benchmarked terrain, photons emitted and gathered on the GPU."""
    from relight_b200.device import Relight
    w = scenes.terrain_scene()
    assert w.lightmap.width == 1024 and sum(m.face_count() for m in w.meshes) == 154050
    rl = Relight()
    rl.emit_photons(w.scene, w.settings, seed=31)
    status = w.scene._device.status()
    return w, rl, _lumels(w.photonmap), status


def test_terrain_benchmark_photons_and_gather(terrain):
    w, rl, g, status = terrain
    assert status == 0
    st = w.settings
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    pm = orc.maps("photonmap")[0]
    stored = orc.emit_photons([pm], st.photon_pass_count, st.photon_bounce_count, st.photon_energy_threshold,
                              st.photon_max_distance, 31)
    assert stored > 500000
    assert np.array_equal(g["photons"], pm.photons)
    np.testing.assert_allclose(g["color"], pm.color, rtol=1e-5, atol=1e-6)
    orc.gather(pm, st.final_gather_radius)
    np.testing.assert_allclose(g["gathered"], pm.gathered, rtol=1e-4, atol=1e-6)


def test_terrain_benchmark_final_gather_bit_exact_on_lumel_subset(terrain):
    from relight_b200 import autotune
    w, rl, g, _ = terrain
    st = w.settings
    # the production launch: library defaults, whole-map iterator (8x8 tiles)
    assert autotune.get("indirect") == {"refill": 24, "block": 256}
    assert autotune.get_width() == 2 and autotune.get_speculative() == 0 and autotune.get_pool() == (0, 32)
    rl.bake_indirect_light(w.scene, w.meshes[0], None, st, seed=77)
    gl = _lumels(w.lightmap)
    assert w.scene._device.status() == 0
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    pm = orc.maps("photonmap")[0]
    pm.gathered[:] = g["gathered"]  # pin the photonmap to the GPU's
    lm = orc.maps()[0]
    for first in (0, 498):
        orc.bake_indirect(lm, [pm], st.final_gather_samples, st.final_gather_distance, st.sky_color,
                          st.ambient_color, 77, first, 997)
    idx = np.concatenate([np.arange(0, lm.flags.size, 997), np.arange(498, lm.flags.size, 997)])
    idx = idx[(lm.flags[idx] & 1) > 0]
    assert len(idx) > 1500
    assert (lm.color[idx].sum(1) > 0).sum() > 1000
    assert np.array_equal(gl["color"][idx].view(np.uint32), lm.color[idx].view(np.uint32))
    # every other lumel of the map was baked too (only the subset is checked):
    # the share left black (lumels whose rays all end on surfaces no photon
    # reached, e.g. under the boxes) matches the subset's
    valid = (gl["flags"] & 1) > 0
    lit_all = (gl["color"][valid].sum(1) > 0).mean()
    lit_sub = (lm.color[idx].sum(1) > 0).mean()
    assert lit_all > 0.9 and abs(lit_all - lit_sub) < 0.02, (lit_all, lit_sub)
