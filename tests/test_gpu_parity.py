"""Parity of the CUDA passes with the oracle (the C restatement), through the
C ABI, on seeded synthetic scenes.

Tolerances:
  - ray tracing, texel rasterisation, direct light, AO, final gather from a
    fixed photonmap, pairwise and hemisphere form factors: bit-exact (the
    kernels follow the oracle's float operation order with --fmad=false and
    draw the same Philox numbers);
  - photon deposit: integer counts exact, colour sums within 1e-5 relative
    (atomic float adds in arbitrary order);
  - radiosity Jacobi (fp32, 50 iterations): within 1e-4 relative of an FP64
    Jacobi on the same form factors.
"""
import ctypes as C

import numpy as np
import pytest

from oracle_bind import LumelMap, Oracle, jacobi_f64
from relight_b200 import scenes

pytestmark = pytest.mark.gpu


def _dev(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _relight(builder=0):
    from relight_b200.device import Relight
    return Relight(builder=builder)


def _lumels(m):
    from relight_b200.device import lumels
    return lumels(m)


def _segments(rng, lo, hi, n):
    a = rng.uniform(lo, hi, (n, 3))
    b = rng.uniform(lo, hi, (n, 3))
    return np.concatenate([a, b], 1).astype(np.float32)


@pytest.mark.parametrize("builder", [0, 1])
@pytest.mark.parametrize("which", ["room", "terrain", "textured"])
def test_trace_segments_match_oracle(cuda, which, builder):
    """Segments through the C ABI; "textured" adds RGBA textures with cut-out
    texels (Texture::colorAt and the HitUseAlpha re-trace)."""
    import torch
    from relight_b200 import _abi
    if which in ("room", "textured"):
        w = scenes.room_scene(size=64, textured=which == "textured")
        scene = w.scene
    else:
        w = scenes.terrain_scene(verts=48, n_boxes=60, size=128, tiles=2)
        scene = w.scene
    flat = scene.flat
    rl = _relight(builder)
    ds = rl.device_scene(scene)
    assert ds.bvh_stats()["depth"] > 4
    orc = Oracle(flat).bind_scene(scene)
    rng = np.random.default_rng(11)
    seg = _segments(rng, flat.bounds_lo - 1, flat.bounds_hi + 1, 20000)
    for flags in (_abi.HIT_ALL, _abi.HIT_UV | _abi.HIT_NORMAL, _abi.HIT_ALL | _abi.HIT_USE_ALPHA):
        ref = orc.trace_segments(seg, flags)
        n = seg.shape[0]
        d_seg = _dev(seg, torch)
        hit = torch.zeros(n, dtype=torch.int32, device="cuda")
        mf = torch.zeros((n, 2), dtype=torch.int32, device="cuda")
        pt = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
        nm = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
        rgba = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
        uv = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
        _abi.check(_abi.lib().rl_trace_segments(ds.handle, n, d_seg.data_ptr(), flags, hit.data_ptr(), None,
                                                mf.data_ptr(), pt.data_ptr(), nm.data_ptr(), rgba.data_ptr(),
                                                uv.data_ptr(), None))
        torch.cuda.synchronize()
        assert np.array_equal(hit.cpu().numpy(), ref["hit"])
        m = ref["hit"] > 0
        assert m.sum() > 1000
        assert np.array_equal(mf.cpu().numpy()[:, 0], ref["mesh"])
        assert np.array_equal(mf.cpu().numpy()[:, 1], ref["face"])
        assert np.array_equal(pt.cpu().numpy()[m], ref["point"][m])
        assert np.array_equal(nm.cpu().numpy()[m], ref["normal"][m])
        assert np.array_equal(uv.cpu().numpy()[m], ref["uv"][m])
        assert np.array_equal(rgba.cpu().numpy()[m], ref["rgba"][m])


def test_texel_rasterisation_matches_oracle(cuda):
    for scene, maps in ((scenes.room_scene(size=96).scene, "lightmap"),
                        (scenes.radiosity_room(size=48).scene, "lightmap")):
        rl = _relight()
        rl.device_scene(scene)
        orc = Oracle(scene.flat).bind_scene(scene)
        for m, lm in zip(scene.flat.lightmaps, orc.maps(maps)):
            g = _lumels(m)
            for f in ("flags", "face", "position", "normal"):
                assert np.array_equal(g[f], getattr(lm, f)), f


def test_direct_light_bit_exact(cuda):
    w = scenes.room_scene(size=128)
    rl = _relight()
    rl.bake_direct_light(w.scene, w.mesh, None)
    g = _lumels(w.lightmap)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    lm = orc.maps()[0]
    orc.bake_direct(lm)
    assert (g["color"].sum(1) > 0).sum() > 1000
    assert np.array_equal(g["color"], lm.color)


def test_textured_direct_light_and_ao_bit_exact(cuda):
    """Direct light whose shadow rays pass through cut-out texels (alpha <=
    0.1, re-traced 1 unit further on), then AO, on the textured room."""
    w = scenes.room_scene(size=128, textured=True)
    rl = _relight()
    rl.bake_direct_light(w.scene, w.mesh, None)
    g_direct = _lumels(w.lightmap)["color"].copy()
    rl.bake_ambient_occlusion(w.scene, w.mesh, None, w.ao, seed=12)
    g = _lumels(w.lightmap)
    assert w.scene._device.status() == 0
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    lm = orc.maps()[0]
    orc.bake_direct(lm)
    assert (lm.color.sum(1) > 0).sum() > 1000
    assert np.array_equal(g_direct, lm.color)
    # the cut-out texels changed the shadows (the same room untextured differs)
    wu = scenes.room_scene(size=128)
    ou = Oracle(wu.scene.flat).bind_scene(wu.scene)
    lu = ou.maps()[0]
    ou.bake_direct(lu)
    assert np.any(lu.color != lm.color, 1).sum() > 100
    orc.bake_ao(lm, w.ao.samples, w.ao.occluded_fraction, w.ao.max_distance, w.ao.exponent, 12)
    assert np.array_equal(g["color"], lm.color)


def test_textured_photon_bounce_colours(cuda):
    """Photon deposits coloured by Face::colorAt through the texture
    (baker/Photons.cpp:116-119, hit.m_color)."""
    from relight_b200.api import Photonmap, Scene
    w = scenes.room_scene(size=64, textured=True)
    sc = Scene()
    sc.begin()
    inst = sc.add_mesh(w.mesh.source[0])
    pm = Photonmap(64, 64)
    pm.add_mesh(inst)
    for l in w.scene.lights:
        sc.add_light(l)
    sc.end()
    st = scenes.IndirectLightSettings(1, 3, 0.05, 20.0, 8, 20.0, 7)
    rl = _relight()
    rl.emit_photons(sc, st, seed=8)
    g = _lumels(pm)
    orc = Oracle(sc.flat).bind_scene(sc)
    opm = orc.maps("photonmap")[0]
    stored = orc.emit_photons([opm], 1, 3, 0.05, 20.0, 8)
    assert stored > 1000
    assert np.array_equal(g["photons"], opm.photons)
    np.testing.assert_allclose(g["color"], opm.color, rtol=1e-5, atol=1e-6)
    # textured albedo: deposits on the boxes are not grey
    c = g["color"][g["photons"] > 0]
    assert np.abs(c[:, 0] - c[:, 1]).max() > 1e-3


def test_direct_light_iterator_subset(cuda):
    from relight_b200.device import LumelBakeIterator
    w = scenes.room_scene(size=64)
    rl = _relight()
    rl.bake_direct_light(w.scene, w.mesh, None, LumelBakeIterator(3, 7))
    g = _lumels(w.lightmap)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    lm = orc.maps()[0]
    orc.bake_direct(lm, 3, 7)
    assert np.array_equal(g["color"], lm.color)


def test_ambient_occlusion_bit_exact(cuda):
    w = scenes.room_scene(size=96)
    rl = _relight()
    rl.bake_direct_light(w.scene, w.mesh, None)
    rl.bake_ambient_occlusion(w.scene, w.mesh, None, w.ao, seed=77)
    g = _lumels(w.lightmap)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    lm = orc.maps()[0]
    orc.bake_direct(lm)
    orc.bake_ao(lm, w.ao.samples, w.ao.occluded_fraction, w.ao.max_distance, w.ao.exponent, 77)
    assert np.array_equal(g["color"], lm.color)


def _small_terrain():
    return scenes.terrain_scene(verts=64, n_boxes=80, size=128, tiles=2, fg_samples=16, passes=1, bounces=3)


def test_photons_from_room_lights_with_area_light(cuda):
    """Point, spot and area lights all emit from their position."""
    w = scenes.room_scene(size=64)
    pm_scene = w.scene
    rl = _relight()
    # the room has no photonmap: add one over the same mesh through a second scene
    from relight_b200.api import Photonmap, Scene
    sc = Scene()
    sc.begin()
    inst = sc.add_mesh(w.mesh.source[0])
    pm = Photonmap(64, 64)
    pm.add_mesh(inst)
    for l in pm_scene.lights:
        sc.add_light(l)
    sc.end()
    st = scenes.IndirectLightSettings(1, 2, 0.05, 20.0, 8, 20.0, 7)
    rl.emit_photons(sc, st, seed=3)
    g = _lumels(pm)
    orc = Oracle(sc.flat).bind_scene(sc)
    opm = orc.maps("photonmap")[0]
    stored = orc.emit_photons([opm], 1, 2, 0.05, 20.0, 3)
    assert stored > 1000
    assert np.array_equal(g["photons"], opm.photons)
    np.testing.assert_allclose(g["color"], opm.color, rtol=1e-5, atol=1e-6)


def test_photons_and_gather(cuda):
    w = _small_terrain()
    st = w.settings
    rl = _relight()
    rl.emit_photons(w.scene, st, seed=5)
    g = _lumels(w.photonmap)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    pm = orc.maps("photonmap")[0]
    stored = orc.emit_photons([pm], st.photon_pass_count, st.photon_bounce_count, st.photon_energy_threshold,
                              st.photon_max_distance, 5)
    assert stored > 1000
    assert np.array_equal(g["photons"], pm.photons)
    np.testing.assert_allclose(g["color"], pm.color, rtol=1e-5, atol=1e-6)
    orc.gather(pm, st.final_gather_radius)
    np.testing.assert_allclose(g["gathered"], pm.gathered, rtol=1e-4, atol=1e-6)


def test_final_gather_bit_exact_on_fixed_photonmap(cuda):
    w = _small_terrain()
    st = w.settings
    rl = _relight()
    rl.emit_photons(w.scene, st, seed=9)
    g = _lumels(w.photonmap)
    # pin the photonmap: the oracle gathers from the GPU's deposits
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    pm = orc.maps("photonmap")[0]
    pm.gathered[:] = g["gathered"]
    lm = orc.maps("lightmap")[0]
    rl.bake_indirect_light(w.scene, w.meshes[0], None, st, seed=21)
    gl = _lumels(w.lightmap)
    orc.bake_indirect(lm, [pm], st.final_gather_samples, st.final_gather_distance, st.sky_color, st.ambient_color, 21)
    assert (lm.color.sum(1) > 0).sum() > 1000
    assert np.array_equal(gl["color"], lm.color)


def _radiosity_inputs(size=32):
    w = scenes.radiosity_room(size=size)
    rl = _relight()
    rl.device_scene(w.scene)
    g = _lumels(w.radiancemap)
    valid = np.nonzero(g["flags"] & 1)[0]
    return w, rl, valid, g["position"][valid], g["normal"][valid]


def _ff_pairwise_gpu(ds, pos, nrm, threshold):
    import torch
    from relight_b200 import _abi
    n = pos.shape[0]
    dp, dn = _dev(pos, torch), _dev(nrm, torch)
    nnz = C.c_int64()
    _abi.check(_abi.lib().rl_ff_pairwise(ds.handle, n, dp.data_ptr(), dn.data_ptr(), threshold, None, None, None, 0,
                                         C.byref(nnz), None))
    row = np.zeros(n + 1, np.int64); cols = np.zeros(max(nnz.value, 1), np.int32)
    vals = np.zeros(max(nnz.value, 1), np.float32)
    _abi.check(_abi.lib().rl_ff_pairwise(ds.handle, n, dp.data_ptr(), dn.data_ptr(), threshold,
                                         row.ctypes.data, cols.ctypes.data, vals.ctypes.data, nnz.value,
                                         C.byref(nnz), None))
    return row, cols[:nnz.value], vals[:nnz.value]


def test_pairwise_form_factors_bit_exact(cuda):
    w, rl, valid, pos, nrm = _radiosity_inputs(32)
    ds = rl.device_scene(w.scene)
    row, cols, vals = _ff_pairwise_gpu(ds, pos, nrm, 0.1)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    r2, c2, v2 = orc.ff_pairwise(pos, nrm, 0.1)
    assert len(c2) > 100
    assert np.array_equal(row, r2) and np.array_equal(cols, c2) and np.array_equal(vals, v2)


def _patch_tables(w, valid):
    W, H = w.radiancemap.width, w.radiancemap.height
    pot = np.full(W * H, -1, np.int32)
    pot[valid] = np.arange(len(valid), dtype=np.int32)
    return (np.array([0], np.int32), np.array([[W, H]], np.int32), np.array([0], np.int64), pot)


def _ff_hemi_gpu(ds, pos, nrm, rays, maxd, seed, tabs):
    import torch
    from relight_b200 import _abi
    mesh_map, dims, base, pot = tabs
    n = pos.shape[0]
    dp, dn = _dev(pos, torch), _dev(nrm, torch)
    nnz = C.c_int64()
    args = (mesh_map.ctypes.data, len(dims), dims.ctypes.data, base.ctypes.data, pot.ctypes.data, pot.size)
    _abi.check(_abi.lib().rl_ff_hemisphere(ds.handle, n, dp.data_ptr(), dn.data_ptr(), rays, maxd, seed, *args,
                                           None, None, None, 0, C.byref(nnz), None))
    row = np.zeros(n + 1, np.int64); cols = np.zeros(max(nnz.value, 1), np.int32)
    vals = np.zeros(max(nnz.value, 1), np.float32)
    _abi.check(_abi.lib().rl_ff_hemisphere(ds.handle, n, dp.data_ptr(), dn.data_ptr(), rays, maxd, seed, *args,
                                           row.ctypes.data, cols.ctypes.data, vals.ctypes.data, nnz.value,
                                           C.byref(nnz), None))
    return row, cols[:nnz.value], vals[:nnz.value]


def test_hemisphere_form_factors_bit_exact(cuda):
    w, rl, valid, pos, nrm = _radiosity_inputs(32)
    ds = rl.device_scene(w.scene)
    tabs = _patch_tables(w, valid)
    row, cols, vals = _ff_hemi_gpu(ds, pos, nrm, 128, 100.0, 3, tabs)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    r2, c2, v2 = orc.ff_hemisphere(pos, nrm, 128, 100.0, 3, *tabs)
    assert len(c2) > 1000
    assert np.array_equal(row, r2) and np.array_equal(cols, c2) and np.array_equal(vals, v2)


def test_hemisphere_form_factors_device_output(cuda):
    """rl_ff_hemisphere_device leaves the same CSR in device memory that
    rl_ff_hemisphere copies to the host, and reports nnz alone without d_cols."""
    import torch
    from relight_b200 import _abi
    w, rl, valid, pos, nrm = _radiosity_inputs(32)
    ds = rl.device_scene(w.scene)
    tabs = _patch_tables(w, valid)
    row, cols, vals = _ff_hemi_gpu(ds, pos, nrm, 64, 100.0, 9, tabs)
    mesh_map, dims, base, pot = tabs
    n = pos.shape[0]
    dp, dn = _dev(pos, torch), _dev(nrm, torch)
    args = (mesh_map.ctypes.data, len(dims), dims.ctypes.data, base.ctypes.data, pot.ctypes.data, pot.size)
    nnz = C.c_int64()
    _abi.check(_abi.lib().rl_ff_hemisphere_device(ds.handle, n, dp.data_ptr(), dn.data_ptr(), 64, 100.0, 9, *args,
                                                  None, None, None, 0, C.byref(nnz), None))
    assert nnz.value == len(cols)
    cap = n * 64
    drow = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    dcols = torch.zeros(cap, dtype=torch.int32, device="cuda")
    dvals = torch.zeros(cap, dtype=torch.float32, device="cuda")
    _abi.check(_abi.lib().rl_ff_hemisphere_device(ds.handle, n, dp.data_ptr(), dn.data_ptr(), 64, 100.0, 9, *args,
                                                  drow.data_ptr(), dcols.data_ptr(), dvals.data_ptr(), cap,
                                                  C.byref(nnz), None))
    torch.cuda.synchronize()
    k = nnz.value
    assert np.array_equal(drow.cpu().numpy(), row)
    assert np.array_equal(dcols[:k].cpu().numpy(), cols)
    assert np.array_equal(dvals[:k].cpu().numpy().view(np.uint32), vals.view(np.uint32))
    rc = _abi.lib().rl_ff_hemisphere_device(ds.handle, n, dp.data_ptr(), dn.data_ptr(), 64, 100.0, 9, *args,
                                            drow.data_ptr(), dcols.data_ptr(), dvals.data_ptr(), k - 1,
                                            C.byref(nnz), None)
    assert rc == _abi.RL_CAPACITY and nnz.value == k


def test_radiosity_jacobi_vs_fp64(cuda):
    import torch
    from relight_b200 import _abi
    w, rl, valid, pos, nrm = _radiosity_inputs(32)
    ds = rl.device_scene(w.scene)
    tabs = _patch_tables(w, valid)
    row, cols, vals = _ff_hemi_gpu(ds, pos, nrm, 256, 100.0, 4, tabs)
    n = len(row) - 1
    rng = np.random.default_rng(5)
    rho = rng.uniform(0.3, 0.9, (n, 3)).astype(np.float32)
    E = np.zeros((n, 3), np.float32)
    E[rng.choice(n, 16, replace=False)] = 1.0
    B = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    dr, dc, dv, dE, drho = (_dev(x, torch) for x in (row, cols, vals, E, rho))
    _abi.check(_abi.lib().rl_radiosity_solve(n, dr.data_ptr(), dc.data_ptr(), dv.data_ptr(), dE.data_ptr(),
                                             drho.data_ptr(), 50, B.data_ptr(), None))
    torch.cuda.synchronize()
    ref = jacobi_f64(row, cols, vals, E, rho, 50)
    np.testing.assert_allclose(B.cpu().numpy(), ref, rtol=1e-4, atol=1e-6)
    # columns and weights 4 bytes past a 16-byte boundary: the scalar-load path
    dc1 = _dev(np.concatenate([[0], cols]).astype(np.int32), torch)
    dv1 = _dev(np.concatenate([[0], vals]).astype(np.float32), torch)
    B1 = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    _abi.check(_abi.lib().rl_radiosity_solve(n, dr.data_ptr(), dc1.data_ptr() + 4, dv1.data_ptr() + 4, dE.data_ptr(),
                                             drho.data_ptr(), 50, B1.data_ptr(), None))
    torch.cuda.synchronize()
    np.testing.assert_allclose(B1.cpu().numpy(), ref, rtol=1e-4, atol=1e-6)


def test_radiosity_solve_large_aligned_and_not(cuda):
    """24,000 patches with 40 nonzeros a row: the solve's 16-byte column and
    weight loads (aligned arrays) and its 4-byte loads (arrays 4 bytes off a
    16-byte boundary), both within the fp32 tolerance of FP64 Jacobi."""
    import torch
    from relight_b200 import _abi
    n, per_row = 24000, 40
    rng = np.random.default_rng(21)
    cols = np.sort(rng.integers(0, n, (n, per_row)), axis=1).astype(np.int32).reshape(-1)
    vals = rng.random((n, per_row)).astype(np.float32)
    vals = (vals * (np.float32(0.9) / vals.sum(1, keepdims=True, dtype=np.float32))).astype(np.float32).reshape(-1)
    row = np.arange(n + 1, dtype=np.int64) * per_row
    rho = rng.uniform(0.3, 0.9, (n, 3)).astype(np.float32)
    E = np.zeros((n, 3), np.float32)
    E[rng.choice(n, 64, replace=False)] = 1.0
    ref = jacobi_f64(row, cols, vals, E, rho, 30)
    dr, dE, drho = (_dev(x, torch) for x in (row, E, rho))
    for off in (0, 1):
        dc = _dev(np.concatenate([np.zeros(off, np.int32), cols]), torch)
        dv = _dev(np.concatenate([np.zeros(off, np.float32), vals]), torch)
        B = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
        _abi.check(_abi.lib().rl_radiosity_solve(n, dr.data_ptr(), dc.data_ptr() + 4 * off, dv.data_ptr() + 4 * off,
                                                 dE.data_ptr(), drho.data_ptr(), 30, B.data_ptr(), None))
        torch.cuda.synchronize()
        np.testing.assert_allclose(B.cpu().numpy(), ref, rtol=1e-4, atol=1e-6)


def test_launch_tuning_changes_no_result(cuda):
    """The autotuner's knobs (refill threshold, block size, BVH width 2 / 4 /
    compressed 8, speculative walk, the final gather's persistent lumel pool
    and its chunk) reschedule rays only: every setting bakes the same bits."""
    from relight_b200 import autotune
    saved = (autotune.get("ao"), autotune.get("indirect"), autotune.get_width(), autotune.get_speculative(),
             autotune.get_pool())
    colors, fg = [], []
    try:
        for refill, block, width, spec, pool in ((1, 64, 2, 0, (0, 32)), (13, 128, 4, 0, (0, 32)),
                                                 (32, 256, 2, 1, (0, 32)), (24, 64, 2, 1, (0, 32)),
                                                 (16, 64, 8, 0, (0, 32)), (32, 128, 8, 0, (0, 32)),
                                                 (24, 256, 2, 0, (1, 32)), (1, 64, 2, 0, (1, 8)),
                                                 (32, 128, 2, 0, (1, 256)), (20, 256, 2, 0, (1, 64))):
            autotune.set_width(width)
            autotune.set_speculative(spec)
            autotune.set_pool(*pool)
            autotune.set(refill, block, "ao")
            autotune.set(refill, block, "indirect")
            rl = _relight()
            ws = scenes.room_scene(size=64)
            rl.bake_ambient_occlusion(ws.scene, ws.mesh, None, ws.ao, seed=3)
            colors.append(_lumels(ws.lightmap)["color"])
            wt = _small_terrain()
            rl.emit_photons(wt.scene, wt.settings, seed=2)
            rl.bake_indirect_light(wt.scene, wt.meshes[0], None, wt.settings, seed=4)
            fg.append(_lumels(wt.lightmap)["color"])
    finally:
        autotune.set(saved[0]["refill"], saved[0]["block"], "ao")
        autotune.set(saved[1]["refill"], saved[1]["block"], "indirect")
        autotune.set_width(saved[2])
        autotune.set_speculative(saved[3])
        autotune.set_pool(*saved[4])
    assert all(np.array_equal(colors[0], c) for c in colors[1:])
    # photon deposits are atomic float sums, so the final gather is compared
    # through the photonmap's tolerance
    for c in fg[1:]:
        np.testing.assert_allclose(c, fg[0], rtol=1e-4, atol=1e-6)


def test_ao_split_changes_no_result(cuda):
    """Lanes sharing one lumel's AO samples (RL_TUNE_AO_SPLIT 1, 2, 4, 8 and
    the size-based default) add integer occlusion counts: every setting bakes
    the same bits, for a whole-map bake and for a LumelBakeIterator(1, 3) slice."""
    import ctypes as C
    from relight_b200 import _abi
    from relight_b200.device import LumelBakeIterator
    L = _abi.lib()
    old = C.c_int()
    _abi.check(L.rl_tune_get(_abi.TUNE_AO_SPLIT, C.byref(old)))
    out = []
    try:
        for split in (1, 2, 4, 8, 0):
            _abi.check(L.rl_tune_set(_abi.TUNE_AO_SPLIT, split))
            got = []
            for it in (None, LumelBakeIterator(1, 3)):
                rl = _relight()
                ws = scenes.room_scene(size=64)
                rl.bake_direct_light(ws.scene, ws.mesh, None)  # AO scales the colour already there
                rl.bake_ambient_occlusion(ws.scene, ws.mesh, None, ws.ao, iterator=it, seed=5)
                got.append(_lumels(ws.lightmap)["color"])
            out.append(got)
    finally:
        _abi.check(L.rl_tune_set(_abi.TUNE_AO_SPLIT, old.value))
    assert (out[0][0].sum(1) > 0).sum() > 1000
    for got in out[1:]:
        for a, b in zip(out[0], got):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_photon_shares_sum_to_the_full_emission(cuda):
    """rl_emit_photons_range: two shares of the photon sequence, deposited into
    two photonmap replicas, sum to the unsplit emission (the multi-GPU split)."""
    import ctypes as C
    from relight_b200 import _abi, parallel
    from relight_b200.device import DeviceMap, _map_array
    w = _small_terrain()
    st, f = w.settings, w.scene.flat
    rl = _relight()
    ds = rl.device_scene(w.scene)
    L = _abi.lib()
    lights = C.c_void_p(f.lights.ctypes.data)
    total = C.c_int64()
    _abi.check(L.rl_photon_count(lights, len(f.lights), st.photon_pass_count, C.byref(total)))
    assert total.value == st.photon_pass_count * 5 * 25000
    reps = []
    for k in range(3):
        m = DeviceMap(1, w.photonmap.width, w.photonmap.height)
        for mesh in w.photonmap.meshes:
            m.add_mesh(ds, w.scene.meshes.index(mesh))
        reps.append(m)
    args = (st.photon_pass_count, st.photon_bounce_count, st.photon_energy_threshold, st.photon_max_distance, 8)
    for k, m in enumerate(reps[:2]):
        first, count = parallel.photon_share(total.value, k, 2)
        _abi.check(L.rl_emit_photons_range(ds.handle, _map_array([m]), 1, lights, len(f.lights), *args, first, count,
                                           None, None))
    _abi.check(L.rl_emit_photons(ds.handle, _map_array([reps[2]]), 1, lights, len(f.lights), *args, None, None))
    a, b, full = (m.download() for m in reps)
    assert full["photons"].sum() > 1000
    assert np.array_equal(a["photons"] + b["photons"], full["photons"])
    np.testing.assert_allclose(a["color"] + b["color"], full["color"], rtol=1e-5, atol=1e-6)


def test_distributed_bake_on_one_rank_matches(cuda):
    """The split bake's CUDA engine under NCCL with one rank (the only
    multi-GPU path a one-GPU box can run): the photon split equals the
    unsplit emission (counts exact, the gather within the atomics'
    tolerance); the final-gather split and the row-sharded radiosity solve
    give the single-GPU bake's bits."""
    import os
    import socket
    import torch
    import torch.distributed as dist
    from relight_b200 import _abi, parallel
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        w1, w2 = _small_terrain(), _small_terrain()
        rl = _relight()
        parallel.emit_photons_distributed(rl, w1.scene, w1.settings, seed=4)
        rl.emit_photons(w2.scene, w2.settings, seed=4)
        a, b = _lumels(w1.photonmap), _lumels(w2.photonmap)
        assert np.array_equal(a["photons"], b["photons"])
        np.testing.assert_allclose(a["gathered"], b["gathered"], rtol=1e-4, atol=1e-6)
        # final gather: the same photonmap and base colours, split and unsplit
        rl.bake_direct_light(w1.scene, w1.meshes[0], None)
        base = _lumels(w1.lightmap)["color"].copy()
        rl.bake_indirect_light(w1.scene, w1.meshes[0], None, w1.settings, seed=9)
        want = _lumels(w1.lightmap)["color"].copy()
        w1.lightmap._device.upload(color=base)
        parallel.bake_indirect_distributed(rl, w1.scene, w1.meshes[0], w1.settings, seed=9)
        got = _lumels(w1.lightmap)["color"]
        assert (want != base).any()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        # radiosity: rows sharded over one rank == rl_radiosity_solve
        n, per = 5000, 24
        rng = np.random.default_rng(8)
        cols = np.sort(rng.integers(0, n, (n, per)), axis=1).astype(np.int32).reshape(-1)
        vals = rng.random(n * per).astype(np.float32) * np.float32(0.9 / per)
        row = np.arange(n + 1, dtype=np.int64) * per
        rho = rng.uniform(0.3, 0.9, (n, 3)).astype(np.float32)
        E = np.zeros((n, 3), np.float32)
        E[rng.choice(n, 16, replace=False)] = 1.0
        dr, dc, dv, dE, drho = (_dev(x, torch) for x in (row, cols, vals, E, rho))
        want = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
        _abi.check(_abi.lib().rl_radiosity_solve(n, dr.data_ptr(), dc.data_ptr(), dv.data_ptr(), dE.data_ptr(),
                                                 drho.data_ptr(), 50, want.data_ptr(), None))
        got = torch.zeros_like(want)
        parallel.radiosity_solve_distributed(rl, n, dr, dc, dv, dE, drho, 50, got)
        torch.cuda.synchronize()
        assert torch.equal(got.view(torch.int32), want.view(torch.int32))
    finally:
        dist.destroy_process_group()


def test_face_iterator_bakes_match_oracle(cuda):
    """FaceBakeIterator(first, step) per mesh of a shared lightmap, for the
    direct, AO and final-gather bakes."""
    from relight_b200.device import FaceBakeIterator
    w = _small_terrain()
    st = w.settings
    rl = _relight()
    rl.emit_photons(w.scene, st, seed=6)
    g = _lumels(w.photonmap)
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    pm = orc.maps("photonmap")[0]
    pm.gathered[:] = g["gathered"]
    lm = orc.maps()[0]
    for k, mesh in enumerate(w.meshes):
        it = FaceBakeIterator(k % 3, 3)
        mi = w.scene.meshes.index(mesh)
        rl.bake_direct_light(w.scene, mesh, None, it)
        orc.bake_direct(lm, k % 3, 3, mesh=mi)
        rl.bake_ambient_occlusion(w.scene, mesh, None, scenes.AmbientOcclusionSettings(8, 0.8, 2.0, 1.0), it, seed=k)
        orc.bake_ao(lm, 8, 0.8, 2.0, 1.0, k, k % 3, 3, mesh=mi)
        rl.bake_indirect_light(w.scene, mesh, None, st, it, seed=100 + k)
        orc.bake_indirect(lm, [pm], st.final_gather_samples, st.final_gather_distance, st.sky_color,
                          st.ambient_color, 100 + k, k % 3, 3, mesh=mi)
    gl = _lumels(w.lightmap)
    assert (lm.color.sum(1) > 0).sum() > 500
    assert np.array_equal(gl["color"], lm.color)


def test_device_lbvh_bakes_what_the_sah_tree_bakes(cuda):
    """The device LBVH and the host SAH tree give bit-identical bakes (hits do
    not depend on the tree), on the full terrain's geometry."""
    colors = []
    for builder in (0, 1):
        w = scenes.terrain_scene(size=256, fg_samples=8, passes=1)
        rl = _relight(builder)
        rl.bake_direct_light(w.scene, w.meshes[0], None)
        rl.bake_ambient_occlusion(w.scene, w.meshes[0], None, scenes.AmbientOcclusionSettings(8, 0.8, 2.0, 1.0),
                                  seed=2)
        colors.append(_lumels(w.lightmap)["color"])
        stats = w.scene._device.bvh_stats()
        assert stats["nodes"] > 30000 and stats["depth"] < 63
    assert (colors[0].sum(1) > 0).sum() > 10000
    assert np.array_equal(colors[0], colors[1])
