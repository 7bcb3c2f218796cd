"""The reference's own bakers over the GPU: Relight compiled from its own
sources with its Embree 2 calls answered by the B200 library
(oracle/embree2_gpu.cpp over rl_intersect_rays_host; oracle/_ref/
librelight_ref_gpu.so) against the same sources over the CPU stand-in for
Embree (oracle/embree2_cpu.cpp).  rt::Embree::traceSegment, its hit
post-processing and HitUseAlpha loop, and every baker above it run
unchanged in both; only where the ray queries run differs.  Bit for bit:
traceSegment on seeded segments, Relight::bakeDirectLight, and
Relight::bakeAmbientOcclusion with the same per-thread rand() seed.

Also rl_intersect_rays on device arrays against the oracle tracer.
"""
import os

import numpy as np
import pytest

import oracle_bind as ob
from relight_b200 import scenes

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (os.path.exists(ob.REF_GPU_LIB) and os.path.exists(ob.REF_LIB)),
                                 reason="reference builds (oracle/_ref) not present")]


def _segments(flat, n, seed):
    rng = np.random.default_rng(seed)
    a = rng.uniform(flat.bounds_lo - 1, flat.bounds_hi + 1, (n, 3))
    b = rng.uniform(flat.bounds_lo - 1, flat.bounds_hi + 1, (n, 3))
    return np.concatenate([a, b], 1).astype(np.float32)


@pytest.mark.parametrize("which", ["room", "textured", "terrain"])
def test_reference_bakers_over_gpu_embree_match_cpu_embree(cuda, which):
    if which == "terrain":
        w = scenes.terrain_scene(verts=24, n_boxes=20, size=48, tiles=2)
        mesh, lmap = w.meshes[0], w.lightmap
    else:
        w = scenes.room_scene(size=48, textured=which == "textured")
        mesh, lmap = w.mesh, w.lightmap
    cpu = ob.RefScene(w.scene)
    gpu = ob.RefScene(w.scene, fast="gpu")
    seg = _segments(w.scene.flat, 3000, 5)
    for flags in (15, 31):
        a, b = cpu.trace_segments(seg, flags), gpu.trace_segments(seg, flags)
        assert np.array_equal(a["hit"], b["hit"])
        m = a["hit"] > 0
        assert m.sum() > 500
        for f in ("point", "normal", "rgba", "uv", "mesh"):
            assert np.array_equal(a[f][m], b[f][m]), (flags, f)
    for ref in (cpu, gpu):
        ref.lib.ref_bake_direct(ref.h, ref.mesh(mesh), 0, 0, 1)
    ca, ga = cpu.lumels(lmap), gpu.lumels(lmap)
    assert (ca.color.sum(1) > 0).sum() > 300
    assert np.array_equal(ca.color.view(np.uint32), ga.color.view(np.uint32))
    for ref in (cpu, gpu):
        ref.lib.ref_set_rand(0, 21)
        ref.lib.ref_bake_ao(ref.h, ref.mesh(mesh), 16, 0.8, 2.0, 1.0, 0, 0, 1)
    ca, ga = cpu.lumels(lmap), gpu.lumels(lmap)
    assert np.array_equal(ca.color.view(np.uint32), ga.color.view(np.uint32))


def test_intersect_rays_match_the_oracle_tracer(cuda):
    """rl_intersect_rays (closest and any hit, device arrays) on Embree-style
    rays: the same (geomID, primID, t, u, v) as the oracle's segments give."""
    import torch
    from oracle_bind import Oracle
    from relight_b200 import _abi
    from relight_b200.device import Relight
    w = scenes.terrain_scene(verts=40, n_boxes=50, size=64, tiles=2)
    ds = Relight().device_scene(w.scene)
    seg = _segments(w.scene.flat, 20000, 9)
    d = (seg[:, 3:] - seg[:, :3]).astype(np.float32)
    length = np.sqrt((d * d).sum(1, dtype=np.float32)).astype(np.float32)
    d = (d / length[:, None]).astype(np.float32)
    rays = np.zeros((len(seg), 8), np.float32)
    rays[:, :3], rays[:, 3], rays[:, 4:7], rays[:, 7] = seg[:, :3], 0.01, d, length
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    # the oracle's segment trace builds the same ray (initializeRay) from the
    # segment's start and end
    ref = orc.trace_segments(seg, 15)
    dr = torch.from_numpy(rays).cuda()
    gp = torch.zeros((len(seg), 2), dtype=torch.int32, device="cuda")
    tuv = torch.zeros((len(seg), 3), dtype=torch.float32, device="cuda")
    for any_hit in (0, 1):
        _abi.check(_abi.lib().rl_intersect_rays(ds.handle, len(seg), dr.data_ptr(), any_hit, gp.data_ptr(),
                                                tuv.data_ptr(), None))
        torch.cuda.synchronize()
        g = gp.cpu().numpy()
        assert np.array_equal(g[:, 0] >= 0, ref["hit"] > 0)
        if not any_hit:
            m = ref["hit"] > 0
            assert m.sum() > 1000
            assert np.array_equal(g[m, 0], ref["mesh"][m]) and np.array_equal(g[m, 1], ref["face"][m])
            t = tuv.cpu().numpy()[m, 0]
            pt = seg[m, :3] + d[m] * t[:, None]
            assert np.array_equal(pt.astype(np.float32), ref["point"][m])
    # host-array variant, from a second thread too
    import threading
    out = {}

    def run(k):
        g2 = np.zeros((len(seg), 2), np.int32)
        t2 = np.zeros((len(seg), 3), np.float32)
        _abi.check(_abi.lib().rl_intersect_rays_host(ds.handle, len(seg), rays.ctypes.data, 0, g2.ctypes.data,
                                                     t2.ctypes.data))
        out[k] = (g2, t2)

    th = [threading.Thread(target=run, args=(k,)) for k in range(2)]
    for t_ in th:
        t_.start()
    for t_ in th:
        t_.join()
    _abi.check(_abi.lib().rl_intersect_rays(ds.handle, len(seg), dr.data_ptr(), 0, gp.data_ptr(), tuv.data_ptr(),
                                            None))
    torch.cuda.synchronize()
    for k in range(2):
        assert np.array_equal(out[k][0], gp.cpu().numpy())
        assert np.array_equal(out[k][1].view(np.uint32), tuv.cpu().numpy().view(np.uint32))
