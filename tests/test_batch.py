"""Batched bakes (rl_batch_*): many jobs over uneven scenes and lightmap
sizes in one persistent launch per pass kind, and its CUDA-graph replay.

The bar is bit-identity with the plain per-job loop (rl_bake_direct /
rl_bake_ao / rl_bake_indirect one job at a time), which the parity tests
pin to the oracle.  Both runs share one resident set (scenes, BVHs and
gathered photonmaps), so the final-gather inputs are the same bits.
"""
import ctypes as C

import numpy as np
import pytest

from relight_b200 import scenes


def _small_workload(n_jobs=10):
    return scenes.batch_workload(n_jobs=n_jobs, n_scenes=3, seed=11, tris=(1_000, 20_000), sides=(24, 96),
                                 ao_samples=8, fg_samples=16, photon_map=64)


def _colors(res):
    return [m.download(fields=("color",))["color"].copy() for m in res.lightmaps]


@pytest.mark.gpu
@pytest.mark.parametrize("pool", [1, 0])
def test_batch_matches_per_job_loop(cuda, pool):
    """pool: the AO and final-gather batch kernels with per-warp lumel pools
    (k_batch_pool, the default) or one lumel per lane per chunk (k_batch);
    the per-job loop runs with the same setting."""
    import torch
    from relight_b200 import autotune, batch
    saved = autotune.get_pool()
    autotune.set_pool(pool)
    try:
        res = batch.make_resident(_small_workload())
        batch.run_per_job(res.jobs)
        torch.cuda.synchronize()
        want = _colors(res)
        assert any(np.abs(w).sum() > 0 for w in want)
        res.clear()
        b = batch.Batch(res.jobs)
    finally:
        autotune.set_pool(*saved)
    assert b.work_items == 3 * sum(m.width * m.height for m in res.lightmaps)
    b.launch()
    torch.cuda.synchronize()
    got = _colors(res)
    for q, (w, g) in enumerate(zip(want, got)):
        assert np.array_equal(w.view(np.uint32), g.view(np.uint32)), f"lightmap {q}"
    b.close()


@pytest.mark.gpu
def test_batch_graph_replay_repeats(cuda):
    import torch
    from relight_b200 import batch
    res = batch.make_resident(_small_workload(6))
    b = batch.Batch(res.jobs)
    b.launch()
    torch.cuda.synchronize()
    want = _colors(res)
    s = torch.cuda.Stream()
    b.capture(s.cuda_stream)
    for _ in range(2):
        res.clear(stream=s.cuda_stream)
        b.replay(s.cuda_stream)
        s.synchronize()
        got = _colors(res)
        for w, g in zip(want, got):
            assert np.array_equal(w.view(np.uint32), g.view(np.uint32))
    b.close()


@pytest.mark.gpu
def test_batch_slices_and_face_jobs(cuda):
    """A job cut into iterator slices, and face-iterator jobs of different
    meshes sharing one lightmap, bake what the whole-map calls bake."""
    import torch
    from relight_b200 import batch
    wl = _small_workload(2)
    res = batch.make_resident(wl)
    j_direct = [j for j in res.jobs if j.kind == batch.DIRECT]
    j_ao = [j for j in res.jobs if j.kind == batch.AO]
    batch.run_per_job(j_direct + j_ao)
    torch.cuda.synchronize()
    want = _colors(res)
    res.clear()
    jobs = []
    for j in j_direct:
        # face iterators, one job per mesh: together they visit every lumel once
        nmesh = len(j.scene.flat.mesh_photonmap)
        for mi in range(nmesh):
            jobs.append(batch.BakeJob(**{**j.__dict__, "iterator": (1, 0, 1, mi)}))
    for j in j_ao:
        n = j.lightmap.width * j.lightmap.height
        cut = n // 3
        jobs.append(batch.BakeJob(**{**j.__dict__, "begin": 0, "end": cut}))
        jobs.append(batch.BakeJob(**{**j.__dict__, "begin": cut, "end": -1}))
    b = batch.Batch(jobs)
    b.launch()
    torch.cuda.synchronize()
    for w, g in zip(want, _colors(res)):
        assert np.array_equal(w.view(np.uint32), g.view(np.uint32))
    b.close()


def test_batch_rejects_overlapping_jobs():
    """Two jobs of one pass over shared lumels of one lightmap would race:
    rl_batch_create refuses them before touching the handles."""
    from relight_b200 import _abi
    from relight_b200._abi import lib
    arr = (_abi.BatchJob * 2)()
    for q in range(2):
        arr[q].kind = 1
        arr[q].scene = 0x1000
        arr[q].lightmap = 0x2000
        arr[q].samples = 8
        arr[q].iterator = _abi.Iterator(0, 0, 1, -1)
        arr[q].begin = 0
        arr[q].end = -1
    h = C.c_void_p()
    rc = lib().rl_batch_create(arr, 2, C.byref(h))
    assert rc == 1 and not h.value  # RL_INVALID_CALL
    assert "shared lumels" in _abi.last_error()
