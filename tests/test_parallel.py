"""The multi-GPU split of one bake (relight_b200/parallel.py), run as two gloo
ranks on CPU with the oracle as the compute engine: photon shares
all-reduced, interleaved final-gather lumels all-reduced, row-sharded
Jacobi all-gathered — each compared with the unsplit single-process result."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from relight_b200 import parallel


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _scene():
    from relight_b200 import scenes
    return scenes.terrain_scene(verts=40, n_boxes=30, size=64, tiles=2, fg_samples=8, passes=2, bounces=2)


def _csr(n, seed):
    rng = np.random.default_rng(seed)
    per = 12
    cols = np.sort(rng.integers(0, n, (n, per)), axis=1).astype(np.int32).reshape(-1)
    vals = rng.random((n, per)).astype(np.float32)
    vals = (vals * (np.float32(0.9) / vals.sum(1, keepdims=True, dtype=np.float32))).reshape(-1)
    row = np.arange(n + 1, dtype=np.int64) * per
    rho = rng.uniform(0.3, 0.9, (n, 3)).astype(np.float32)
    E = np.zeros((n, 3), np.float32)
    E[rng.choice(n, 8, replace=False)] = 1.0
    return row, cols, vals, E, rho


def _worker(rank, world, port, outdir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle_bind import Oracle
        w = _scene()
        st = w.settings
        orc = Oracle(w.scene.flat).bind_scene(w.scene)
        pm = orc.maps("photonmap")[0]
        total = int(sum(int(l["intensity"] * 25000) for l in w.scene.flat.lights if l["emitter"])) * \
            st.photon_pass_count

        def emit_range(first, count):
            orc.emit_photons_range([pm], st.photon_pass_count, st.photon_bounce_count, st.photon_energy_threshold,
                                   st.photon_max_distance, 7, first, count)

        parallel.sharded_photons(emit_range, [torch.from_numpy(pm.color), torch.from_numpy(pm.photons)], total,
                                 rank, world, lambda t: dist.all_reduce(t, op=dist.ReduceOp.SUM))
        orc.gather(pm, st.final_gather_radius)
        lm = orc.maps()[0]
        base = np.full_like(lm.color, 0.25)
        contrib = lm.copy()
        contrib.color[:] = 0

        def bake_subset(first, step):
            orc.bake_indirect(contrib, [pm], st.final_gather_samples, st.final_gather_distance, st.sky_color,
                              st.ambient_color, 13, first, step)

        parallel.sharded_final_gather(bake_subset, torch.from_numpy(contrib.color), base, rank, world,
                                      lambda t: dist.all_reduce(t, op=dist.ReduceOp.SUM),
                                      lambda b, c: np.add(b, c.numpy(), out=b))
        row, cols, vals, E, rho = _csr(300, 3)
        B = torch.from_numpy(E.copy())
        r0, r1 = parallel.row_block(300, rank, world)
        local = torch.zeros((r1 - r0, 3), dtype=torch.float32)

        def step_rows(a, b, Bin, out):
            x = Bin.numpy().astype(np.float64)
            for i in range(a, b):
                s = (vals[row[i]:row[i + 1], None].astype(np.float64) * x[cols[row[i]:row[i + 1]]]).sum(0)
                out[i - a] = torch.from_numpy((E[i] + rho[i] * s).astype(np.float32))

        def all_gather_rows(out, Bfull):
            sizes = [parallel.row_block(300, r, world) for r in range(world)]
            parts = [torch.zeros((q1 - q0, 3), dtype=torch.float32) for q0, q1 in sizes]
            dist.all_gather(parts, out)
            Bfull.copy_(torch.cat(parts))

        parallel.sharded_jacobi(step_rows, B, local, 20, 300, rank, world, all_gather_rows)
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), photons=pm.photons, color=pm.color, gathered=pm.gathered,
                 fg=base, B=B.numpy())
    finally:
        dist.destroy_process_group()


def test_photon_share_partition():
    for total in (0, 1, 7, 1000001):
        for world in (1, 2, 3, 8):
            shares = [parallel.photon_share(total, r, world) for r in range(world)]
            assert shares[0][0] == 0
            assert all(a[0] + a[1] == b[0] for a, b in zip(shares, shares[1:]))
            assert sum(c for _, c in shares) == total


def test_two_gloo_ranks_reproduce_the_unsplit_bake():
    from oracle_bind import Oracle, jacobi_f64
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(2, _free_port(), d), nprocs=2, join=True, start_method="spawn")
        r = [np.load(os.path.join(d, f"rank{k}.npz")) for k in range(2)]
    for f in ("photons", "color", "gathered", "fg", "B"):
        assert np.array_equal(r[0][f], r[1][f]), f
    # unsplit, single process
    w = _scene()
    st = w.settings
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    pm = orc.maps("photonmap")[0]
    orc.emit_photons([pm], st.photon_pass_count, st.photon_bounce_count, st.photon_energy_threshold,
                     st.photon_max_distance, 7)
    assert pm.photons.sum() > 100
    assert np.array_equal(pm.photons, r[0]["photons"])
    np.testing.assert_allclose(pm.color, r[0]["color"], rtol=1e-5, atol=1e-7)
    # final gather from the all-reduced photonmap: bit-identical to one process
    pm.color[:] = r[0]["color"]
    orc.gather(pm, st.final_gather_radius)
    assert np.array_equal(pm.gathered, r[0]["gathered"])
    lm = orc.maps()[0]
    lm.color[:] = 0.25
    orc.bake_indirect(lm, [pm], st.final_gather_samples, st.final_gather_distance, st.sky_color, st.ambient_color, 13)
    assert np.array_equal(lm.color, r[0]["fg"])
    row, cols, vals, E, rho = _csr(300, 3)
    np.testing.assert_allclose(r[0]["B"], jacobi_f64(row, cols, vals, E, rho, 20), rtol=1e-5, atol=1e-7)
