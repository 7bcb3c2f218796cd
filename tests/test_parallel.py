"""The multi-GPU split of one bake (relight_b200/parallel.py), run as two gloo
ranks on CPU with the oracle as the compute engine, through the same
*_distributed functions the CUDA engine runs under NCCL: photon shares
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


class OracleEngine:
    """relight_b200.parallel's engine interface over the oracle (CPU):
    torch tensors that share the oracle's numpy lumel arrays."""

    def __init__(self, scene):
        from oracle_bind import Oracle
        self.orc = Oracle(scene.flat).bind_scene(scene)
        self.lms = dict(zip(map(id, scene.flat.lightmaps), self.orc.maps()))
        self.pms = dict(zip(map(id, scene.flat.photonmaps), self.orc.maps("photonmap")))

    def photon_total(self, scene, st):
        return int(sum(int(l["intensity"] * 25000) for l in scene.flat.lights if l["emitter"])) * st.photon_pass_count

    def emit_photon_range(self, scene, st, seed, first, count):
        self.orc.emit_photons_range(list(self.pms.values()), st.photon_pass_count, st.photon_bounce_count,
                                    st.photon_energy_threshold, st.photon_max_distance, seed, first, count)

    def photon_accumulators(self, scene):
        pms = list(self.pms.values())
        return [torch.from_numpy(p.color) for p in pms] + [torch.from_numpy(p.photons) for p in pms]

    def gather_photons(self, scene, st):
        for p in self.pms.values():
            self.orc.gather(p, st.final_gather_radius)

    def color_tensor(self, lightmap):
        return torch.from_numpy(self.lms[id(lightmap)].color)

    def bake_indirect_light(self, scene, mesh, progress, st, iterator, seed):
        self.orc.bake_indirect(self.lms[id(mesh.lightmap)], list(self.pms.values()), st.final_gather_samples,
                               st.final_gather_distance, st.sky_color, st.ambient_color, seed, iterator.first,
                               iterator.step)

    def radiosity_step(self, r0, r1, row, cols, vals, E, rho, B, B_next):
        x = B.numpy().astype(np.float64)
        r, c, v = row.numpy(), cols.numpy(), vals.numpy().astype(np.float64)
        for i in range(r0, r1):
            s = (v[r[i]:r[i + 1], None] * x[c[r[i]:r[i + 1]]]).sum(0)
            B_next[i] = torch.from_numpy((E[i].numpy() + rho[i].numpy() * s).astype(np.float32))


def _worker(rank, world, port, outdir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = _scene()
        st = w.settings
        eng = OracleEngine(w.scene)
        parallel.emit_photons_distributed(eng, w.scene, st, 7)
        pm = eng.pms[id(w.photonmap)]
        lm = eng.lms[id(w.lightmap)]
        lm.color[:] = 0.25
        parallel.bake_indirect_distributed(eng, w.scene, w.meshes[0], st, 13)
        row, cols, vals, E, rho = (torch.from_numpy(a) for a in _csr(300, 3))
        B = torch.zeros((300, 3), dtype=torch.float32)
        parallel.radiosity_solve_distributed(eng, 300, row, cols, vals, E, rho, 20, B)
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), photons=pm.photons, color=pm.color, gathered=pm.gathered,
                 fg=lm.color, B=B.numpy())
    finally:
        dist.destroy_process_group()


def test_photon_share_partition():
    for total in (0, 1, 7, 1000001):
        for world in (1, 2, 3, 8):
            shares = [parallel.photon_share(total, r, world) for r in range(world)]
            assert shares[0][0] == 0
            assert all(a[0] + a[1] == b[0] for a, b in zip(shares, shares[1:]))
            assert sum(c for _, c in shares) == total


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_reproduce_the_unsplit_bake(world):
    from oracle_bind import Oracle, jacobi_f64
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, _free_port(), d), nprocs=world, join=True, start_method="spawn")
        r = [np.load(os.path.join(d, f"rank{k}.npz")) for k in range(world)]
    for k in range(1, world):
        for f in ("photons", "color", "gathered", "fg", "B"):
            assert np.array_equal(r[0][f], r[k][f]), f
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
