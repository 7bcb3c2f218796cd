"""Per-ray algorithmic byte model of the traversal roofline, measured on the
canonical binary SAH BVH (the oracle tracer, ort.c):

    B_ray = 48 B ray I/O + 32 B x N_box + 48 B x N_tri

N_box = child-box tests and N_tri = triangle tests per ray, counted by the
instrumented CPU traversal over a seeded sample of each workload's rays.
Test infrastructure: run offline, the printed figures are frozen into
bench.py (RAY_MODEL, ROOM_AO_BYTES_PER_RAY, RAD_*) and the baseline notes.

Ray sets (seeded, 200,000 rays each unless noted):
  terrain_final_gather_closest  final-gather rays of the terrain workload
      (uniform hemisphere at valid lumels, length 50), closest hit;
  room_ao_any                   AO rays of the room workload (length 2),
      first hit (the AO kernel's walk);
  radiosity_pairwise_any        visibility segments of the pairwise form
      factors at 16,384 patches (pairs that pass the cos / threshold cull,
      RadiosityBuilder.cpp:142-176), first hit;
  radiosity_hemisphere_closest  the 512-ray cosine-distributed form-factor
      rays at 16,384 patches (length 100), closest hit.

    python oracle/ray_bytes.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

from oracle_bind import Oracle  # noqa: E402
from relight_b200 import scenes  # noqa: E402


def hemisphere_segments(lm, n, length, seed):
    rng = np.random.default_rng(seed)
    valid = np.nonzero(lm.flags & 1)[0]
    tex = rng.choice(valid, n)
    p = lm.position[tex].astype(np.float64)
    nrm = lm.normal[tex].astype(np.float64)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    flip = (d * nrm).sum(1) < 0
    d[flip] = -d[flip]
    return np.concatenate([p, p + d * length], 1).astype(np.float32)


def model(stats):
    rays, boxes, tris = (float(x) for x in stats)
    nb, nt = boxes / rays, tris / rays
    return {"n_box": round(nb, 2), "n_tri": round(nt, 2), "bytes_per_ray": round(48 + 32 * nb + 48 * nt, 1)}


def cosine_segments(pos, nrm, n, length, seed):
    """Cosine-distributed directions about each sampled patch normal."""
    rng = np.random.default_rng(seed)
    k = rng.integers(0, len(pos), n)
    p = pos[k].astype(np.float64)
    z = nrm[k].astype(np.float64)
    a = np.where(np.abs(z[:, :1]) > 0.9, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    x = np.cross(a, z)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    y = np.cross(z, x)
    u1, u2 = rng.random(n), rng.random(n)
    r, phi = np.sqrt(u1), 2 * np.pi * u2
    d = x * (r * np.cos(phi))[:, None] + y * (r * np.sin(phi))[:, None] + z * np.sqrt(1 - u1)[:, None]
    return np.concatenate([p, p + d * length], 1).astype(np.float32)


def pairwise_segments(pos, nrm, n, threshold, seed):
    """Segments of patch pairs i < j that pass the form-factor cull."""
    rng = np.random.default_rng(seed)
    out = []
    while sum(len(o) for o in out) < n:
        i = rng.integers(0, len(pos), 4 * n)
        j = rng.integers(0, len(pos), 4 * n)
        keep = i < j
        i, j = i[keep], j[keep]
        d = pos[j].astype(np.float64) - pos[i]
        r = np.linalg.norm(d, axis=1)
        ok = r > 0
        d[ok] /= r[ok, None]
        cba = (d * nrm[i]).sum(1)
        cab = -(d * nrm[j]).sum(1)
        w = np.where(ok, cba * cab / (np.pi * np.maximum(r, 1e-30) ** 2), 0.0)
        m = ok & (cba >= 0) & (cab >= 0) & (w >= threshold)
        out.append(np.concatenate([pos[i[m]], pos[j[m]]], 1))
    return np.concatenate(out)[:n].astype(np.float32)


def main():
    out = {}
    w = scenes.terrain_scene()
    orc = Oracle(w.scene.flat).bind_scene(w.scene)
    lm = orc.maps()[0]
    seg = hemisphere_segments(lm, 200000, w.settings.final_gather_distance, 1)
    out["terrain_final_gather_closest"] = model(orc.trace_stats(seg, any_hit=False))
    r = scenes.room_scene()
    orc = Oracle(r.scene.flat).bind_scene(r.scene)
    lm = orc.maps()[0]
    seg = hemisphere_segments(lm, 200000, r.ao.max_distance, 2)
    out["room_ao_any"] = model(orc.trace_stats(seg, any_hit=True))
    rw = scenes.radiosity_room(size=128)
    orc = Oracle(rw.scene.flat).bind_scene(rw.scene)
    rm = orc.maps()[0]
    valid = np.nonzero(rm.flags & 1)[0]
    pos, nrm = rm.position[valid], rm.normal[valid]
    seg = pairwise_segments(pos, nrm, 200000, 0.1, 3)
    out["radiosity_pairwise_any"] = model(orc.trace_stats(seg, any_hit=True))
    seg = cosine_segments(pos, nrm, 200000, 100.0, 4)
    out["radiosity_hemisphere_closest"] = model(orc.trace_stats(seg, any_hit=False))
    for k, v in out.items():
        print(k, v)


if __name__ == "__main__":
    main()
