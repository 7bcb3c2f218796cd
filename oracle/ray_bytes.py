"""Per-ray algorithmic byte model of the traversal roofline, measured on the
canonical binary SAH BVH (the oracle tracer, ort.c):

    B_ray = 48 B ray I/O + 32 B x N_box + 48 B x N_tri

N_box = child-box tests and N_tri = triangle tests per ray, counted by the
instrumented CPU traversal over a seeded sample of each workload's rays.
Test infrastructure: run offline, the printed figures are frozen into
bench.py (RAY_MODEL) and the design notes.

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
    for k, v in out.items():
        print(k, v)


if __name__ == "__main__":
    main()
