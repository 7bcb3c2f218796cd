"""Generate the golden fixtures under tests/golden/ by running the reference
baker compiled from its own sources (oracle/_ref/librelight_ref.so, built by
`make -C oracle ref` where the reference sources are present).

    python tests/golden/make_golden.py

Every fixture is a deterministic output of the reference's code:
  room64.npz        Lightmap::addMesh lumels + Relight::bakeDirectLight
                    colours on a 64x64 room (point, spot, area lights), the
                    scene's transformed vertices and area-light samples.
  trace_room.npz    rt::Embree::traceSegment results for 4,000 seeded segments
                    (hit, point, normal, rgba, lightmap uv, mesh) with HitAll.
  gather.npz        Photonmap::gather(7) over seeded photon accumulators on
                    square and non-square maps.
  ff_room24.npz     RadiosityBuilder::build(0.1) on a 24x24-texel
                    radiancemap room: form-factor CSR and patch positions.
The inputs are rebuilt from relight_b200.scenes with the same seeds.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))

from oracle_bind import LumelMap, RefScene, ptr  # noqa: E402
from relight_b200 import scenes  # noqa: E402


def segments(flat, n, seed):
    rng = np.random.default_rng(seed)
    a = rng.uniform(flat.bounds_lo - 1, flat.bounds_hi + 1, (n, 3))
    b = rng.uniform(flat.bounds_lo - 1, flat.bounds_hi + 1, (n, 3))
    return np.concatenate([a, b], 1).astype(np.float32)


def gather_inputs(W, H, seed):
    rng = np.random.default_rng(seed)
    color = rng.random((W * H, 3)).astype(np.float32)
    photons = rng.integers(0, 5, W * H).astype(np.int32)
    photons[rng.random(W * H) < 0.3] = 0
    color[photons == 0] = 0
    return color, photons


def main():
    out = {}
    # room, direct light
    w = scenes.room_scene(size=64)
    ref = RefScene(w.scene)
    pos, nrm = ref.mesh_vertices(w.mesh)
    lv = [ref.light_vertices(i) for i, l in enumerate(w.scene.lights) if l.vertices is not None]
    ref.lib.ref_bake_direct(ref.h, ref.mesh(w.mesh), 0, 0, 1)
    lm = ref.lumels(w.lightmap)
    np.savez_compressed(os.path.join(HERE, "room64.npz"), flags=lm.flags, face=lm.face, position=lm.position,
                        normal=lm.normal, color=lm.color, mesh_pos=pos, mesh_nrm=nrm, light_vertices=lv[0])
    out["room64"] = int((lm.flags & 1).sum())
    # traceSegment
    w = scenes.room_scene(size=64)
    ref = RefScene(w.scene)
    seg = segments(w.scene.flat, 4000, 7)
    r = ref.trace_segments(seg, 15)
    np.savez_compressed(os.path.join(HERE, "trace_room.npz"), seg=seg, **r)
    out["trace_room"] = int(r["hit"].sum())
    # Photonmap::gather
    g = {}
    for (W, H) in ((48, 48), (56, 40), (40, 56)):
        color, photons = gather_inputs(W, H, W * 100 + H)
        k = ref.lib.ref_create_map(ref.h, 1, W, H)
        ref.lib.ref_map_set_photons(ref.h, k, ptr(color), ptr(photons))
        ref.lib.ref_photonmap_gather(ref.h, k, 7)
        m = LumelMap(W, H)
        ref.lib.ref_map_lumels(ref.h, k, None, None, None, None, None, None, ptr(m.gathered))
        g[f"gathered_{W}x{H}"] = m.gathered
    np.savez_compressed(os.path.join(HERE, "gather.npz"), **g)
    # RadiosityBuilder
    w = scenes.radiosity_room(size=24)
    ref = RefScene(w.scene, radiancemaps=(w.radiancemap,))
    row, cols, vals, ppos, pnrm = ref.radiosity(0.1)
    np.savez_compressed(os.path.join(HERE, "ff_room24.npz"), row=row, cols=cols, vals=vals, pos=ppos, nrm=pnrm)
    out["ff_room24"] = int(len(cols))
    print(out)


if __name__ == "__main__":
    main()
