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
  textured_room48.npz  the textured room (RGBA texture with cut-out texels on
                    the boxes, coloured walls) at 48x48: traceSegment with
                    HitAll and with HitAll | HitUseAlpha on 6,000 segments,
                    and Relight::bakeDirectLight colours (alpha shadow rays).
  gather.npz        Photonmap::gather(7) over seeded photon accumulators on
                    square and non-square maps.
  ff_room24.npz     RadiosityBuilder::build(0.1) on a 24x24-texel
                    radiancemap room: form-factor CSR and patch positions.
  obj.npz           Mesh::createFromFile (MeshLoader) on the synthetic OBJ
                    files of obj_texts(): vertices, lightmap uvs, indices.
  post.npz          Lightmap::expand, Lightmap::blur and the files
                    Lightmap::save writes (RawHdr, TgaDoubleLdr, TgaRgbm)
                    for seeded lumel flags and colours (NaN, inf and
                    negative colours included) on four map shapes.
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


def obj_texts():
    """Synthetic OBJ files exercising MeshLoader's rules: submeshes (v / vt /
    vn blocks after faces), quads (first triangle only), shared and -0.0 /
    0.0 vertices, uvs outside [0, 1], octal / hex / signed indices, CRLF
    endings, no final newline, position-only faces."""
    rng = np.random.default_rng(42)
    texts = {}
    # two objects, each with its own v / vt / vn blocks, triangles and quads
    lines = []
    base_v = base_t = base_n = 0
    for obj in range(2):
        nv = 12
        lines.append(f"o part{obj}")
        for _ in range(nv):
            x, y, z = rng.uniform(-3, 3, 3)
            lines.append(f"v {x:.6f} {y:.6f} {z:.6f}")
        for _ in range(nv):
            u, v = rng.uniform(-0.3, 1.3, 2)
            lines.append(f"vt {u:.5f} {v:.5f}")
        for _ in range(4):
            n = rng.normal(size=3)
            n /= np.linalg.norm(n)
            lines.append(f"vn {n[0]:.4f} {n[1]:.4f} {n[2]:.4f}")
        for f in range(16):
            k = 4 if f % 5 == 0 else 3
            vs = rng.choice(nv, k, replace=False) + 1 + base_v
            ts = rng.choice(nv, k, replace=False) + 1 + base_t
            ns = rng.integers(0, 4, k) + 1 + base_n
            lines.append("f " + " ".join(f"{a}/{b}/{c}" for a, b, c in zip(vs, ts, ns)))
        base_v += nv; base_t += nv; base_n += 4
    texts["objects"] = "\n".join(lines) + "\n"
    # shared corners, -0.0 vs 0.0, integer forms, CRLF, no final newline
    texts["shared"] = ("v 0 0 0\r\nv -0.0 0 1\r\nv 1 0 0\r\nv 0.0 0 1\r\nv 1 1 1e-3\r\n"
                       "vt 0.5 0.5\r\nvt 2 -1\r\nvn 0 1 0\r\nvn -0 1 0\r\n"
                       "f 1/1/1 2/1/1 3/2/1\r\nf 1/1/1 4/1/2 3/2/1\r\nf 01/1/1 0x3/2/1 +5/1/2\r\n"
                       "f 2/1/1 4/1/1 5/2/2")
    # position-only faces
    texts["plain"] = "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nf 1 2 3\nf 2 4 3\nf 3 2 1 4\n"
    return texts


def obj_fixture():
    import tempfile
    from oracle_bind import ref_lib
    L = ref_lib()
    g = {}
    for name, text in obj_texts().items():
        fd, path = tempfile.mkstemp(suffix=".obj")
        with os.fdopen(fd, "wb") as f:
            f.write(text.encode())
        ni = __import__("ctypes").c_int()
        nv = L.ref_load_obj(path.encode(), __import__("ctypes").byref(ni))
        os.unlink(path)
        arr = {k: np.zeros(shape, np.float32) for k, shape in
               (("pos", (nv, 3)), ("nrm", (nv, 3)), ("uv0", (nv, 2)), ("uv1", (nv, 2)))}
        idx = np.zeros(ni.value, np.int32)
        L.ref_obj_arrays(ptr(arr["pos"]), ptr(arr["nrm"]), ptr(arr["uv0"]), ptr(arr["uv1"]), ptr(idx))
        for k, v in arr.items():
            g[f"{name}_{k}"] = v
        g[f"{name}_idx"] = idx
    np.savez_compressed(os.path.join(HERE, "obj.npz"), **g)
    return len(g)


POST_SHAPES = [(37, 23, 0.3), (64, 64, 0.6), (2, 5, 0.5), (48, 40, 0.85)]


def post_inputs(W, H, density, seed):
    rng = np.random.default_rng(seed)
    flags = (rng.random(W * H) < density).astype(np.int32)
    color = rng.uniform(-0.5, 3.0, (W * H, 3)).astype(np.float32)
    color[rng.random(W * H) < 0.02] = np.nan
    color[rng.random(W * H) < 0.02, 1] = np.inf
    color[rng.random(W * H) < 0.02, 2] = -1e10
    return flags, color


def post_fixture():
    import tempfile
    w = scenes.room_scene(size=16)
    ref = RefScene(w.scene)
    g = {}
    for c, (W, H, dens) in enumerate(POST_SHAPES):
        flags, color = post_inputs(W, H, dens, 100 + c)
        for op in ("expand", "blur"):
            k = ref.post_map(W, H, flags, color)
            getattr(ref.lib, "ref_map_" + op)(ref.h, k)
            g[f"{op}{c}"] = ref.map_colors(k, W, H)
        for fmt in (0, 1, 2):
            k = ref.post_map(W, H, flags, color)
            fd, path = tempfile.mkstemp()
            os.close(fd)
            ref.lib.ref_map_save(ref.h, k, path.encode(), fmt)
            with open(path, "rb") as f:
                g[f"file{c}_{fmt}"] = np.frombuffer(f.read(), np.uint8)
            os.unlink(path)
    np.savez_compressed(os.path.join(HERE, "post.npz"), **g)
    return len(POST_SHAPES)


def main():
    out = {}
    if sys.argv[1:] == ["post"]:
        print({"post": post_fixture()})
        return
    if sys.argv[1:] == ["obj"]:
        print({"obj": obj_fixture()})
        return
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
    # textured room: Texture::colorAt and the HitUseAlpha re-trace
    w = scenes.room_scene(size=48, textured=True)
    ref = RefScene(w.scene)
    seg = segments(w.scene.flat, 6000, 13)
    t = {"seg": seg}
    for flags in (15, 31):
        r = ref.trace_segments(seg, flags)
        t.update({f"{k}_{flags}": v for k, v in r.items()})
    ref.lib.ref_bake_direct(ref.h, ref.mesh(w.mesh), 0, 0, 1)
    lm = ref.lumels(w.lightmap)
    np.savez_compressed(os.path.join(HERE, "textured_room48.npz"), color=lm.color, flags=lm.flags, **t)
    out["textured_room48"] = int((lm.color.sum(1) > 0).sum())
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
    out["post"] = post_fixture()
    out["obj"] = obj_fixture()
    print(out)


if __name__ == "__main__":
    main()
