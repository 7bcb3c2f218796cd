"""Seeded synthetic bake workloads, built through the Relight-style API.

  room_scene      10x10x10 closed room (6 inward quads) + N axis-aligned boxes,
                  one mesh, one lightmap; point, spot (45 deg cone) and 1x1
                  area (16-triangle) lights.  The direct-light + AO workload.
                  textured=True gives the walls plain coloured materials and
                  the boxes an RGBA texture with cut-out texels (alpha <= 0.1),
                  so shadow rays take Relight's alpha re-trace.
  terrain_scene   256x256-vertex fBm heightfield (amplitude 5) split into 2x2
                  tiles (16-bit index limit) + 2,000 boxes; per-vertex albedo in
                  [0.2, 0.8]; one sun + 4 point lights; one shared 1024^2
                  lightmap and photonmap.  The photon + final-gather workload.
  radiosity_room  10x5x10 room whose 128x128 radiancemap texels are the
                  16,384 radiosity patches.
  batch_workload  uneven-size batching: scenes of log-uniform triangle
                  counts (heightfield patch + boxes, terrain_scene's recipe)
                  and bake jobs with log-uniform lightmap sides, each job
                  baked with direct light, AO and final gather.

Every chart is an axis-aligned rectangle in the lightmap with a one-texel
gutter, so texel rasterisation (Lightmap::initializeLumels) covers it fully.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List

import numpy as np

from .api import (AmbientOcclusionSettings, IndirectLightSettings, Light, LinearLightAttenuation, Material, Mesh,
                  Photonmap, Lightmap, Scene, Texture, TexturedMaterial)

F32 = np.float32


def _quad(corners, normal, uv_rect, transpose=False):
    """Four corners (lo-lo, hi-lo, hi-hi, lo-hi in the face's tangent axes),
    a flat normal and a uv rectangle (u0, v0, u1, v1): two triangles.
    transpose maps the face's second tangent axis to u instead of the first."""
    u0, v0, u1, v1 = uv_rect
    pos = np.asarray(corners, F32)
    if transpose:
        pos = pos[[0, 3, 2, 1]]
    nrm = np.tile(np.asarray(normal, F32), (4, 1))
    uv = np.array([[u0, v0], [u1, v0], [u1, v1], [u0, v1]], F32)
    idx = np.array([0, 1, 2, 0, 2, 3], np.int32)
    return pos, nrm, uv, idx


def _box_faces(lo, hi, inward=False):
    """Six axis-aligned faces of a box as (corners, normal)."""
    lo = np.asarray(lo, F32); hi = np.asarray(hi, F32)
    faces = []
    for axis in range(3):
        i, j = [(1, 2), (2, 0), (0, 1)][axis]
        for side in (0, 1):
            c = hi[axis] if side else lo[axis]
            n = np.zeros(3, F32)
            n[axis] = 1.0 if side else -1.0
            if inward:
                n = -n
            pts = []
            for (a, b) in ((0, 0), (1, 0), (1, 1), (0, 1)):
                p = np.zeros(3, F32)
                p[axis] = c
                p[i] = hi[i] if a else lo[i]
                p[j] = hi[j] if b else lo[j]
                pts.append(p)
            faces.append((np.array(pts), n))
    return faces


def _cell_rect(cell, cols, cell_px, width, height, x0=0, y0=0, gutter=1):
    cx, cy = cell % cols, cell // cols
    u0 = (x0 + cx * cell_px + gutter) / width
    u1 = (x0 + (cx + 1) * cell_px - gutter) / width
    v0 = (y0 + cy * cell_px + gutter) / height
    v1 = (y0 + (cy + 1) * cell_px - gutter) / height
    return u0, v0, u1, v1


@dataclass
class RoomWorkload:
    scene: Scene
    mesh: Mesh
    lightmap: Lightmap
    ao: AmbientOcclusionSettings


def alpha_texture(size: int = 16, seed: int = 5) -> Texture:
    """An RGBA texture of random colours whose alpha is a checkerboard of
    4x4-texel cells: cut-out cells hold alpha 0 or 25 (25/255 <= 0.1, so
    Relight's HitUseAlpha passes through them) and opaque cells 26 (just
    above 0.1), 128 or 255."""
    rng = np.random.default_rng(seed)
    px = np.zeros((size, size, 4), np.uint8)
    px[..., :3] = rng.integers(40, 256, (size, size, 3))
    y, x = np.mgrid[0:size, 0:size]
    cut = ((x // 4 + y // 4) % 2) == 0
    px[..., 3] = np.where(cut, rng.choice([0, 25], (size, size)), rng.choice([26, 128, 255], (size, size)))
    return Texture.create(size, size, 4, px.reshape(-1))


def room_scene(seed: int = 1, size: int = 256, n_boxes: int = 8, room: float = 10.0,
               area_light: bool = True, spot_light: bool = True, material=None,
               textured: bool = False) -> RoomWorkload:
    rng = np.random.default_rng(seed)
    faces = _box_faces((0, 0, 0), (room, room, room), inward=True)
    for _ in range(n_boxes):
        s = rng.uniform(0.5, 2.0, 3)
        c = rng.uniform(s / 2 + 0.05, room - s / 2 - 0.05)
        faces += _box_faces(c - s / 2, c + s / 2)
    cols = int(math.ceil(math.sqrt(len(faces))))
    cell = size // cols
    mats = [material] * len(faces)
    uv0s = [None] * len(faces)
    if textured:
        # own generator: the geometry stays that of the untextured room
        trng = np.random.default_rng(seed + 1000)
        tex = alpha_texture(16, seed + 2000)
        for k in range(6):
            mats[k] = Material(trng.uniform(0.3, 0.9, 3))
        box_mats = [TexturedMaterial(tex, trng.uniform(0.5, 1.0, 3)) for _ in range(3)]
        for k in range(6, len(faces)):
            mats[k] = box_mats[k % 3]
            # diffuse uvs over 1 or 2 texture periods (wrap), some starting
            # below 0 (Texture::colorAt's out-of-range colour)
            span = 1.0 + (k % 2)
            u0, v0 = (-0.5, -0.25) if k % 5 == 0 else (0.0, 0.0)
            uv0s[k] = np.array([[u0, v0], [u0 + span, v0], [u0 + span, v0 + span], [u0, v0 + span]], F32)
    src = Mesh.create()
    for k, (corners, n) in enumerate(faces):
        pos, nrm, uv, idx = _quad(corners, n, _cell_rect(k, cols, cell, size, size))
        src.add_faces(pos, nrm, uv0s[k], uv, idx, mats[k])
    scene = Scene()
    scene.begin()
    mesh = scene.add_mesh(src)
    lm = Lightmap(size, size)
    lm.add_mesh(mesh)
    scene.add_light(Light.create_point_light((room / 2, room * 0.95, room / 2), room, (1, 1, 1), 1.0, True))
    if spot_light:
        p = np.array([room * 0.2, room * 0.8, room * 0.2], F32)
        d = np.array([room / 2, 0, room / 2], F32) - p
        d = (d / np.float32(np.sqrt((d * d).sum()))).astype(F32)
        scene.add_light(Light.create_spot_light(p, d, math.cos(math.radians(22.5)), room, (1.0, 0.9, 0.7), 1.0, True))
    if area_light:
        lmesh = Mesh.create()
        # 1x1 quad as a 4x2 grid of cells, two triangles each: 16 triangles
        gx, gz = 4, 2
        pts, idx = [], []
        for z in range(gz + 1):
            for x in range(gx + 1):
                pts.append([-0.5 + x / gx, 0.0, -0.5 + z / gz])
        for z in range(gz):
            for x in range(gx):
                a = z * (gx + 1) + x
                idx += [a, a + 1, a + gx + 2, a, a + gx + 2, a + gx + 1]
        lmesh.add_faces(np.array(pts, F32), np.tile([0, -1, 0], (len(pts), 1)), None, None, np.array(idx))
        al = Light.create_area_light(lmesh, (room * 0.7, room * 0.9, room * 0.7), (0.8, 0.9, 1.0), 1.0, True)
        al.set_attenuation(LinearLightAttenuation(room))
        scene.add_light(al)
    scene.end()
    return RoomWorkload(scene, mesh, lm, AmbientOcclusionSettings(64, 0.8, 2.0, 1.0))


# ------------------------------------------------------------------ terrain

def _value_noise(rng, n, octaves=5):
    """Seeded fBm of bilinear value noise on an n x n grid, in [0, 1]."""
    out = np.zeros((n, n), np.float64)
    amp, total = 1.0, 0.0
    for o in range(octaves):
        cells = 4 * (2 ** o)
        lattice = rng.random((cells + 2, cells + 2))
        t = np.linspace(0, cells, n, endpoint=False)
        i = np.floor(t).astype(int)
        f = t - i
        f = f * f * (3 - 2 * f)
        a = lattice[i][:, i]; b = lattice[i + 1][:, i]; c = lattice[i][:, i + 1]; d = lattice[i + 1][:, i + 1]
        fx = f[:, None]; fz = f[None, :]
        out += amp * ((a * (1 - fx) + b * fx) * (1 - fz) + (c * (1 - fx) + d * fx) * fz)
        total += amp
        amp *= 0.5
    out /= total
    out -= out.min()
    return out / max(out.max(), 1e-12)


@dataclass
class TerrainWorkload:
    scene: Scene
    meshes: List[Mesh]
    lightmap: Lightmap
    photonmap: Photonmap
    settings: IndirectLightSettings


def terrain_scene(seed: int = 2, verts: int = 256, n_boxes: int = 2000, size: int = 1024,
                  amplitude: float = 5.0, tiles: int = 2, fg_samples: int = 256, passes: int = 8,
                  bounces: int = 3) -> TerrainWorkload:
    rng = np.random.default_rng(seed)
    h = (_value_noise(rng, verts) * amplitude).astype(F32)
    palette = [Material(rng.uniform(0.2, 0.8, 3)) for _ in range(256)]
    # normals from central differences of the height field
    gx = np.zeros_like(h); gz = np.zeros_like(h)
    gx[1:-1, :] = (h[2:, :] - h[:-2, :]) * 0.5
    gx[0, :] = h[1, :] - h[0, :]; gx[-1, :] = h[-1, :] - h[-2, :]
    gz[:, 1:-1] = (h[:, 2:] - h[:, :-2]) * 0.5
    gz[:, 0] = h[:, 1] - h[:, 0]; gz[:, -1] = h[:, -1] - h[:, -2]
    nrm = np.stack([-gx, np.ones_like(h), -gz], axis=-1).astype(F32)
    nrm /= np.sqrt((nrm * nrm).sum(-1, keepdims=True)).astype(F32)
    vmat = rng.integers(0, len(palette), (verts, verts))
    scene = Scene()
    scene.begin()
    lm = Lightmap(size, size)
    pm = Photonmap(size, size)
    meshes = []
    quads = verts - 1
    edges = np.linspace(0, quads, tiles + 1).astype(int)
    terrain_rows = (size * 3) // 4
    region_w, region_h = size // tiles, terrain_rows // tiles
    for tz in range(tiles):
        for tx in range(tiles):
            x0, x1 = edges[tx], edges[tx + 1]
            z0, z1 = edges[tz], edges[tz + 1]
            nx, nz = x1 - x0 + 1, z1 - z0 + 1
            xs, zs = np.meshgrid(np.arange(x0, x1 + 1), np.arange(z0, z1 + 1), indexing="ij")
            pos = np.stack([xs, h[xs, zs], zs], axis=-1).reshape(-1, 3).astype(F32)
            tn = nrm[xs, zs].reshape(-1, 3)
            fu = (xs - x0) / (x1 - x0); fv = (zs - z0) / (z1 - z0)
            u = (tx * region_w + 1 + fu * (region_w - 2)) / size
            v = (tz * region_h + 1 + fv * (region_h - 2)) / size
            uv = np.stack([u, v], axis=-1).reshape(-1, 2).astype(F32)
            ii, jj = np.meshgrid(np.arange(nx - 1), np.arange(nz - 1), indexing="ij")
            a = (ii * nz + jj).reshape(-1)
            b = a + nz; c = a + nz + 1; d = a + 1
            idx = np.stack([a, b, c, a, c, d], axis=-1).reshape(-1)
            src = Mesh.create()
            src.add_faces(pos, tn, None, uv, idx)
            src.materials = [palette[k] for k in vmat[xs, zs].reshape(-1)]
            inst = scene.add_mesh(src)
            lm.add_mesh(inst); pm.add_mesh(inst)
            meshes.append(inst)
    # boxes standing on the terrain, in cells below the terrain region: 4x4
    # texels when they fit, smaller otherwise, and shared (wrapped) beyond
    # that, so every lightmap uv stays inside [0, 1] (Lightmap::lumel(uv)
    # does not range-check, Lightmap.cpp:61-67)
    src = Mesh.create()
    rows_px = size - terrain_rows
    cell = 4
    while cell > 1 and (size // cell) * (rows_px // cell) < 6 * n_boxes:
        cell //= 2
    cols = size // cell
    ncells = cols * (rows_px // cell)
    k = 0
    per_mesh = (Mesh.MAX_INDEX + 1) // 24  # 24 vertices per box, 16-bit indices
    for b in range(n_boxes):
        if b > 0 and b % per_mesh == 0:
            inst = scene.add_mesh(src)
            lm.add_mesh(inst); pm.add_mesh(inst)
            meshes.append(inst)
            src = Mesh.create()
        s = rng.uniform(0.5, 2.0, 3).astype(F32)
        cx, cz = rng.uniform(2, quads - 2, 2)
        base = h[int(round(cx)), int(round(cz))] - 0.1
        lo = np.array([cx - s[0] / 2, base, cz - s[2] / 2], F32)
        hi = np.array([cx + s[0] / 2, base + s[1], cz + s[2] / 2], F32)
        mat = palette[int(rng.integers(0, len(palette)))]
        for corners, n in _box_faces(lo, hi):
            pos, nn, uv, idx = _quad(corners, n, _cell_rect(k % ncells, cols, cell, size, size, y0=terrain_rows,
                                                            gutter=1 if cell >= 3 else 0))
            src.add_faces(pos, nn, None, uv, idx, mat)
            k += 1
    inst = scene.add_mesh(src)
    lm.add_mesh(inst); pm.add_mesh(inst)
    meshes.append(inst)
    sun = np.array([0.3, -1.0, 0.2], F32)
    sun = (sun / np.float32(np.sqrt((sun * sun).sum()))).astype(F32)
    scene.add_light(Light.create_directional_light(sun, (1.0, 0.95, 0.85), 1.0, True))
    for (px, pz) in ((0.25, 0.25), (0.75, 0.25), (0.25, 0.75), (0.75, 0.75)):
        scene.add_light(Light.create_point_light((px * quads, amplitude + 10.0, pz * quads), 40.0,
                                                 (1.0, 0.9, 0.8), 1.0, True))
    scene.end()
    st = IndirectLightSettings(passes, bounces, 0.05, 200.0, fg_samples, 50.0, 7, (0.5, 0.6, 0.8), (0, 0, 0))
    return TerrainWorkload(scene, meshes, lm, pm, st)


# ---------------------------------------------------------------- radiosity

@dataclass
class RadiosityWorkload:
    scene: Scene
    mesh: Mesh
    radiancemap: Lightmap
    albedo_seed: int


def radiosity_room(size: int = 128, seed: int = 3, dims=(10.0, 5.0, 10.0)) -> RadiosityWorkload:
    """A closed room; its radiancemap's texels are the patches.  Layout of the
    size x size map: floor | ceiling in the top half, the four walls in the
    bottom half, texel pitch equal on every face, every texel valid."""
    W, H, D = dims
    half = size // 2
    q = size // 4
    faces = _box_faces((0, 0, 0), (W, H, D), inward=True)
    # _box_faces order: -x, +x, -y, +y, -z, +z
    rects = {
        2: (0, 0, half, half),           # floor   (y = 0)
        3: (half, 0, size, half),        # ceiling (y = H)
        0: (0, half, half, half + q),    # wall x = 0
        1: (half, half, size, half + q), # wall x = W
        4: (0, half + q, half, size),    # wall z = 0
        5: (half, half + q, size, size), # wall z = D
    }
    src = Mesh.create()
    for k, (corners, n) in enumerate(faces):
        x0, y0, x1, y1 = rects[k]
        pos, nrm, uv, idx = _quad(corners, n, (x0 / size, y0 / size, x1 / size, y1 / size), transpose=k in (0, 1))
        src.add_faces(pos, nrm, None, uv, idx)
    scene = Scene()
    scene.begin()
    mesh = scene.add_mesh(src)
    rm = Lightmap(size, size)
    rm.add_mesh(mesh)
    scene.end()
    return RadiosityWorkload(scene, mesh, rm, seed)


# ------------------------------------------------------------------ batches

@dataclass
class BatchJobSpec:
    scene: int          # index into BatchWorkload.scenes
    side: int           # lightmap width = height
    seed: int


@dataclass
class BatchWorkload:
    scenes: List[TerrainWorkload]
    triangles: List[int]
    jobs: List[BatchJobSpec]
    ao: AmbientOcclusionSettings


def _log_uniform(rng, lo, hi):
    return float(np.exp(rng.uniform(np.log(lo), np.log(hi))))


def batch_workload(n_jobs: int = 512, n_scenes: int = 32, seed: int = 4, tris=(1_000, 500_000),
                   sides=(32, 1024), ao_samples: int = 64, fg_samples: int = 128, photon_map: int = 256,
                   photon_passes: int = 1) -> BatchWorkload:
    """Scenes: a heightfield patch (about 90% of the triangles, tiled under
    the 16-bit index limit) plus boxes (about 10%), with terrain_scene's sun
    and 4 point lights and one `photon_map`-sided photonmap.  Jobs: a scene
    drawn uniformly and a lightmap side log-uniform in `sides`."""
    rng = np.random.default_rng(seed)
    scenes, counts = [], []
    for k in range(n_scenes):
        t = _log_uniform(rng, *tris)
        verts = max(8, int(round(math.sqrt(0.9 * t / 2.0))) + 1)
        n_boxes = max(1, int(round(0.1 * t / 12.0)))
        tiles = max(1, int(math.ceil((verts - 1) / 255.0)))
        wl = terrain_scene(seed=seed * 1000 + k, verts=verts, n_boxes=n_boxes, size=photon_map, tiles=tiles,
                           fg_samples=fg_samples, passes=photon_passes)
        scenes.append(wl)
        counts.append(int(sum(m.face_count() for m in wl.meshes)))
    jobs = []
    for q in range(n_jobs):
        side = int(round(_log_uniform(rng, *sides)))
        jobs.append(BatchJobSpec(int(rng.integers(0, n_scenes)), side, int(rng.integers(0, 2 ** 63))))
    return BatchWorkload(scenes, counts, jobs, AmbientOcclusionSettings(ao_samples, 0.8, 2.0, 1.0))
