"""Host-side mirror of Relight's baking API (relight::Relight, Scene, Mesh,
Light, Material, Texture, Lightmap, Photonmap and the quality presets).

Names, argument meaning and error behaviour follow the reference:
  Relight            Relight.h:155-189, Relight.cpp:175-271
  settings presets   Relight.h:108-152, Relight.cpp:43-172
  Scene              scene/Scene.h:38-117, scene/Scene.cpp:80-142
  Mesh / Face        scene/Mesh.h:37-295, scene/Mesh.cpp:146-297
  Light + models     scene/Light.h:38-412, scene/Light.cpp:165-500
  Material/Texture   scene/Material.h:37-139, scene/Material.cpp:35-205
  Lightmap/Photonmap Lightmap.h:35-170, Lightmap.cpp:93-413

Everything here is host logic: it builds the flat, scene-space description
(`FlatScene`) that the CUDA library consumes.  Arithmetic that the
reference performs while building a scene (Mesh::transform, the area light's
face centroids, the directional emitter's plane) is done in float32 in the
reference's operation order, so the flat arrays equal the reference's
in-memory scene bit for bit.  Baking itself is delegated to
``relight_b200.device`` (the C-ABI in include/relight_b200.h).
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

F32 = np.float32


class RelightStatus(enum.IntEnum):
    """Relight.h:82-86."""
    RelightSuccess = 0
    RelightInvalidCall = 1
    RelightNotImplemented = 2


class RelightError(RuntimeError):
    """Raised for a non-success status from the CUDA library."""


# --------------------------------------------------------------- settings

@dataclass
class IndirectLightSettings:
    """Relight.h:108-128; presets Relight.cpp:43-120."""
    photon_pass_count: int = 8
    photon_bounce_count: int = 1
    photon_energy_threshold: float = 0.05
    photon_max_distance: float = 10.0
    final_gather_samples: int = 32
    final_gather_distance: float = 50.0
    final_gather_radius: int = 7
    sky_color: Sequence[float] = (0.0, 0.0, 0.0)
    ambient_color: Sequence[float] = (0.0, 0.0, 0.0)

    @staticmethod
    def _make(passes, bounces, samples, sky, ambient, photon_max_distance, final_gather_distance):
        return IndirectLightSettings(passes, bounces, 0.05, photon_max_distance, samples, final_gather_distance, 7,
                                     tuple(sky), tuple(ambient))

    @staticmethod
    def draft(sky=(0, 0, 0), ambient=(0, 0, 0), photon_max_distance=10.0, final_gather_distance=50.0):
        return IndirectLightSettings._make(8, 1, 32, sky, ambient, photon_max_distance, final_gather_distance)

    @staticmethod
    def fast(sky=(0, 0, 0), ambient=(0, 0, 0), photon_max_distance=10.0, final_gather_distance=50.0):
        return IndirectLightSettings._make(16, 3, 64, sky, ambient, photon_max_distance, final_gather_distance)

    @staticmethod
    def best(sky=(0, 0, 0), ambient=(0, 0, 0), photon_max_distance=10.0, final_gather_distance=50.0):
        return IndirectLightSettings._make(32, 3, 128, sky, ambient, photon_max_distance, final_gather_distance)

    @staticmethod
    def production(sky=(0, 0, 0), ambient=(0, 0, 0), photon_max_distance=10.0, final_gather_distance=50.0):
        return IndirectLightSettings._make(64, 4, 1024, sky, ambient, photon_max_distance, final_gather_distance)


@dataclass
class AmbientOcclusionSettings:
    """Relight.h:131-152; presets Relight.cpp:123-172 (128/256/1024/2048 samples)."""
    samples: int = 128
    occluded_fraction: float = 0.8
    max_distance: float = 0.6
    exponent: float = 1.0

    @staticmethod
    def draft(occluded_fraction=0.8, max_distance=0.6, exponent=1.0):
        return AmbientOcclusionSettings(128, occluded_fraction, max_distance, exponent)

    @staticmethod
    def fast(occluded_fraction=0.8, max_distance=0.6, exponent=1.0):
        return AmbientOcclusionSettings(256, occluded_fraction, max_distance, exponent)

    @staticmethod
    def best(occluded_fraction=0.8, max_distance=0.6, exponent=1.0):
        return AmbientOcclusionSettings(1024, occluded_fraction, max_distance, exponent)

    @staticmethod
    def production(occluded_fraction=0.8, max_distance=0.6, exponent=1.0):
        return AmbientOcclusionSettings(2048, occluded_fraction, max_distance, exponent)


# -------------------------------------------------------------- materials

class Material:
    """scene/Material.h:37-61: a diffuse colour (alpha 1)."""

    def __init__(self, color):
        self.color = np.asarray(color, dtype=F32).reshape(3)
        self.texture: Optional[Texture] = None


class Texture:
    """scene/Material.h:66-121: 8-bit RGB/RGBA pixels, nearest lookup with wrap."""

    def __init__(self, width, height, channels, pixels):
        self.width, self.height, self.channels = int(width), int(height), int(channels)
        self.pixels = np.ascontiguousarray(np.asarray(pixels, dtype=np.uint8).reshape(-1))
        if self.pixels.size != self.width * self.height * self.channels:
            raise ValueError("pixel buffer does not match width * height * channels")

    @staticmethod
    def create(width, height, channels, pixels):
        return Texture(width, height, channels, pixels)

    @staticmethod
    def create_from_file(file_name):
        """Texture::createFromFile (scene/Material.cpp:154-205): uncompressed
        24/32-bit TGA, red and blue swapped on load; None on failure."""
        try:
            with open(file_name, "rb") as f:
                data = f.read()
        except OSError:
            return None
        if len(data) < 18:
            return None
        header = data[12:18]
        width = header[1] * 256 + header[0]
        height = header[3] * 256 + header[2]
        if width <= 0 or height <= 0 or header[4] not in (24, 32):
            return None
        bpp = header[4] // 8
        px = np.frombuffer(data[18:18 + width * height * bpp], dtype=np.uint8).copy()
        if px.size < width * height * bpp:
            px = np.concatenate([px, np.zeros(width * height * bpp - px.size, np.uint8)])
        px = px.reshape(-1, bpp)
        px[:, [0, 2]] = px[:, [2, 0]]
        return Texture(width, height, bpp, px)


class TexturedMaterial(Material):
    """scene/Material.h:126-139: colour times texture colour."""

    def __init__(self, texture: Texture, color):
        super().__init__(color)
        if texture is None:
            raise ValueError("TexturedMaterial needs a texture")
        self.texture = texture


# ------------------------------------------------------------------ mesh

class Mesh:
    """Indexed triangle list with 16-bit indices (Relight.h:59, scene/Mesh.h:174-295)."""

    MAX_INDEX = 65535

    def __init__(self):
        self.positions = np.zeros((0, 3), F32)
        self.normals = np.zeros((0, 3), F32)
        self.uv0 = np.zeros((0, 2), F32)
        self.uv1 = np.zeros((0, 2), F32)
        self.materials: List[Optional[Material]] = []
        self.indices = np.zeros((0,), np.int32)
        self.lightmap: Optional[Lightmap] = None
        self.photonmap: Optional[Photonmap] = None
        self.user_data = None
        self.source = None  # (source mesh, transform, material) of a scene instance

    @staticmethod
    def create():
        return Mesh()

    @staticmethod
    def create_from_file(file_name) -> Optional["Mesh"]:
        """Mesh::createFromFile (scene/Mesh.cpp:111-122): a Wavefront OBJ
        read with MeshLoader's rules (rl_obj_load), uvs in the lightmap
        layer, no material; None if the file cannot be opened."""
        import ctypes as C
        import os
        from ._abi import check, lib
        if not os.path.isfile(file_name):
            return None
        h = C.c_void_p()
        check(lib().rl_obj_load(str(file_name).encode(), C.byref(h)))
        try:
            nv, ni, ns = C.c_int32(), C.c_int32(), C.c_int32()
            check(lib().rl_obj_mesh_counts(h, C.byref(nv), C.byref(ni), C.byref(ns)))
            pos = np.zeros((nv.value, 3), np.float32)
            nrm = np.zeros((nv.value, 3), np.float32)
            uv = np.zeros((nv.value, 2), np.float32)
            idx = np.zeros(ni.value, np.int32)
            ptr = lambda a: C.c_void_p(a.ctypes.data)
            check(lib().rl_obj_mesh_arrays(h, ptr(pos), ptr(nrm), ptr(uv), ptr(idx)))
        finally:
            lib().rl_obj_mesh_destroy(h)
        m = Mesh()
        if nv.value:
            m.add_faces(pos, nrm, None, uv, idx)
        return m

    def vertex_count(self):
        return int(self.positions.shape[0])

    def index_count(self):
        return int(self.indices.shape[0])

    def face_count(self):
        return self.index_count() // 3

    def bounds(self):
        """Mesh::bounds (scene/Mesh.cpp:214-217): min/max over vertices."""
        if self.vertex_count() == 0:
            return (np.full(3, np.finfo(F32).max, F32), np.full(3, -np.finfo(F32).max, F32))
        return self.positions.min(axis=0), self.positions.max(axis=0)

    def add_faces(self, positions, normals, uv0, uv1, indices, material: Optional[Material] = None):
        """Mesh::addFaces (scene/Mesh.cpp:146-165): append vertices with one
        material and indices offset by the current vertex count."""
        positions = np.asarray(positions, F32).reshape(-1, 3)
        n = positions.shape[0]
        normals = np.zeros((n, 3), F32) if normals is None else np.asarray(normals, F32).reshape(-1, 3)
        uv0 = np.zeros((n, 2), F32) if uv0 is None else np.asarray(uv0, F32).reshape(-1, 2)
        uv1 = np.zeros((n, 2), F32) if uv1 is None else np.asarray(uv1, F32).reshape(-1, 2)
        idx = np.asarray(indices, np.int64).reshape(-1) + self.vertex_count()
        if self.vertex_count() + n > self.MAX_INDEX + 1 or (idx.size and idx.max() > self.MAX_INDEX):
            raise ValueError("Relight meshes use 16-bit indices: at most 65536 vertices per mesh")
        self.indices = np.concatenate([self.indices, idx.astype(np.int32)])
        self.positions = np.concatenate([self.positions, positions])
        self.normals = np.concatenate([self.normals, normals])
        self.uv0 = np.concatenate([self.uv0, uv0])
        self.uv1 = np.concatenate([self.uv1, uv1])
        self.materials.extend([material] * n)
        return self

    def override_material(self, material: Material):
        """Mesh::overrideMaterial (scene/Mesh.cpp:126-131)."""
        self.materials = [material] * self.vertex_count()

    def transformed(self, matrix=None) -> "Mesh":
        """Mesh::transformed -> Mesh::transform (scene/Mesh.cpp:277-297):
        p' = M * p (Types.h:1188-1196), n' = normalize(M.rotate(n))
        (Types.h:1304-1312, 852-859), evaluated in float32 in that order."""
        m = np.eye(4, dtype=F32).reshape(16) if matrix is None else np.asarray(matrix, F32).reshape(16)
        out = Mesh()
        p = self.positions
        x, y, z = p[:, 0], p[:, 1], p[:, 2]
        out.positions = np.stack([x * m[0] + y * m[4] + z * m[8] + m[12],
                                  x * m[1] + y * m[5] + z * m[9] + m[13],
                                  x * m[2] + y * m[6] + z * m[10] + m[14]], axis=1).astype(F32)
        n = self.normals
        nx, ny, nz = n[:, 0], n[:, 1], n[:, 2]
        r = np.stack([nx * m[0] + ny * m[4] + nz * m[8],
                      nx * m[1] + ny * m[5] + nz * m[9],
                      nx * m[2] + ny * m[6] + nz * m[10]], axis=1).astype(F32)
        out.normals = _normalize_rows(r)
        out.uv0 = self.uv0.copy()
        out.uv1 = self.uv1.copy()
        out.materials = list(self.materials)
        out.indices = self.indices.copy()
        return out


def _normalize_rows(v):
    """Vec3::normalize (Types.h:852-859) per row, float32: len = sqrt(x*x + y*y + z*z)."""
    v = np.asarray(v, F32)
    x, y, z = v[:, 0], v[:, 1], v[:, 2]
    ln = np.sqrt(x * x + y * y + z * z).astype(F32)
    safe = np.where(ln != 0, ln, F32(1))
    out = np.stack([x / safe, y / safe, z / safe], axis=1).astype(F32)
    return np.where((ln != 0)[:, None], out, v)


# ------------------------------------------------------------------ lights

@dataclass
class LinearLightAttenuation:
    """scene/Light.h:117-136: 1 / (1 + c + l*r + q*r*r), r = d / radius."""
    radius: float
    constant: float = 0.0
    linear: float = 0.0
    quadratic: float = 25.0


@dataclass
class LightSpotCutoff:
    """scene/Light.h:60-89."""
    direction: Sequence[float]
    cutoff: float
    exponent: float = 1.0


INFLUENCE_NONE, INFLUENCE_POINT, INFLUENCE_DIRECTIONAL = 0, 1, 2
CUTOFF_NONE, CUTOFF_OMNI, CUTOFF_SPOT = 0, 1, 2
EMITTER_NONE, EMITTER_POINT, EMITTER_DIRECTIONAL = 0, 1, 2


class Light:
    """A Relight light: influence, attenuation, cutoff, vertex generator and
    photon emitter models (scene/Light.h:228-336)."""

    def __init__(self):
        self.position = np.zeros(3, F32)
        self.color = np.ones(3, F32)
        self.intensity = F32(0)
        self.casts_shadow = False
        self.influence = INFLUENCE_NONE
        self.direction = np.zeros(3, F32)
        self.attenuation: Optional[LinearLightAttenuation] = None
        self.cutoff = CUTOFF_NONE
        self.spot: Optional[LightSpotCutoff] = None
        self.emitter = EMITTER_NONE
        self.emitter_plane = np.zeros(4, F32)
        self.vertices: Optional[np.ndarray] = None  # light-local sample points
        self.factory = None  # (name, args) of the creating factory call
        self.attenuation_overridden = False

    # setters mirroring scene/Light.cpp:52-163
    def set_attenuation(self, value: Optional[LinearLightAttenuation]):
        self.attenuation = value
        self.attenuation_overridden = True

    def set_photon_emitter(self, kind: int):
        self.emitter = kind

    def set_position(self, value):
        self.position = np.asarray(value, F32).reshape(3)

    def set_color(self, value):
        self.color = np.asarray(value, F32).reshape(3)

    def set_intensity(self, value):
        self.intensity = F32(value)

    def set_casts_shadow(self, value):
        self.casts_shadow = bool(value)

    @staticmethod
    def create_point_light(position, radius, color=(1, 1, 1), intensity=1.0, casts_shadow=True):
        """Light::createPointLight (scene/Light.cpp:166-180)."""
        l = Light()
        l.influence = INFLUENCE_POINT
        l.attenuation = LinearLightAttenuation(float(radius))
        l.emitter = EMITTER_POINT
        l.cutoff = CUTOFF_OMNI
        l.casts_shadow = bool(casts_shadow)
        l.set_position(position); l.set_color(color); l.set_intensity(intensity)
        l.factory = ("point", (position, radius, color, intensity, casts_shadow))
        return l

    @staticmethod
    def create_spot_light(position, direction, cutoff, radius, color=(1, 1, 1), intensity=1.0, casts_shadow=True):
        """Light::createSpotLight (scene/Light.cpp:183-197): spot exponent 1."""
        l = Light.create_point_light(position, radius, color, intensity, casts_shadow)
        l.cutoff = CUTOFF_SPOT
        l.spot = LightSpotCutoff(tuple(np.asarray(direction, F32).reshape(3)), float(cutoff), 1.0)
        l.factory = ("spot", (position, direction, cutoff, radius, color, intensity, casts_shadow))
        return l

    @staticmethod
    def create_directional_light(direction, color=(1, 1, 1), intensity=1.0, casts_shadow=True):
        """Light::createDirectionalLight (scene/Light.cpp:200-211).  The
        emitter's plane is Plane::calculate(direction, position) with the
        position still at its default (0, 0, 0) (Types.h:1656-1658)."""
        l = Light()
        d = np.asarray(direction, F32).reshape(3)
        l.influence = INFLUENCE_DIRECTIONAL
        l.direction = d.copy()
        l.emitter = EMITTER_DIRECTIONAL
        dist = -(d[0] * F32(0) + d[1] * F32(0) + d[2] * F32(0))
        l.emitter_plane = np.array([d[0], d[1], d[2], dist], F32)
        l.casts_shadow = bool(casts_shadow)
        l.set_color(color); l.set_intensity(intensity)
        l.factory = ("directional", (direction, color, intensity, casts_shadow))
        return l

    @staticmethod
    def create_area_light(mesh: Mesh, position, color=(1, 1, 1), intensity=1.0, casts_shadow=True):
        """Light::createAreaLight (scene/Light.cpp:214-234): attenuation radius
        = light mesh bounds volume, one light vertex per face centroid
        (FaceLightVertexGenerator(mesh, true, 0), :293-323).  The centroid is
        Triangle(face)'s (m_a + m_b + m_c) / 3 (scene/Mesh.cpp:321-326) where
        Face::vertex maps 0,1,2 to a, c, b (scene/Mesh.cpp:441-451)."""
        l = Light.create_point_light(position, 1.0, color, intensity, casts_shadow)
        lo, hi = mesh.bounds()
        vol = (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2])
        l.attenuation = LinearLightAttenuation(float(F32(vol)))
        idx = mesh.indices.reshape(-1, 3)
        a = mesh.positions[idx[:, 0]]
        b = mesh.positions[idx[:, 1]]
        c = mesh.positions[idx[:, 2]]
        l.vertices = ((a + c + b) / F32(3.0)).astype(F32)
        l.factory = ("area", (mesh, position, color, intensity, casts_shadow))
        return l


# ---------------------------------------------------------------- lightmaps

class Lightmap:
    """Lightmap.h:58-150.  Lumel arrays live on the device after a bake; the
    host copy is read with `lumels()` / `to_hdr()`."""

    KIND = 0

    def __init__(self, width: int, height: int):
        if width <= 0 or height <= 0:
            raise ValueError("lightmap size must be positive")
        self.width = int(width)
        self.height = int(height)
        self.meshes: List[Mesh] = []
        self._device = None  # set by the device layer once the scene ends

    def add_mesh(self, mesh: Mesh) -> RelightStatus:
        """Lightmap::addMesh (Lightmap.cpp:93-106): a mesh takes one lightmap."""
        if mesh.lightmap is not None:
            return RelightStatus.RelightInvalidCall
        mesh.lightmap = self
        self.meshes.append(mesh)
        return RelightStatus.RelightSuccess


class Photonmap(Lightmap):
    """Lightmap.h:153-170."""

    KIND = 1

    def add_mesh(self, mesh: Mesh, copy_vertex_color=False) -> RelightStatus:
        if mesh.photonmap is not None:
            return RelightStatus.RelightInvalidCall
        mesh.photonmap = self
        self.meshes.append(mesh)
        return RelightStatus.RelightSuccess


# ------------------------------------------------------------------- scene

LIGHT_DTYPE = np.dtype([
    ("influence", np.int32), ("casts_shadow", np.int32),
    ("position", np.float32, 3), ("color", np.float32, 3), ("intensity", np.float32),
    ("direction", np.float32, 3),
    ("attenuation", np.int32), ("att_radius", np.float32), ("att_const", np.float32),
    ("att_linear", np.float32), ("att_quadratic", np.float32),
    ("cutoff", np.int32), ("spot_direction", np.float32, 3), ("spot_cutoff", np.float32),
    ("spot_exponent", np.float32),
    ("emitter", np.int32), ("emitter_plane", np.float32, 4),
    ("vertex_first", np.int32), ("vertex_count", np.int32),
])
assert LIGHT_DTYPE.itemsize == 120


@dataclass
class FlatScene:
    """All meshes concatenated in scene space: the layout of rl_scene_desc
    (include/relight_b200.h) that the CUDA library and the oracle take."""
    pos: np.ndarray
    nrm: np.ndarray
    uv0: np.ndarray
    uv1: np.ndarray
    vmat: np.ndarray
    tris: np.ndarray
    mesh_first_tri: np.ndarray
    mesh_lightmap: np.ndarray
    mesh_photonmap: np.ndarray
    mat_rgb: np.ndarray
    mat_tex: np.ndarray
    tex_dims: np.ndarray
    tex_offset: np.ndarray
    tex_pixels: np.ndarray
    bounds_lo: np.ndarray
    bounds_hi: np.ndarray
    lights: np.ndarray
    light_vertices: np.ndarray
    lightmaps: List[Lightmap] = field(default_factory=list)
    photonmaps: List[Photonmap] = field(default_factory=list)

    @property
    def ntris(self):
        return int(self.tris.shape[0])

    @property
    def nmeshes(self):
        return int(self.mesh_first_tri.shape[0] - 1)


class Scene:
    """scene/Scene.h:38-117."""

    STATE_INITIAL, STATE_ADDING, STATE_READY = 0, 1, 2

    def __init__(self):
        self.meshes: List[Mesh] = []
        self.lights: List[Light] = []
        self.state = Scene.STATE_INITIAL
        self.flat: Optional[FlatScene] = None
        self._device = None

    def begin(self) -> RelightStatus:
        """Scene::begin (scene/Scene.cpp:110-119)."""
        if self.state != Scene.STATE_INITIAL:
            return RelightStatus.RelightInvalidCall
        self.state = Scene.STATE_ADDING
        return RelightStatus.RelightSuccess

    def add_mesh(self, mesh: Mesh, transform=None, material: Optional[Material] = None) -> Mesh:
        """Scene::addMesh (scene/Scene.cpp:98-107): a transformed copy."""
        inst = mesh.transformed(transform)
        if material is not None:
            inst.override_material(material)
        inst.source = (mesh, transform, material)
        self.meshes.append(inst)
        return inst

    def add_light(self, light: Light) -> RelightStatus:
        self.lights.append(light)
        return RelightStatus.RelightSuccess

    def light_count(self):
        return len(self.lights)

    def mesh_count(self):
        return len(self.meshes)

    def bounds(self):
        """Scene::updateBounds (scene/Scene.cpp:81-88)."""
        lo = np.full(3, np.finfo(F32).max, F32)
        hi = np.full(3, -np.finfo(F32).max, F32)
        for m in self.meshes:
            a, b = m.bounds()
            lo = np.minimum(lo, a); hi = np.maximum(hi, b)
        return lo, hi

    def end(self) -> RelightStatus:
        """Scene::end (scene/Scene.cpp:122-142): freezes the scene and builds
        the flat description; the device layer builds the BVH from it."""
        if self.state != Scene.STATE_ADDING:
            return RelightStatus.RelightInvalidCall
        self.flat = flatten(self)
        self.state = Scene.STATE_READY
        return RelightStatus.RelightSuccess


def flatten(scene: Scene) -> FlatScene:
    meshes = scene.meshes
    lightmaps: List[Lightmap] = []
    photonmaps: List[Photonmap] = []
    for m in meshes:
        if m.lightmap is not None and m.lightmap not in lightmaps:
            lightmaps.append(m.lightmap)
        if m.photonmap is not None and m.photonmap not in photonmaps:
            photonmaps.append(m.photonmap)
    mats: List[Material] = []
    mat_ids = {}
    vmat_parts = []
    for m in meshes:
        ids = np.empty(m.vertex_count(), np.int32)
        for i, mat in enumerate(m.materials):
            if mat is None:
                ids[i] = -1
                continue
            k = id(mat)
            if k not in mat_ids:
                mat_ids[k] = len(mats)
                mats.append(mat)
            ids[i] = mat_ids[k]
        vmat_parts.append(ids)
    texs: List[Texture] = []
    for mat in mats:
        if mat.texture is not None and all(t is not mat.texture for t in texs):
            texs.append(mat.texture)
    vbase = np.cumsum([0] + [m.vertex_count() for m in meshes])
    tris = [m.indices.reshape(-1, 3).astype(np.int32) + np.int32(vbase[i]) for i, m in enumerate(meshes)]
    first = np.cumsum([0] + [m.face_count() for m in meshes]).astype(np.int32)
    tex_dims = np.array([[t.width, t.height, t.channels] for t in texs], np.int32).reshape(-1, 3)
    tex_off = np.cumsum([0] + [t.pixels.size for t in texs]).astype(np.int64)
    lo, hi = scene.bounds()
    lights = np.zeros(len(scene.lights), LIGHT_DTYPE)
    lverts = []
    nv = 0
    for i, l in enumerate(scene.lights):
        rec = lights[i]
        rec["influence"] = l.influence
        rec["casts_shadow"] = int(l.casts_shadow)
        rec["position"] = l.position
        rec["color"] = l.color
        rec["intensity"] = l.intensity
        rec["direction"] = l.direction
        if l.attenuation is not None:
            a = l.attenuation
            rec["attenuation"] = 1
            rec["att_radius"], rec["att_const"] = a.radius, a.constant
            rec["att_linear"], rec["att_quadratic"] = a.linear, a.quadratic
        rec["cutoff"] = l.cutoff
        if l.spot is not None:
            rec["spot_direction"] = l.spot.direction
            rec["spot_cutoff"] = l.spot.cutoff
            rec["spot_exponent"] = l.spot.exponent
        rec["emitter"] = l.emitter
        rec["emitter_plane"] = l.emitter_plane
        if l.vertices is not None and len(l.vertices):
            rec["vertex_first"] = nv
            rec["vertex_count"] = len(l.vertices)
            lverts.append(l.vertices)
            nv += len(l.vertices)
    return FlatScene(
        pos=np.ascontiguousarray(np.concatenate([m.positions for m in meshes]) if meshes else np.zeros((0, 3), F32)),
        nrm=np.ascontiguousarray(np.concatenate([m.normals for m in meshes]) if meshes else np.zeros((0, 3), F32)),
        uv0=np.ascontiguousarray(np.concatenate([m.uv0 for m in meshes]) if meshes else np.zeros((0, 2), F32)),
        uv1=np.ascontiguousarray(np.concatenate([m.uv1 for m in meshes]) if meshes else np.zeros((0, 2), F32)),
        vmat=np.ascontiguousarray(np.concatenate(vmat_parts) if meshes else np.zeros(0, np.int32)),
        tris=np.ascontiguousarray(np.concatenate(tris) if meshes else np.zeros((0, 3), np.int32)),
        mesh_first_tri=first,
        mesh_lightmap=np.array([lightmaps.index(m.lightmap) if m.lightmap is not None else -1 for m in meshes],
                               np.int32),
        mesh_photonmap=np.array([photonmaps.index(m.photonmap) if m.photonmap is not None else -1 for m in meshes],
                                np.int32),
        mat_rgb=np.array([m.color for m in mats], F32).reshape(-1, 3),
        mat_tex=np.array([texs.index(m.texture) if m.texture is not None else -1 for m in mats], np.int32),
        tex_dims=tex_dims,
        tex_offset=tex_off[:-1].copy() if len(texs) else np.zeros(0, np.int64),
        tex_pixels=np.concatenate([t.pixels for t in texs]) if texs else np.zeros(1, np.uint8),
        bounds_lo=lo.astype(F32), bounds_hi=hi.astype(F32),
        lights=lights,
        light_vertices=np.ascontiguousarray(np.concatenate(lverts).astype(F32) if lverts else np.zeros((1, 3), F32)),
        lightmaps=lightmaps, photonmaps=photonmaps,
    )
