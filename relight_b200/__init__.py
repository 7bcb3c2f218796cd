"""relight_b200 — Relight's ray-bound bake passes (direct light, ambient
occlusion, photons + final gather, radiosity form factors + solve) as
sm_100a CUDA kernels behind a C ABI (include/relight_b200.h), with a host
mirror of Relight's scene / mesh / light / lightmap baking API.

Importing the package does not load the CUDA library; `relight_b200.device`
does, and fails loudly if librelight_b200.so is missing.
"""
from .api import (AmbientOcclusionSettings, IndirectLightSettings, Light, LinearLightAttenuation, Lightmap,
                  Material, Mesh, Photonmap, RelightStatus, Scene, Texture, TexturedMaterial)

__all__ = ["AmbientOcclusionSettings", "IndirectLightSettings", "Light", "LinearLightAttenuation", "Lightmap",
           "Material", "Mesh", "Photonmap", "RelightStatus", "Scene", "Texture", "TexturedMaterial"]
