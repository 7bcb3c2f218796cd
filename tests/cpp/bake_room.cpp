// A Relight-style C++ program (the scene comes from room_scene.h): builds a closed
// room with a box, a point, a spot and a 2-triangle area light, bakes direct
// light, AO, photons and the final gather through relight::Relight, and
// writes the lightmap (flags + RGB) after AO and after the final gather.
//
//   bake_room <out-prefix>    -> <out-prefix>.direct_ao.bin, <out-prefix>.final.bin
#include "room_scene.h"

using namespace relight;
using namespace room_example;

int main(int argc, char** argv) {
    std::string out = argc > 1 ? argv[1] : "bake_room";
    RoomScene rs;
    if (!build_room(rs)) return 2;
    Relight* relight = rs.relight;
    Scene* scene = rs.scene;
    Mesh* r = rs.room;
    Lightmap* lm = rs.lightmap;
    if (relight->bakeDirectLight(scene, r, nullptr) != RelightSuccess) return 3;
    AmbientOcclusionSettings ao = AmbientOcclusionSettings::draft(0.8f, 2.0f);
    ao.m_samples = 16;
    if (relight->bakeAmbientOcclusion(scene, r, nullptr, ao) != RelightSuccess) return 4;
    if (!dump(lm, out + ".direct_ao.bin")) return 5;
    IndirectLightSettings ind = IndirectLightSettings::draft(Rgb(0.2f, 0.2f, 0.3f), Rgb(0, 0, 0), 20.0f, 20.0f);
    ind.m_photonPassCount = 1;
    ind.m_finalGatherSamples = 16;
    if (relight->emitPhotons(scene, ind) != RelightSuccess) {
        fprintf(stderr, "emitPhotons: %s\n", relight->lastError().c_str());
        return 6;
    }
    if (relight->bakeIndirectLight(scene, r, nullptr, ind) != RelightSuccess) {
        fprintf(stderr, "bakeIndirectLight: %s\n", relight->lastError().c_str());
        return 7;
    }
    if (!dump(lm, out + ".final.bin")) return 8;
    printf("bake_room ok: %s\n", out.c_str());
    return 0;
}
