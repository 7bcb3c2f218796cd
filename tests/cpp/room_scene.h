// The scene of the C++ example programs: a closed 10^3 room (grey) with a
// red crate, both in one 64x64 lightmap and photonmap; a point light, a spot
// light and a 2-triangle area light.  Built through relight::Relight's own
// scene API, as a Relight program would.
#ifndef RELIGHT_B200_TEST_ROOM_SCENE_H
#define RELIGHT_B200_TEST_ROOM_SCENE_H

#include <relight/Relight.h>

#include <cstdio>
#include <string>

namespace room_example {

using namespace relight;

static void quad(VertexBuffer& vb, IndexBuffer& ib, Vec3 p0, Vec3 p1, Vec3 p2, Vec3 p3, Vec3 n, float u0, float v0,
                 float u1, float v1) {
    Index base = (Index)vb.size();
    Vec3 ps[4] = {p0, p1, p2, p3};
    Uv uvs[4] = {Uv(u0, v0), Uv(u1, v0), Uv(u1, v1), Uv(u0, v1)};
    for (int k = 0; k < 4; k++) {
        Vertex v;
        v.position = ps[k];
        v.normal = n;
        v.uv[Vertex::Lightmap] = uvs[k];
        vb.push_back(v);
    }
    Index idx[6] = {0, 1, 2, 0, 2, 3};
    for (Index i : idx) ib.push_back((Index)(base + i));
}

// An axis-aligned box: lo/hi corners, inward or outward normals, chart cells
// starting at `cell` in a 4x4 grid of the unit uv square.
static void box(VertexBuffer& vb, IndexBuffer& ib, Vec3 lo, Vec3 hi, bool inward, int cell) {
    for (int axis = 0; axis < 3; axis++) {
        int i = (axis + 1) % 3, j = (axis + 2) % 3;
        for (int side = 0; side < 2; side++) {
            float c = side ? (&hi.x)[axis] : (&lo.x)[axis];
            Vec3 n;
            (&n.x)[axis] = (side ? 1.0f : -1.0f) * (inward ? -1.0f : 1.0f);
            Vec3 p[4];
            int ab[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
            for (int k = 0; k < 4; k++) {
                (&p[k].x)[axis] = c;
                (&p[k].x)[i] = ab[k][0] ? (&hi.x)[i] : (&lo.x)[i];
                (&p[k].x)[j] = ab[k][1] ? (&hi.x)[j] : (&lo.x)[j];
            }
            int cx = cell % 4, cy = cell / 4;
            cell++;
            quad(vb, ib, p[0], p[1], p[2], p[3], n, (cx * 16 + 1) / 64.0f, (cy * 16 + 1) / 64.0f,
                 (cx * 16 + 15) / 64.0f, (cy * 16 + 15) / 64.0f);
        }
    }
}

static bool dump(Lightmap* lm, const std::string& path) {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) return false;
    Lumel* l = lm->lumels();
    int n = lm->width() * lm->height();
    for (int i = 0; i < n; i++) fwrite(&l[i].m_flags, sizeof(int), 1, f);
    for (int i = 0; i < n; i++) fwrite(&l[i].m_color, sizeof(float), 3, f);
    fclose(f);
    return true;
}

struct RoomScene {
    Relight* relight;
    Scene* scene;
    Mesh* room;
    Mesh* crate;
    Lightmap* lightmap;
    Photonmap* photonmap;
};

// Returns false if Scene::end fails.
static bool build_room(RoomScene& out) {
    Relight* relight = Relight::create();
    Scene* scene = relight->createScene();
    scene->begin();

    Material* grey = new Material(Rgb(0.7f, 0.7f, 0.7f));
    Material* red = new Material(Rgb(0.8f, 0.2f, 0.2f));
    VertexBuffer vb;
    IndexBuffer ib;
    box(vb, ib, Vec3(0, 0, 0), Vec3(10, 10, 10), true, 0);
    Mesh* room = Mesh::create();
    room->addFaces(vb, ib, grey);
    vb.clear();
    ib.clear();
    box(vb, ib, Vec3(3, 0, 4), Vec3(6, 3, 6), false, 6);
    Mesh* crate = Mesh::create();
    crate->addFaces(vb, ib, red);

    Mesh* r = scene->addMesh(room, Matrix4());
    Mesh* c = scene->addMesh(crate, Matrix4());
    Lightmap* lm = relight->createLightmap(64, 64);
    Photonmap* pm = relight->createPhotonmap(64, 64);
    lm->addMesh(r); lm->addMesh(c);
    pm->addMesh(r); pm->addMesh(c);

    scene->addLight(Light::createPointLight(Vec3(5, 9, 5), 10.0f, Rgb(1, 1, 1), 1.0f));
    scene->addLight(Light::createSpotLight(Vec3(2, 8, 2), Vec3(0.5f, -0.7f, 0.5f), 0.9238795f, 10.0f,
                                           Rgb(1.0f, 0.9f, 0.7f), 1.0f));
    VertexBuffer lv;
    IndexBuffer li;
    quad(lv, li, Vec3(-0.5f, 0, -0.5f), Vec3(0.5f, 0, -0.5f), Vec3(0.5f, 0, 0.5f), Vec3(-0.5f, 0, 0.5f),
         Vec3(0, -1, 0), 0, 0, 1, 1);
    Mesh* lightMesh = Mesh::create();
    lightMesh->addFaces(lv, li);
    Light* area = Light::createAreaLight(lightMesh, Vec3(7, 9, 7), Rgb(0.8f, 0.9f, 1.0f), 1.0f);
    area->setAttenuation(new LinearLightAttenuation(area, 10.0f));
    scene->addLight(area);
    if (scene->end() != RelightSuccess) return false;

    out.relight = relight;
    out.scene = scene;
    out.room = r;
    out.crate = c;
    out.lightmap = lm;
    out.photonmap = pm;
    return true;
}

}  // namespace room_example

#endif
