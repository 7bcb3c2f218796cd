// Relight-style C++ program: Mesh::createFromFile, then the mesh's vertex
// positions, normals, lightmap uvs and indices written as raw binary
// (int32 counts, float32 arrays, int32 indices) for the test to compare.
#include <relight/Relight.h>

#include <cstdio>
#include <vector>

using namespace relight;

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    Mesh* mesh = Mesh::createFromFile(argv[1]);
    if (!mesh) return 3;
    FILE* f = fopen(argv[2], "wb");
    if (!f) return 4;
    int nv = mesh->vertexCount(), ni = mesh->indexCount();
    fwrite(&nv, sizeof nv, 1, f);
    fwrite(&ni, sizeof ni, 1, f);
    for (int i = 0; i < nv; i++) {
        const Vertex& v = mesh->vertex(i);
        float a[8] = {v.position.x, v.position.y, v.position.z, v.normal.x,
                      v.normal.y,   v.normal.z,   v.uv[Vertex::Lightmap].x, v.uv[Vertex::Lightmap].y};
        fwrite(a, sizeof(float), 8, f);
    }
    for (int i = 0; i < ni; i++) {
        int idx = mesh->index(i);
        fwrite(&idx, sizeof idx, 1, f);
    }
    fclose(f);
    delete mesh;
    return 0;
}
