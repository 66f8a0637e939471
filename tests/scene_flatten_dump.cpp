// Test driver: loads a scene file with the library's SceneLoader (the JSON schema of the
// reference, meshes from OBJ files) and writes the flattened arrays it would pass to
// fm_scene_create, as records (name, element size, count, raw bytes), or prints
// "error: <message>" when loading throws.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "fm_scene_loader.h"

template <class T>
static void put(std::FILE* f, const char* name, const std::vector<T>& v)
{
    char tag[16] = {0};
    std::strncpy(tag, name, 15);
    const uint64_t es = sizeof(T), n = v.size();
    std::fwrite(tag, 1, 16, f);
    std::fwrite(&es, 8, 1, f);
    std::fwrite(&n, 8, 1, f);
    if (n) std::fwrite(v.data(), sizeof(T), n, f);
}

int main(int argc, char** argv)
{
    if (argc != 3) return 2;
    try {
        fmhost::SceneLoader L;
        L.Load(argv[1]);
        const fmhost::FlatScene& F = L.flat();
        std::FILE* f = std::fopen(argv[2], "wb");
        if (!f) return 3;
        put(f, "obj_material", F.obj_material);
        put(f, "obj_emission", F.obj_emission);
        put(f, "tri_pos", F.tri_pos);
        put(f, "tri_normal", F.tri_normal);
        put(f, "tri_uv", F.tri_uv);
        put(f, "tri_has_normal", F.tri_has_normal);
        put(f, "tri_object", F.tri_object);
        put(f, "rect_pts", F.rect_pts);
        put(f, "rect_object", F.rect_object);
        put(f, "sphere_radius", F.sphere_radius);
        put(f, "sphere_xform", F.sphere_xform);
        put(f, "sphere_object", F.sphere_object);
        std::fclose(f);
        std::printf("ok\n");
    } catch (const std::exception& e) {
        std::printf("error: %s\n", e.what());
    }
    return 0;
}
