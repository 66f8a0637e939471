// Test driver: reads an OBJ file with the library's reader (fmhost::load_obj) and writes
// what it read as text (counts, then v, vt, vn values with %.9g, then face corners), or
// "error: <message>" when the reader throws.
#include <cstdio>
#include <stdexcept>

#include "fm_scene_loader.h"

int main(int argc, char** argv)
{
    if (argc != 2) return 2;
    try {
        const fmhost::ObjData o = fmhost::load_obj(argv[1]);
        std::printf("%zu %zu %zu %zu\n", o.v.size(), o.vt.size(), o.vn.size(), o.faces.size());
        for (const auto* arr : {&o.v, &o.vt, &o.vn}) {
            for (float x : *arr) std::printf("%.9g ", x);
            std::printf("\n");
        }
        for (const auto& f : o.faces)
            for (const auto& c : f) std::printf("%d %d %d ", c.v, c.vt, c.vn);
        std::printf("\n");
    } catch (const std::exception& e) {
        std::printf("error: %s\n", e.what());
    }
    return 0;
}
