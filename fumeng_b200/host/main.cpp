// Command-line renderer with the reference's contract (src/cmd/src/main.cpp:13-35):
//   fumeng_b200_cli scene.json
// renders the scene on CUDA device 0 and writes the PNG outputs the scene file names.
#include <cstdio>
#include <string>

#include "../../include/fumeng_b200.h"

int main(int argc, char* argv[])
{
    std::fprintf(stderr, "[fumeng_b200] Fumeng Engine (B200 path-tracing core)\n");
    std::fprintf(stderr, "[fumeng_b200] Using float precision.\n");
    if (argc < 2) {
        std::fprintf(stderr, "[fumeng_b200] Please input the scene file.\n");
        return -1;
    }
    const std::string scene{argv[1]};
    if (scene.find(".json") == std::string::npos) {
        std::fprintf(stderr, "[fumeng_b200] Please specify the correct scene file.\n");
        return -1;
    }
    fm_ctx* ctx = nullptr;
    if (fm_ctx_create(0, &ctx) != FM_OK) {
        std::fprintf(stderr, "[fumeng_b200] No usable CUDA device.\n");
        return -1;
    }
    const fm_status st = fm_draw_frame(ctx, scene.c_str());
    if (st != FM_OK) std::fprintf(stderr, "[fumeng_b200] Unexpected error: %s\n", fm_last_error(ctx));
    fm_ctx_destroy(ctx);
    return st == FM_OK ? 0 : -1;
}
