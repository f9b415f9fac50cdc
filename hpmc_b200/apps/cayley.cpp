// cayley.cpp -- headless port of apps/cayley/cayley.cpp: the Cayley cubic
// 1 - 16xyz - 4x^2 - 4y^2 - 4z^2 (p mapped to [-1,1]^3) evaluated by a field
// functor instead of texture reads.  The reference hands HPMCsetFieldCustom a
// GLSL HPMC_fetch / HPMC_fetchGrad snippet (cayley.cpp:75-94) and treats the
// field as binary (cayley.cpp:171-173); here the snippet is the registered
// functor "hpmc:cayley".  Per frame: iso = sin(t), build, extract.
//
//   hpmc_cayley [size | xsize ysize zsize] [--continuous] [--frames N] [--iso X] [--ply out.ply] [--quiet]
#include "app_common.hpp"

int main(int argc, char** argv) {
    app::Options o;
    bool continuous = false;
    std::vector<char*> rest{argv[0]};
    for (int i = 1; i < argc; i++) {
        if (std::strcmp(argv[i], "--continuous") == 0) continuous = true;
        else rest.push_back(argv[i]);
    }
    const auto args = app::parse((int)rest.size(), rest.data(), o);
    int sx = 64, sy = 64, sz = 64;  // cayley.cpp:319-323
    if (args.size() == 1) {
        sx = sy = sz = std::atoi(args[0].c_str());
    } else if (args.size() == 3) {
        sx = std::atoi(args[0].c_str());
        sy = std::atoi(args[1].c_str());
        sz = std::atoi(args[2].c_str());
    } else if (!args.empty()) {
        std::fprintf(stderr, "Usage: %s [size | xsize ysize zsize] [--continuous] [--frames N] [--iso X] "
                             "[--ply out.ply] [--quiet]\n", argv[0]);
        return EXIT_FAILURE;
    }
    HPMCConstants* hpmc_c = HPMCcreateConstants(4, 3);
    if (!hpmc_c) {
        std::fprintf(stderr, "HPMCcreateConstants failed (no usable CUDA device)\n");
        return EXIT_FAILURE;
    }
    // --- create HistoPyramid (cayley.cpp:147-175) ---
    HPMCHistoPyramid* hpmc_h = HPMCcreateHistoPyramid(hpmc_c);
    HPMCsetLatticeSize(hpmc_h, sx, sy, sz);
    HPMCsetGridSize(hpmc_h, sx - 1, sy - 1, sz - 1);
    HPMCsetGridExtent(hpmc_h, 1.0f, 1.0f, 1.0f);
    HPMCsetFieldCustom(hpmc_h, "hpmc:cayley", 0, GL_TRUE);
    if (!continuous) HPMCsetFieldAsBinary(hpmc_h);
    HPMCTraversalHandle* th = HPMCcreateTraversalHandle(hpmc_h);
    app::check_hpmc(hpmc_h, "set-up");

    app::Buffers buf;
    unsigned n = 0;
    float iso = 0.f;
    const auto t0 = app::Clock::now();
    for (int frame = 0; frame < o.frames; frame++) {
        const float t = frame / 60.0f;
        iso = o.fixed_iso ? o.iso : sinf(t);
        HPMCbuildHistopyramid(hpmc_h, iso);
        n = HPMCacquireNumberOfVertices(hpmc_h);
        buf.ensure(n);
        HPMCsetTraversalHandleBuffers(th, buf.pos, buf.nrm, buf.cap);
        if (n && !HPMCextractVertices(th)) app::check_hpmc(hpmc_h, "HPMCextractVertices");
    }
    app::check(cudaDeviceSynchronize(), "frames");
    const double dt = app::seconds(t0, app::Clock::now());
    if (!o.quiet) app::report(o.frames / dt, sx, sy, sz, n, iso);
    app::save_float4(o, buf, n);
    std::printf("vertices %u\n", n);
    HPMCdestroyTraversalHandle(th);
    HPMCdestroyHandle(hpmc_h);
    HPMCdestroyConstants(hpmc_c);
    return EXIT_SUCCESS;
}
