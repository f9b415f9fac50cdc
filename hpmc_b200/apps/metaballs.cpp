// metaballs.cpp -- headless port of apps/metaballs/metaballs.cpp: eight
// metaballs in a twisted domain, moving over time.  The reference passes a
// GLSL fetch snippet with uniforms `twist` and `centers[8]`
// (metaballs.cpp:72-94) and sets them on HPMCgetBuilderProgram's program every
// frame (metaballs.cpp:268-281); here the functor "hpmc:twist_metaballs" takes
// the same values through HPMCsetBuilderUniforms {twist, c0.xyz, ..., c7.xyz}.
// iso = 10 (metaballs.cpp:294).
//
//   hpmc_metaballs [size | xsize ysize zsize] [--frames N] [--iso X] [--ply out.ply] [--quiet]
#include "app_common.hpp"

int main(int argc, char** argv) {
    app::Options o;
    const auto args = app::parse(argc, argv, o);
    int sx = 64, sy = 64, sz = 64;
    if (args.size() == 1) {
        sx = sy = sz = std::atoi(args[0].c_str());
    } else if (args.size() == 3) {
        sx = std::atoi(args[0].c_str());
        sy = std::atoi(args[1].c_str());
        sz = std::atoi(args[2].c_str());
    } else if (!args.empty()) {
        std::fprintf(stderr, "Usage: %s [size | xsize ysize zsize] [--frames N] [--iso X] [--ply out.ply] "
                             "[--quiet]\n", argv[0]);
        return EXIT_FAILURE;
    }
    HPMCConstants* hpmc_c = HPMCcreateConstants(4, 3);
    if (!hpmc_c) {
        std::fprintf(stderr, "HPMCcreateConstants failed (no usable CUDA device)\n");
        return EXIT_FAILURE;
    }
    // --- create HistoPyramid (metaballs.cpp:141-165) ---
    HPMCHistoPyramid* hpmc_h = HPMCcreateHistoPyramid(hpmc_c);
    HPMCsetLatticeSize(hpmc_h, sx, sy, sz);
    HPMCsetGridSize(hpmc_h, sx - 1, sy - 1, sz - 1);
    HPMCsetGridExtent(hpmc_h, 1.0f, 1.0f, 1.0f);
    HPMCsetFieldCustom(hpmc_h, "hpmc:twist_metaballs", 0, GL_FALSE);
    HPMCTraversalHandle* th = HPMCcreateTraversalHandle(hpmc_h);
    app::check_hpmc(hpmc_h, "set-up");

    app::Buffers buf;
    unsigned n = 0;
    float iso = 10.0f;
    const auto t0 = app::Clock::now();
    for (int frame = 0; frame < o.frames; frame++) {
        const double t = frame / 60.0;
        // --- update metaballs position (metaballs.cpp:268-276) ---
        float uniforms[1 + 3 * 8];
        uniforms[0] = (float)(5.0 * sin(0.1 * t));
        for (int i = 0; i < 8; i++) {
            uniforms[1 + 3 * i + 0] = (float)(0.5 + 0.3 * sin(t + sin(0.1 * t) * i));
            uniforms[1 + 3 * i + 1] = (float)(0.5 + 0.3 * cos(0.9 * t + sin(0.1 * t) * i));
            uniforms[1 + 3 * i + 2] = (float)(0.5 + 0.3 * cos(0.7 * t + sin(0.01 * t) * i));
        }
        if (HPMCgetBuilderProgram(hpmc_h) == 0) app::check_hpmc(hpmc_h, "HPMCgetBuilderProgram");
        if (HPMCsetBuilderUniforms(hpmc_h, uniforms, 1 + 3 * 8) != HPMC_OK) app::check_hpmc(hpmc_h, "uniforms");
        iso = o.fixed_iso ? o.iso : 10.0f;
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
