// transform_feedback.cpp -- headless port of
// apps/transform_feedback/transform_feedback.cpp: the Cayley cubic (continuous
// field, functor with gradient) extracted by transform-feedback capture into an
// interleaved N3F_V3F buffer that grows to 1.1x the vertex count when too
// small (transform_feedback.cpp:384-431).  The GL buffer object becomes a
// device buffer bound with HPMCsetTraversalHandleFeedbackBuffer; the capture
// call is the same.  Per frame: iso = sin(t).
//
//   hpmc_transform_feedback [size | xsize ysize zsize] [--frames N] [--iso X] [--ply out.ply] [--quiet]
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
    // --- create HistoPyramid (transform_feedback.cpp:206-231) ---
    HPMCHistoPyramid* hpmc_h = HPMCcreateHistoPyramid(hpmc_c);
    HPMCsetLatticeSize(hpmc_h, sx, sy, sz);
    HPMCsetGridSize(hpmc_h, sx - 1, sy - 1, sz - 1);
    HPMCsetGridExtent(hpmc_h, 1.0f, 1.0f, 1.0f);
    HPMCsetFieldCustom(hpmc_h, "hpmc:cayley", 0, GL_TRUE);
    HPMCTraversalHandle* hpmc_th_flat = HPMCcreateTraversalHandle(hpmc_h);
    app::check_hpmc(hpmc_h, "set-up");

    float* mc_tri_vbo = nullptr;  // N3F_V3F
    unsigned mc_tri_vbo_N = 0;
    unsigned N = 0;
    float iso = 0.f;
    const auto t0 = app::Clock::now();
    for (int frame = 0; frame < o.frames; frame++) {
        const float t = frame / 60.0f;
        iso = o.fixed_iso ? o.iso : sinf(t);
        HPMCbuildHistopyramid(hpmc_h, iso);
        N = HPMCacquireNumberOfVertices(hpmc_h);
        if (mc_tri_vbo_N < N) {  // resize buffer if needed
            mc_tri_vbo_N = (unsigned)(1.1f * (float)N);
            if (!o.quiet) std::fprintf(stderr, "resizing mc_tri_vbo to hold %u vertices.\n", mc_tri_vbo_N);
            cudaFree(mc_tri_vbo);
            app::check(cudaMalloc(&mc_tri_vbo, (3 + 3) * sizeof(float) * (size_t)mc_tri_vbo_N), "cudaMalloc vbo");
            HPMCsetTraversalHandleFeedbackBuffer(hpmc_th_flat, mc_tri_vbo, mc_tri_vbo_N);
        }
        if (N && !HPMCextractVerticesTransformFeedback(hpmc_th_flat))
            app::check_hpmc(hpmc_h, "HPMCextractVerticesTransformFeedback");
    }
    app::check(cudaDeviceSynchronize(), "frames");
    const double dt = app::seconds(t0, app::Clock::now());
    if (!o.quiet) app::report(o.frames / dt, sx, sy, sz, N, iso);
    if (!o.ply.empty()) {
        std::vector<float> v(6 * (size_t)N);
        app::check(cudaMemcpy(v.data(), mc_tri_vbo, sizeof(float) * v.size(), cudaMemcpyDeviceToHost), "copy vbo");
        if (!app::write_ply(o.ply, v.data() + 3, v.data(), N, 6, 6)) return EXIT_FAILURE;
    }
    std::printf("vertices %u\n", N);
    cudaFree(mc_tri_vbo);
    HPMCdestroyTraversalHandle(hpmc_th_flat);
    HPMCdestroyHandle(hpmc_h);
    HPMCdestroyConstants(hpmc_c);
    return EXIT_SUCCESS;
}
