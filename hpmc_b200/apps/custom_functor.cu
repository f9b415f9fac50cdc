// custom_functor.cu -- a caller that brings its own field functor.
//
// The reference's applications hand HPMCsetFieldCustom a GLSL HPMC_fetch /
// HPMC_fetchGrad snippet of their own (e.g. apps/cayley/cayley.cpp:75-94).
// This example does the same with a CUDA functor type compiled in this file:
// include/hpmc_functor.cuh instantiates the library's classification and
// traversal kernels for the type here, HPMCregisterFieldFunctor makes the
// name "app:torus" valid for HPMCsetFieldCustom, and the two parameters
// (major and minor radius) are set with HPMCgetBuilderProgram /
// HPMCsetBuilderUniforms as an application sets its snippet's uniforms.
//
//   hpmc_custom_functor [size | xsize ysize zsize] [--gradient] [--central] [--radii R r]
//                       [--frames N] [--iso X] [--ply out.ply] [--quiet]
#include <cuda_runtime.h>

#include "app_common.hpp"
#include "hpmc_functor.cuh"

namespace {

// (sqrt(x^2 + y^2) - R)^2 + z^2 - r^2 with (x, y, z) = 2p - 1: a torus around
// the z axis.  Round-to-nearest intrinsics in a fixed order, so that a plain
// FP32 restatement on the host gives the same values bit for bit.
struct Torus {
    static constexpr bool kHasGradient = true;

    __device__ static float value(const float* prm, int /*count*/, float px, float py, float pz) {
        const float x = __fsub_rn(__fmul_rn(2.0f, px), 1.0f);
        const float y = __fsub_rn(__fmul_rn(2.0f, py), 1.0f);
        const float z = __fsub_rn(__fmul_rn(2.0f, pz), 1.0f);
        const float d = __fsub_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y))), prm[0]);
        return __fsub_rn(__fadd_rn(__fmul_rn(d, d), __fmul_rn(z, z)), __fmul_rn(prm[1], prm[1]));
    }

    // in the functor's own coordinates (x = 2p - 1), as HPMC_fetchGrad returns them
    __device__ static void gradient(const float* prm, int /*count*/, float px, float py, float pz, float g[3]) {
        const float x = __fsub_rn(__fmul_rn(2.0f, px), 1.0f);
        const float y = __fsub_rn(__fmul_rn(2.0f, py), 1.0f);
        const float z = __fsub_rn(__fmul_rn(2.0f, pz), 1.0f);
        const float q = __fsqrt_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)));
        const float d = __fsub_rn(q, prm[0]);
        g[0] = __fdiv_rn(__fmul_rn(__fmul_rn(2.0f, d), x), q);
        g[1] = __fdiv_rn(__fmul_rn(__fmul_rn(2.0f, d), y), q);
        g[2] = __fmul_rn(2.0f, z);
    }
};

}  // namespace

HPMC_FIELD_FUNCTOR(torus_ops, Torus);

int main(int argc, char** argv) {
    app::Options o;
    bool gradient = false, central = false;
    float radii[2] = {0.5f, 0.25f};
    std::vector<char*> rest{argv[0]};
    for (int i = 1; i < argc; i++) {
        if (std::strcmp(argv[i], "--gradient") == 0) gradient = true;
        else if (std::strcmp(argv[i], "--central") == 0) central = true;
        else if (std::strcmp(argv[i], "--radii") == 0 && i + 2 < argc) {
            radii[0] = (float)std::atof(argv[++i]);
            radii[1] = (float)std::atof(argv[++i]);
        } else rest.push_back(argv[i]);
    }
    const auto args = app::parse((int)rest.size(), rest.data(), o);
    int sx = 64, sy = 64, sz = 64;
    if (args.size() == 1) {
        sx = sy = sz = std::atoi(args[0].c_str());
    } else if (args.size() == 3) {
        sx = std::atoi(args[0].c_str());
        sy = std::atoi(args[1].c_str());
        sz = std::atoi(args[2].c_str());
    } else if (!args.empty()) {
        std::fprintf(stderr, "Usage: %s [size | xsize ysize zsize] [--gradient] [--central] [--radii R r] "
                             "[--frames N] [--iso X] [--ply out.ply] [--quiet]\n", argv[0]);
        return EXIT_FAILURE;
    }
    if (HPMCregisterFieldFunctor("app:torus", &torus_ops) != HPMC_OK) {
        std::fprintf(stderr, "HPMCregisterFieldFunctor refused the table\n");
        return EXIT_FAILURE;
    }
    HPMCConstants* c = HPMCcreateConstants(4, 3);
    if (!c) {
        std::fprintf(stderr, "HPMCcreateConstants failed (no usable CUDA device)\n");
        return EXIT_FAILURE;
    }
    HPMCHistoPyramid* h = HPMCcreateHistoPyramid(c);
    HPMCsetLatticeSize(h, sx, sy, sz);
    HPMCsetGridSize(h, sx - 1, sy - 1, sz - 1);
    HPMCsetGridExtent(h, 1.0f, 1.0f, 1.0f);
    HPMCsetFieldCustom(h, "app:torus", 0, gradient ? GL_TRUE : GL_FALSE);
    HPMCsetNormalMode(h, central ? HPMC_NORMALS_CENTRAL : HPMC_NORMALS_FORWARD);
    if (HPMCgetBuilderProgram(h) == 0) app::check_hpmc(h, "HPMCgetBuilderProgram");
    HPMCsetBuilderUniforms(h, radii, 2);
    HPMCTraversalHandle* th = HPMCcreateTraversalHandle(h);
    app::check_hpmc(h, "set-up");

    app::Buffers buf;
    unsigned n = 0;
    float iso = 0.f;
    const auto t0 = app::Clock::now();
    for (int frame = 0; frame < o.frames; frame++) {
        // the minor radius breathes with the iso-value (iso shifts f by a constant)
        iso = o.fixed_iso ? o.iso : 0.02f * sinf(frame / 60.0f);
        HPMCbuildHistopyramid(h, iso);
        n = HPMCacquireNumberOfVertices(h);
        buf.ensure(n);
        HPMCsetTraversalHandleBuffers(th, buf.pos, buf.nrm, buf.cap);
        if (n && !HPMCextractVertices(th)) app::check_hpmc(h, "HPMCextractVertices");
    }
    app::check(cudaDeviceSynchronize(), "frames");
    const double dt = app::seconds(t0, app::Clock::now());
    if (!o.quiet) app::report(o.frames / dt, sx, sy, sz, n, iso);
    app::save_float4(o, buf, n);
    std::printf("vertices %u\n", n);
    HPMCdestroyTraversalHandle(th);
    HPMCdestroyHandle(h);
    HPMCdestroyConstants(c);
    HPMCunregisterFieldFunctor("app:torus");
    return EXIT_SUCCESS;
}
