// texture3d.cpp -- headless port of apps/texture3d/texture3d.cpp: iso-surfaces
// of a raw uint8 volume.  The reference uploads the bytes as a GL_ALPHA /
// GL_UNSIGNED_BYTE 3-D texture (read as b/255, GL_CLAMP, NEAREST); here they
// go to a device array registered as an HPMC_SCALAR_UNORM8 field.  Per frame:
// iso = 0.5 + 0.48 cos(t), build, extract, status line (texture3d.cpp:253-289).
//
//   hpmc_texture3d xsize ysize zsize rawfile [--frames N] [--iso X] [--ply out.ply] [--quiet]
#include <fstream>

#include "app_common.hpp"

int main(int argc, char** argv) {
    app::Options o;
    const auto args = app::parse(argc, argv, o);
    if (args.size() != 4) {
        std::fprintf(stderr,
                     "HPMC demo application that extracts iso-surfaces of raw volumes (headless).\n\n"
                     "Usage: %s xsize ysize zsize rawfile [--frames N] [--iso X] [--ply out.ply] [--quiet]\n",
                     argv[0]);
        return EXIT_FAILURE;
    }
    const int sx = std::atoi(args[0].c_str()), sy = std::atoi(args[1].c_str()), sz = std::atoi(args[2].c_str());
    std::vector<unsigned char> dataset((size_t)sx * sy * sz);
    std::ifstream datafile(args[3], std::ios::in | std::ios::binary);
    if (!datafile.good() || !datafile.read(reinterpret_cast<char*>(dataset.data()), dataset.size())) {
        std::fprintf(stderr, "cannot read %zu bytes from %s\n", dataset.size(), args[3].c_str());
        return EXIT_FAILURE;
    }
    // --- upload volume (glTexImage3D in the reference) ---
    unsigned char* d_volume = nullptr;
    app::check(cudaMalloc(&d_volume, dataset.size()), "cudaMalloc volume");
    app::check(cudaMemcpy(d_volume, dataset.data(), dataset.size(), cudaMemcpyHostToDevice), "upload volume");
    const GLuint volume_tex = HPMCregisterDeviceField(d_volume, HPMC_SCALAR_UNORM8, sx, sy, sz, 0, 0);

    // --- create HistoPyramid (texture3d.cpp:143-166) ---
    HPMCConstants* hpmc_c = HPMCcreateConstants(4, 3);
    if (!hpmc_c) {
        std::fprintf(stderr, "HPMCcreateConstants failed (no usable CUDA device)\n");
        return EXIT_FAILURE;
    }
    HPMCHistoPyramid* hpmc_h = HPMCcreateHistoPyramid(hpmc_c);
    HPMCsetLatticeSize(hpmc_h, sx, sy, sz);
    HPMCsetGridSize(hpmc_h, sx - 1, sy - 1, sz - 1);
    const float max_size = (float)std::max(sx, std::max(sy, sz));
    HPMCsetGridExtent(hpmc_h, sx / max_size, sy / max_size, sz / max_size);
    HPMCsetFieldTexture3D(hpmc_h, volume_tex, GL_FALSE);
    HPMCTraversalHandle* th = HPMCcreateTraversalHandle(hpmc_h);
    app::check_hpmc(hpmc_h, "set-up");

    app::Buffers buf;
    unsigned n = 0;
    float iso = 0.f;
    const auto t0 = app::Clock::now();
    for (int frame = 0; frame < o.frames; frame++) {
        const float t = frame / 60.0f;
        iso = o.fixed_iso ? o.iso : 0.5f + 0.48f * cosf(t);
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
    HPMCunregisterDeviceField(volume_tex);
    cudaFree(d_volume);
    return EXIT_SUCCESS;
}
