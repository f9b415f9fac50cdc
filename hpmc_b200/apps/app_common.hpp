// app_common.hpp -- shared bits of the headless caller ports: options, the
// reference apps' status line, device buffers and .ply output.
//
// The reference apps (apps/*/ in the HPMC tree) draw with GL/GLUT; these ports
// keep their HPMC call sequences and per-frame iso-value schedules, replace the
// GL program and draw with device output buffers, and print the same status
// line ("fps, samples, mvps, triangles, iso").
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "hpmc.h"

namespace app {

struct Options {
    int frames = 10;         // frames to run (time t advances by 1/60 s per frame)
    bool fixed_iso = false;  // --iso X: use X in every frame instead of the app's schedule
    float iso = 0.f;
    std::string ply;         // --ply PATH: write the last frame's vertices
    bool quiet = false;
};

// Parses the trailing options; returns the positional arguments.
inline std::vector<std::string> parse(int argc, char** argv, Options& o) {
    std::vector<std::string> pos;
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        if (a == "--frames" && i + 1 < argc) o.frames = std::atoi(argv[++i]);
        else if (a == "--iso" && i + 1 < argc) {
            o.fixed_iso = true;
            o.iso = (float)std::atof(argv[++i]);
        } else if (a == "--ply" && i + 1 < argc) o.ply = argv[++i];
        else if (a == "--quiet") o.quiet = true;
        else pos.push_back(a);
    }
    return pos;
}

inline void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
        std::exit(EXIT_FAILURE);
    }
}

inline void check_hpmc(HPMCHistoPyramid* h, const char* what) {
    const int st = HPMCgetLastError(h);
    if (st != HPMC_OK) {
        std::fprintf(stderr, "%s: HPMC status %d\n", what, st);
        std::exit(EXIT_FAILURE);
    }
}

// The reference apps' status line (e.g. apps/texture3d/texture3d.cpp:279-289).
inline void report(double fps, int sx, int sy, int sz, unsigned vertices, float iso) {
    std::printf("%.1f fps, %dx%dx%d samples, %d mvps, %u triangles, iso=%.2f\n", fps, sx, sy, sz,
                (int)(((double)(sx - 1) * (sy - 1) * (sz - 1) * fps) / 1e6), vertices / 3, iso);
}

// Binary little-endian .ply of n vertices given as separate xyz(w) streams
// (stride in floats), three consecutive vertices per triangle.
inline bool write_ply(const std::string& path, const float* pos, const float* nrm, size_t n, int stride_pos,
                      int stride_nrm) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    std::fprintf(f,
                 "ply\nformat binary_little_endian 1.0\nelement vertex %zu\nproperty float x\nproperty float y\n"
                 "property float z\nproperty float nx\nproperty float ny\nproperty float nz\nelement face %zu\n"
                 "property list uchar int vertex_indices\nend_header\n",
                 n, n / 3);
    for (size_t i = 0; i < n; i++) {
        const float v[6] = {pos[i * stride_pos], pos[i * stride_pos + 1], pos[i * stride_pos + 2],
                            nrm[i * stride_nrm], nrm[i * stride_nrm + 1], nrm[i * stride_nrm + 2]};
        std::fwrite(v, sizeof v, 1, f);
    }
    for (size_t t = 0; t < n / 3; t++) {
        const unsigned char three = 3;
        const int idx[3] = {(int)(3 * t), (int)(3 * t + 1), (int)(3 * t + 2)};
        std::fwrite(&three, 1, 1, f);
        std::fwrite(idx, sizeof idx, 1, f);
    }
    std::fclose(f);
    return true;
}

// Device float4 position/normal buffers that grow with the vertex count
// (the reference apps draw straight from the pyramid instead).
struct Buffers {
    float* pos = nullptr;
    float* nrm = nullptr;
    size_t cap = 0;
    void ensure(size_t n) {
        if (n <= cap) return;
        cudaFree(pos);
        cudaFree(nrm);
        cap = n + n / 4 + 1024;
        check(cudaMalloc(&pos, 16 * cap), "cudaMalloc positions");
        check(cudaMalloc(&nrm, 16 * cap), "cudaMalloc normals");
    }
    ~Buffers() {
        cudaFree(pos);
        cudaFree(nrm);
    }
};

// Copies the last frame's float4 streams to the host and writes them.
inline void save_float4(const Options& o, const Buffers& b, unsigned n) {
    if (o.ply.empty()) return;
    std::vector<float> p(4 * (size_t)n), q(4 * (size_t)n);
    check(cudaMemcpy(p.data(), b.pos, 16 * (size_t)n, cudaMemcpyDeviceToHost), "copy positions");
    check(cudaMemcpy(q.data(), b.nrm, 16 * (size_t)n, cudaMemcpyDeviceToHost), "copy normals");
    if (!write_ply(o.ply, p.data(), q.data(), n, 4, 4)) {
        std::fprintf(stderr, "cannot write %s\n", o.ply.c_str());
        std::exit(EXIT_FAILURE);
    }
}

using Clock = std::chrono::steady_clock;

inline double seconds(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
}

}  // namespace app
