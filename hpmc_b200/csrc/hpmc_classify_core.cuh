// hpmc_classify_core.cuh -- the generic base-level classification on sm_100a
// (shadergen.cpp:86-171 fused with the first five reductions): one CTA per
// 32x32 block of the virtual cell grid, for any tiling, pitch or field source.
//
// Included by kernels_build.cu (the library's field types; its TMA column
// classifier shares the helpers) and by include/hpmc_functor.cuh (a caller's
// functor types, instantiated in the caller's own translation unit).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "hpmc_device.cuh"
#include "hpmc_fetch.cuh"
#include "_gen/hpmc_case_tables.h"

namespace hpmc {

// Vertex counts per case (HPMC's tables, generated at build time), one copy
// per translation unit's device module.
static __constant__ uint8_t c_vertex_count[256] = HPMC_GEN_VERTEX_COUNT;

namespace {

// The four codes of a 2x2 quad of cells from the 3-bit sample groups of its
// three rows in the lower (gb) and upper (gt) sample layers; bit
// (dx + 2dy + 4dz) set iff the sample is below iso (shadergen.cpp:132-153).
__device__ __forceinline__ uint32_t quad_codes(const uint32_t gb[3], const uint32_t gt[3], bool vx0,
                                               bool vx1, bool vy0, bool vy1) {
    uint32_t packed = 0;
#pragma unroll
    for (int dy = 0; dy < 2; dy++) {
#pragma unroll
        for (int dx = 0; dx < 2; dx++) {
            uint32_t c = ((gb[dy] >> dx) & 3u) | (((gb[dy + 1] >> dx) & 3u) << 2) |
                         (((gt[dy] >> dx) & 3u) << 4) | (((gt[dy + 1] >> dx) & 3u) << 6);
            const bool valid = (dx ? vx1 : vx0) && (dy ? vy1 : vy0);
            if (!valid) c = 0;  // masked cells (shadergen.cpp:112-125, 163)
            packed |= c << (8 * (dx + 2 * dy));
        }
    }
    return packed;
}

__device__ __forceinline__ void write_codes(const Volume& V, uint32_t packed, int x, int y, int z) {
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int xx = x + (c & 1), yy = y + (c >> 1);
        if (xx < V.cells[0] && yy < V.cells[1])
            V.codes_out[((long long)z * V.cells[1] + yy) * V.cells[0] + xx] = (uint8_t)(packed >> (8 * c));
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Generic classification: CTA = one 32x32 block of the virtual cell grid,
// for any tiling (tiles narrower than 32 cells), unaligned pitches and
// functor fields.  Each thread loads its quad's 3x3x2 samples directly; the
// quads are numbered in Morton order, so thread t's four codes are word t of
// the block's arena slot, and threads 8l .. 8l+7 (one eighth of a warp) hold
// Morton tile l, whose active mask and vertices they combine by shuffles.
template <int FT, class UF = NoUserField>
__device__ __forceinline__ void classify_block_body(const Volume& V, uint64_t b, uint8_t* s_cnt,
                                                    uint32_t* s_warp) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float iso = V.binary ? 0.5f : V.iso;
    int qx, qy;
    morton10((uint32_t)tid, qx, qy);
    const uint32_t X = (morton_compact(b) << 5) + 2u * (uint32_t)qx;
    const uint32_t Y = (morton_compact(b >> 1) << 5) + 2u * (uint32_t)qy;
    int x = 0, y = 0, z = 0;
    uint32_t packed = 0;
    const uint32_t tu = X >> V.wx_l2, tv = Y >> V.wy_l2;
    if (tu < (uint32_t)V.layout_x && tv < (uint32_t)V.layout_y) {
        x = (int)(X & ((1u << V.wx_l2) - 1u));
        y = (int)(Y & ((1u << V.wy_l2) - 1u));
        z = (int)((tv << V.lx_l2) | tu);
        if (z < V.cells[2] && x < V.cells[0] && y < V.cells[1]) {
            uint32_t gb[3], gt[3];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                uint32_t bb = 0, bt = 0;
#pragma unroll
                for (int i = 0; i < 3; i++) {
                    bb |= (uint32_t)(fetch<FT, UF>(V, x + i, y + j, z) < iso) << i;
                    bt |= (uint32_t)(fetch<FT, UF>(V, x + i, y + j, z + 1) < iso) << i;
                }
                gb[j] = bb;
                gt[j] = bt;
            }
            packed = quad_codes(gb, gt, true, x + 1 < V.cells[0], true, y + 1 < V.cells[1]);
            if (V.codes_out) write_codes(V, packed, x, y, z);
        }
    }
    // thread = quad = cells 4 tid .. 4 tid + 3 in Morton order: its vertices
    // and active cells, the tile's by shuffles within its eight lanes, one
    // block reduction for the block's count
    uint32_t vs = 0, nib = 0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const uint32_t n = s_cnt[(packed >> (8 * c)) & 0xffu];
        vs += n;
        nib |= (n ? 1u : 0u) << c;
    }
    uint32_t tmask = nib << (4 * (tid & 7)), tcnt = vs;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
        tmask |= __shfl_xor_sync(0xffffffffu, tmask, o);
        tcnt += __shfl_xor_sync(0xffffffffu, tcnt, o);
    }
    const uint32_t wsum = __reduce_add_sync(0xffffffffu, vs);
    if (lane == 0) s_warp[warp] = wsum;
    __syncthreads();
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kWarps; w++) total += s_warp[w];
    if (tid == 0) V.levels[V.level_off[kBlockLevel] + b] = total;
    if (total) {
        uint32_t* slot = V.arena + block_slot(V, b) * kSlotWords;
        slot[tid] = packed;
        if ((tid & 7) == 0) reinterpret_cast<uint2*>(slot + kSlotTileWord)[tid >> 3] = make_uint2(tmask, tcnt);
    }
    __syncthreads();
}

// UF: a caller's functor type when FT == kFieldUser (include/hpmc_functor.cuh).
template <int FT, class UF = NoUserField>
__global__ void __launch_bounds__(kThreads) classify_blocks(const __grid_constant__ Volume V) {
    __shared__ uint8_t s_cnt[256];
    __shared__ uint32_t s_warp[kWarps];
    s_cnt[threadIdx.x] = c_vertex_count[threadIdx.x];
    __syncthreads();
    for (uint64_t b = blockIdx.x; b < (uint64_t)V.nblocks; b += gridDim.x)
        classify_block_body<FT, UF>(V, b, s_cnt, s_warp);
}

}  // namespace hpmc
