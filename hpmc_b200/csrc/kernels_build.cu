// kernels_build.cu -- HistoPyramid build on sm_100a: classification fused
// with the first five reductions, then the upper reductions.
//
// Reference passes replaced (hpmc/src/buildpass.cpp:42-178):
//   base level  (shadergen.cpp:86-171)  -> classify_column_tma / classify_blocks
//   first reduction + 4 upper levels    -> fused into classification (a 32x32
//                                          cell block = 4^5 keys is summed in
//                                          registers and warp reductions)
//   remaining upper reductions          -> reduce_levels (one launch,
//                                          last-block-done chaining)
//   top readback (buildpass.cpp:161-168)-> Ctrl::total in device memory
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "hpmc_device.cuh"
#include "hpmc_fetch.cuh"
#include "hpmc_kernels.h"
#include "hpmc_tma.cuh"
#include "_gen/hpmc_case_tables.h"

namespace hpmc {

__constant__ uint8_t c_vertex_count[256] = HPMC_GEN_VERTEX_COUNT;

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

__device__ __forceinline__ uint32_t quad_count(const uint8_t* s_cnt, uint32_t packed) {
    return (uint32_t)s_cnt[packed & 0xffu] + s_cnt[(packed >> 8) & 0xffu] + s_cnt[(packed >> 16) & 0xffu] +
           s_cnt[packed >> 24];
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
// Column classification: CTA = one 32x32 cell footprint of the slice tiles,
// streaming kColumnSlices slices through a TMA ring of sample layers.  Each
// sample is fetched from HBM once (layer halo rows/columns are shared with
// the neighbouring CTAs through L2).  Layer values become one bit per sample
// (f < iso) in shared memory; every thread then forms the codes of one 2x2
// quad of cells, counts them and the CTA sums 1024 cells into one level-5
// entry.  Non-empty blocks store their codes in the arena.
template <int FT>
__global__ void __launch_bounds__(kThreads) classify_column_tma(const __grid_constant__ CUtensorMap tmap,
                                                                const __grid_constant__ Volume V) {
    using T = typename std::conditional<FT == kFieldF32, float, uint8_t>::type;
    constexpr int BXE = (FT == kFieldF32) ? 36 : 48;       // box width (16-byte multiple)
    constexpr int STAGE_BYTES = BXE * 33 * (int)sizeof(T);  // one sample layer
    constexpr int STAGE_STRIDE = (STAGE_BYTES + 127) & ~127;

    extern __shared__ __align__(128) uint8_t s_dyn[];
    // TMA destinations must be 128-byte aligned: align the ring explicitly
    // (the launch reserves 128 spare bytes)
    uint8_t* const s_ring = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(s_dyn) + 127) & ~uintptr_t(127));
    __shared__ __align__(8) uint64_t s_bar[kRingStages];
    __shared__ uint64_t s_rows[3][33];
    __shared__ uint32_t s_warp[2][kWarps];
    __shared__ uint8_t s_cnt[256];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int fx = blockIdx.x, fy = blockIdx.y;
    const int x0 = fx * 32, y0 = fy * 32;
    const int z0 = blockIdx.z * kColumnSlices;
    const int z1 = min(V.cells[2], z0 + kColumnSlices);
    const int nlayers = z1 - z0 + 1;
    const float iso = V.binary ? 0.5f : V.iso;

    s_cnt[tid] = c_vertex_count[tid];
    if (tid == 0) {
        for (int s = 0; s < kRingStages; s++) mbar_init(&s_bar[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (tid == 0) {
        for (int s = 0; s < kRingStages && s < nlayers; s++) {
            mbar_arrive_expect_tx(&s_bar[s], STAGE_BYTES);
            tma_load_3d(s_ring + s * STAGE_STRIDE, &tmap, x0, y0, z0 + s, &s_bar[s]);
        }
    }

    // this thread's quad (Morton order inside the 16x16 quads of the block)
    int qx, qy;
    morton10((uint32_t)tid, qx, qy);
    const int cx0 = x0 + 2 * qx, cy0 = y0 + 2 * qy;
    const bool vx0 = cx0 < V.cells[0], vx1 = cx0 + 1 < V.cells[0];
    const bool vy0 = cy0 < V.cells[1], vy1 = cy0 + 1 < V.cells[1];

    uint32_t packed_prev = 0;
    bool timed_out = false;
    int li = 0;
    for (; li < nlayers; li++) {
        const int s = li % kRingStages;
        const uint32_t parity = (uint32_t)(li / kRingStages) & 1u;
        if (!mbar_wait_bounded(&s_bar[s], parity, kSpinLimit)) timed_out = true;
        if (!timed_out) {
            // layer li -> one bit per sample, rows of 33 bits
            const T* st = reinterpret_cast<const T*>(s_ring + s * STAGE_STRIDE);
            for (int r = warp; r < 33; r += kWarps) {
                const float v = (float)st[r * BXE + lane];
                const float v32 = (float)st[r * BXE + 32];
                float vv = v, vv32 = v32;
                if (FT == kFieldUNorm8) {
                    vv = __fdiv_rn(v, 255.0f);
                    vv32 = __fdiv_rn(v32, 255.0f);
                }
                const uint32_t b = __ballot_sync(0xffffffffu, vv < iso);
                if (lane == 0) s_rows[li % 3][r] = (uint64_t)b | ((uint64_t)(vv32 < iso) << 32);
            }
        }
        if (__syncthreads_or(timed_out)) break;  // barrier A: stage s is free, rows li ready
        if (tid == 0 && li + kRingStages < nlayers) {
            mbar_arrive_expect_tx(&s_bar[s], STAGE_BYTES);
            tma_load_3d(s_ring + s * STAGE_STRIDE, &tmap, x0, y0, z0 + li + kRingStages, &s_bar[s]);
        }
        // finalise slice li-2 (its warp sums were published before this barrier)
        if (li >= 2) {
            const int z = z0 + li - 2;
            uint32_t total = 0;
#pragma unroll
            for (int w = 0; w < kWarps; w++) total += s_warp[(li - 2) & 1][w];
            const uint64_t b = column_block_index(V, z, fx, fy);
            if (tid == 0) V.levels[V.level_off[kBlockLevel] + b] = total;
            if (total) {
                const long long slot = ((long long)z * V.nfy + fy) * V.nfx + fx;
                V.arena[slot * kBlockWords + tid] = packed_prev;
            }
            if (V.codes_out) write_codes(V, packed_prev, cx0, cy0, z);
        }
        // classify slice li-1 from sample layers li-1 (bottom) and li (top)
        if (li >= 1) {
            const uint64_t* rb = s_rows[(li - 1) % 3];
            const uint64_t* rt = s_rows[li % 3];
            uint32_t gb[3], gt[3];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                gb[j] = (uint32_t)(rb[2 * qy + j] >> (2 * qx)) & 7u;
                gt[j] = (uint32_t)(rt[2 * qy + j] >> (2 * qx)) & 7u;
            }
            const uint32_t packed = quad_codes(gb, gt, vx0, vx1, vy0, vy1);
            const uint32_t cnt = __reduce_add_sync(0xffffffffu, quad_count(s_cnt, packed));
            if (lane == 0) s_warp[(li - 1) & 1][warp] = cnt;
            packed_prev = packed;
        }
    }
    if (timed_out) {
        // drain the loads still in flight (bounded) before the CTA exits
        if (tid == 0) {
            for (int l = li; l < nlayers && l < li + kRingStages; l++)
                mbar_wait_bounded(&s_bar[l % kRingStages], (uint32_t)(l / kRingStages) & 1u, kSpinLimit);
            atomicOr(&V.ctrl->status, kStatusTimeout);
        }
        return;
    }
    __syncthreads();
    if (nlayers >= 2) {  // finalise the last slice
        const int z = z0 + nlayers - 2;
        uint32_t total = 0;
#pragma unroll
        for (int w = 0; w < kWarps; w++) total += s_warp[(nlayers - 2) & 1][w];
        const uint64_t b = column_block_index(V, z, fx, fy);
        if (tid == 0) V.levels[V.level_off[kBlockLevel] + b] = total;
        if (total) {
            const long long slot = ((long long)z * V.nfy + fy) * V.nfx + fx;
            V.arena[slot * kBlockWords + tid] = packed_prev;
        }
        if (V.codes_out) write_codes(V, packed_prev, cx0, cy0, z);
    }
}

// ---------------------------------------------------------------------------
// Generic classification: CTA = one 32x32 block of the virtual cell grid,
// for any tiling (tiles narrower than 32 cells), unaligned pitches and
// functor fields.  Each thread loads its quad's 3x3x2 samples directly.
template <int FT>
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
    const uint32_t wx = 2u * (uint32_t)V.tile_x, wy = 2u * (uint32_t)V.tile_y;
    const uint32_t tu = X / wx, tv = Y / wy;
    if (tu < (uint32_t)V.layout_x && tv < (uint32_t)V.layout_y) {
        x = (int)(X - tu * wx);
        y = (int)(Y - tv * wy);
        z = (int)(tv * (uint32_t)V.layout_x + tu);
        if (z < V.cells[2] && x < V.cells[0] && y < V.cells[1]) {
            uint32_t gb[3], gt[3];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                uint32_t bb = 0, bt = 0;
#pragma unroll
                for (int i = 0; i < 3; i++) {
                    bb |= (uint32_t)(fetch<FT>(V, x + i, y + j, z) < iso) << i;
                    bt |= (uint32_t)(fetch<FT>(V, x + i, y + j, z + 1) < iso) << i;
                }
                gb[j] = bb;
                gt[j] = bt;
            }
            packed = quad_codes(gb, gt, true, x + 1 < V.cells[0], true, y + 1 < V.cells[1]);
            if (V.codes_out) write_codes(V, packed, x, y, z);
        }
    }
    const uint32_t cnt = __reduce_add_sync(0xffffffffu, quad_count(s_cnt, packed));
    if (lane == 0) s_warp[warp] = cnt;
    __syncthreads();
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kWarps; w++) total += s_warp[w];
    if (tid == 0) V.levels[V.level_off[kBlockLevel] + b] = total;
    if (total) V.arena[block_slot(V, b) * kBlockWords + tid] = packed;
    __syncthreads();
}

template <int FT>
__global__ void __launch_bounds__(kThreads) classify_blocks(const __grid_constant__ Volume V) {
    __shared__ uint8_t s_cnt[256];
    __shared__ uint32_t s_warp[kWarps];
    s_cnt[threadIdx.x] = c_vertex_count[threadIdx.x];
    __syncthreads();
    for (uint64_t b = blockIdx.x; b < (uint64_t)V.nblocks; b += gridDim.x) classify_block_body<FT>(V, b, s_cnt, s_warp);
}

// ---------------------------------------------------------------------------
// Upper reductions (shadergen.cpp:174-225 without the floor filter): level
// j+1 entry e = sum of level j entries 4e..4e+3.  CTA c reduces 4096 entries
// of level j_in in shared memory (6 levels); the last CTA to finish carries
// on from those partial tops to level j_stop.  The top entry is the vertex
// count (hpiface.cpp:323-327).
constexpr int kReduceChunk = 4096;

__device__ __forceinline__ bool level5_valid(const Volume& V, uint64_t b) {
    int z, fx, fy;
    return column_block(V, b, z, fx, fy);
}

__device__ void reduce_tree(const Volume& V, uint32_t* buf0, uint32_t* buf1, int& j, int j_stop, long long n,
                            long long out_base, bool& overflow) {
    // buf0 holds n entries of level j (n a power of 4); out_base = index of the
    // first entry of level j in this chunk.
    uint32_t* src = buf0;
    uint32_t* dst = buf1;
    while (j < j_stop && n >= 4) {
        n >>= 2;
        out_base >>= 2;
        j++;
        for (long long i = threadIdx.x; i < n; i += blockDim.x) {
            const unsigned long long s = (unsigned long long)src[4 * i] + src[4 * i + 1] + src[4 * i + 2] + src[4 * i + 3];
            if (s > 0xffffffffull) overflow = true;
            dst[i] = (uint32_t)s;
            V.levels[V.level_off[j] + out_base + i] = (uint32_t)s;
        }
        __syncthreads();
        uint32_t* t = src;
        src = dst;
        dst = t;
    }
    if (src != buf0) {  // leave the result in buf0
        for (long long i = threadIdx.x; i < n; i += blockDim.x) buf0[i] = src[i];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads) reduce_levels(const __grid_constant__ Volume V, int j_in, int j_stop,
                                                          int mask_level5) {
    __shared__ uint32_t buf0[kReduceChunk];
    __shared__ uint32_t buf1[kReduceChunk / 4];
    __shared__ int s_last;
    bool overflow = false;
    const long long n_in = level_entries(V.size_l2, j_in);
    const long long base = (long long)blockIdx.x * kReduceChunk;
    const long long n = min((long long)kReduceChunk, n_in - base);
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        uint32_t v = V.levels[V.level_off[j_in] + base + i];
        if (mask_level5 && !level5_valid(V, (uint64_t)(base + i))) v = 0;
        buf0[i] = v;
    }
    __syncthreads();
    int j = j_in;
    reduce_tree(V, buf0, buf1, j, j_stop, n, base, overflow);
    if (j < j_stop) {
        // more levels remain above this chunk's top: last CTA continues
        __threadfence();
        if (threadIdx.x == 0) s_last = (atomicAdd(&V.ctrl->reduce_done, 1u) == gridDim.x - 1);
        __syncthreads();
        if (!s_last) {
            if (overflow) atomicOr(&V.ctrl->status, kStatusOverflow);
            return;
        }
        __threadfence();
        const long long m = level_entries(V.size_l2, j);  // == gridDim.x entries
        for (long long i = threadIdx.x; i < m; i += blockDim.x)
            buf0[i] = __ldcg(&V.levels[V.level_off[j] + i]);
        __syncthreads();
        reduce_tree(V, buf0, buf1, j, j_stop, m, 0, overflow);
        if (threadIdx.x == 0) V.ctrl->reduce_done = 0;
    }
    if (overflow) atomicOr(&V.ctrl->status, kStatusOverflow);
    if (j == V.jtop && threadIdx.x == 0) V.ctrl->total = buf0[0];
}

// Top entry when the whole pyramid is one block (no reduction launch needed).
__global__ void copy_total(const __grid_constant__ Volume V) {
    if (threadIdx.x == 0) V.ctrl->total = V.levels[V.level_off[V.jtop]];
}

// ---------------------------------------------------------------------------
// Host launchers
constexpr int kRingBytesF32 = kRingStages * ((36 * 33 * 4 + 127) & ~127) + 128;
constexpr int kRingBytesU8 = kRingStages * ((48 * 33 + 127) & ~127) + 128;

cudaError_t launch_classify(const Volume& V, const CUtensorMap* tmap, int max_ctas, cudaStream_t st) {
    if (V.column_layout && tmap) {
        const int nz = (V.cells[2] + kColumnSlices - 1) / kColumnSlices;
        const dim3 grid(V.nfx, V.nfy, nz);
        if (V.ftype == kFieldF32)
            classify_column_tma<kFieldF32><<<grid, kThreads, kRingBytesF32, st>>>(*tmap, V);
        else if (V.ftype == kFieldU8)
            classify_column_tma<kFieldU8><<<grid, kThreads, kRingBytesU8, st>>>(*tmap, V);
        else
            classify_column_tma<kFieldUNorm8><<<grid, kThreads, kRingBytesU8, st>>>(*tmap, V);
    } else {
        const long long nb = V.nblocks;
        const int grid = (int)(nb < (long long)max_ctas ? nb : (long long)max_ctas);
        switch (V.ftype) {
            case kFieldF32: classify_blocks<kFieldF32><<<grid, kThreads, 0, st>>>(V); break;
            case kFieldU8: classify_blocks<kFieldU8><<<grid, kThreads, 0, st>>>(V); break;
            case kFieldUNorm8: classify_blocks<kFieldUNorm8><<<grid, kThreads, 0, st>>>(V); break;
            default: classify_blocks<kFieldFunctor><<<grid, kThreads, 0, st>>>(V); break;
        }
    }
    return cudaGetLastError();
}

cudaError_t launch_reduce(const Volume& V, cudaStream_t st) {
    if (V.jtop == kBlockLevel) {
        copy_total<<<1, 32, 0, st>>>(V);
        return cudaGetLastError();
    }
    int j_in = kBlockLevel;
    while (j_in < V.jtop) {
        // one launch reduces 6 levels per CTA plus up to 6 more in the last CTA
        const int j_stop = (V.jtop - j_in <= 12) ? V.jtop : j_in + 6;
        const long long n_in = level_entries(V.size_l2, j_in);
        const long long grid = (n_in + kReduceChunk - 1) / kReduceChunk;
        reduce_levels<<<(unsigned)grid, kThreads, 0, st>>>(V, j_in, j_stop,
                                                            (j_in == kBlockLevel && V.column_layout) ? 1 : 0);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        j_in = j_stop;
    }
    return cudaSuccess;
}

bool column_smem_ok() {
    static int configured = 0;
    if (!configured) {
        cudaFuncSetAttribute(classify_column_tma<kFieldF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRingBytesF32);
        cudaFuncSetAttribute(classify_column_tma<kFieldU8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRingBytesU8);
        cudaFuncSetAttribute(classify_column_tma<kFieldUNorm8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kRingBytesU8);
        configured = 1;
    }
    return true;
}

}  // namespace hpmc
