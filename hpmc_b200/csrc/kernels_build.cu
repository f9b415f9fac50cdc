// kernels_build.cu -- HistoPyramid build on sm_100a: classification fused
// with the first five reductions, then the upper reductions.
//
// Reference passes replaced (hpmc/src/buildpass.cpp:42-178):
//   base level  (shadergen.cpp:86-171)  -> classify_columns / classify_blocks
//   first reduction + 4 upper levels    -> fused into classification (a 32x32
//                                          cell block = 4^5 keys is summed in
//                                          registers and warp reductions)
//   remaining upper reductions          -> reduce_levels (one launch,
//                                          last-block-done chaining)
//   top readback (buildpass.cpp:161-168)-> Ctrl::total in device memory
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "hpmc_batch.cuh"
#include "hpmc_device.cuh"
#include "hpmc_fetch.cuh"
#include "hpmc_kernels.h"
#include "hpmc_tma.cuh"
#include "hpmc_classify_core.cuh"

namespace hpmc {

// ---------------------------------------------------------------------------
// Column classification: a column = one 32x32 cell footprint of the slice
// tiles x column_slices slices, streamed through a TMA ring of 8-layer
// sample boxes (each sample leaves HBM once; halo rows/columns are shared
// with neighbouring columns through L2).  The single-volume kernel is
// persistent (columns from a device queue); the batched one takes one column
// brick per CTA.
//
// Per layer, every warp turns rows of samples into bits (f < iso) with one
// ballot per row.  Per slice, ONE warp classifies the whole 32x32 block,
// bit-sliced: lane y holds the 32 cells of row y as eight 32-bit words, word
// k = bit k (dx + 2dy + 4dz) of the 32 codes.  AND/OR over the eight words
// marks the cells that are neither all-inside nor all-outside (the only ones
// with vertices); only those go through the count table.  The warp sum is the
// block's level-5 entry; non-empty blocks also store their 1024 codes in
// Morton order and each 32-cell tile's active mask and vertex count in their
// arena slot (1.25 KiB), from which a traversal warp builds the block's
// active-cell list when it enters the block.
//
// Measured alternatives for the list: written by the classifier (each
// non-empty block's serial gathers stall the box barrier: +20 us at 512^3),
// or by a separate pass over queued slots beside the reduction (issue-bound,
// ~500 warp instructions per list, not hidden by the 7 us reduction tree:
// +11 us) -- both slower than one build per warp in the traversal, where the
// latency of the list's gathers overlaps other warps' vertex work.
namespace {

template <int FT, typename T>
__device__ __forceinline__ bool below(T v, float iso, int u8_thr) {
    if constexpr (FT == kFieldF32)
        return v < iso;  // strict; NaN -> false (shadergen.cpp:137-142)
    else
        return (int)v < u8_thr;
}

// 8x8 bit-matrix transpose: byte r bit c -> byte c bit r.
__device__ __forceinline__ uint64_t transpose8(uint64_t x) {
    uint64_t t;
    t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
    x = x ^ t ^ (t << 7);
    t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
    x = x ^ t ^ (t << 14);
    t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
    x = x ^ t ^ (t << 28);
    return x;
}

// Bit-sliced codes of one 32-cell row -> 32 byte codes (w[i] = cells 4i..4i+3).
__device__ __forceinline__ void slices_to_codes(const uint32_t c[8], uint32_t w[8]) {
#pragma unroll
    for (int g = 0; g < 4; g++) {
        const uint32_t sel = (uint32_t)g | ((uint32_t)(g + 4) << 4);
        const uint32_t lo = __byte_perm(__byte_perm(c[0], c[1], sel), __byte_perm(c[2], c[3], sel), 0x5410);
        const uint32_t hi = __byte_perm(__byte_perm(c[4], c[5], sel), __byte_perm(c[6], c[7], sel), 0x5410);
        const uint64_t x = transpose8((uint64_t)lo | ((uint64_t)hi << 32));
        w[2 * g] = (uint32_t)x;
        w[2 * g + 1] = (uint32_t)(x >> 32);
    }
}

// 16 bits -> Morton positions of an 8x2 cell tile: bit x of the low byte goes
// to bit (x0 | x1 << 2 | x2 << 4), bit x of the high byte to that + 8.
__device__ __forceinline__ uint32_t spread16(uint32_t t) {
    t = (t | (t << 12)) & 0x0F0F0F0Fu;
    return (t | (t << 2)) & 0x33333333u;
}

// One warp: classify slice z of footprint (fx, fy) from sample-bit rows of the
// lower layer (rows_b/col_b) and the upper layer (rows_t/col_t).  Every block
// gets its level-5 count; blocks with vertices store their codes in Morton
// order in their slot.  full: every cell of the footprint lies inside the
// grid (vmask is all ones in every lane).  b: the block's level-5 index,
// column_block_index(V, z, fx, fy).
__device__ __forceinline__ void classify_slice_warp(const Volume& V, int z, int fx, int fy, uint32_t b, int lane,
                                                    uint32_t vmask, bool full, const uint32_t* rows_b,
                                                    uint64_t col_b, const uint32_t* rows_t, uint64_t col_t,
                                                    const uint8_t* s_cnt) {
    // rows y and y+1 of both layers; bit 32 of a row (column x0+32) comes
    // from the column word: (row >> 1) | colbit << 31 is the row shifted by one cell
    const uint32_t cbl = (uint32_t)col_b, cbh = (uint32_t)(col_b >> 32);
    const uint32_t ctl = (uint32_t)col_t, cth = (uint32_t)(col_t >> 32);
    const uint32_t a0 = rows_b[lane], a1 = rows_b[lane + 1];
    const uint32_t b0 = rows_t[lane], b1 = rows_t[lane + 1];
    if (full && !V.codes_out) {
        // A full block has no vertices iff its 33x33x2 samples all lie on one
        // side of the iso-value (two samples that differ have some edge
        // between them that differs, and every edge belongs to a cell of the
        // block): one AND and one OR of the lane's two rows in both layers
        // and of its two column bits, two votes.
        const uint32_t cb = __funnelshift_r(cbl, cbh, lane) & 3u, ct = __funnelshift_r(ctl, cth, lane) & 3u;
        const bool below_all = ((a0 & a1 & b0 & b1) == 0xffffffffu) && ((cb & ct) == 3u);
        const bool above_all = ((a0 | a1 | b0 | b1) == 0u) && ((cb | ct) == 0u);
        if (__all_sync(0xffffffffu, below_all) || __all_sync(0xffffffffu, above_all)) {
            if (lane == 0) V.levels[V.level_off[kBlockLevel] + b] = 0u;
            return;
        }
    }
    uint32_t c[8];
    c[0] = a0;                                                   // (x,   y,   z)
    c[1] = (a0 >> 1) | (((cbl >> lane) & 1u) << 31);             // (x+1, y,   z)
    c[2] = a1;                                                   // (x,   y+1, z)
    c[3] = (a1 >> 1) | ((__funnelshift_rc(cbl, cbh, lane + 1) & 1u) << 31);
    c[4] = b0;                                                   // (x,   y,   z+1)
    c[5] = (b0 >> 1) | (((ctl >> lane) & 1u) << 31);
    c[6] = b1;
    c[7] = (b1 >> 1) | ((__funnelshift_rc(ctl, cth, lane + 1) & 1u) << 31);
    uint32_t all = c[0], any = c[0];
#pragma unroll
    for (int k = 1; k < 8; k++) {
        all &= c[k];
        any |= c[k];
    }
    // cells that are neither all-inside nor all-outside: the only ones with
    // vertices (every other MC case has at least one triangle)
    const uint32_t active = (all ^ any) & vmask;
    const bool has_vertices = __any_sync(0xffffffffu, active != 0u);
    if (!has_vertices) {
        if (lane == 0) V.levels[V.level_off[kBlockLevel] + b] = 0u;
        if (!V.codes_out) return;
    }
    // codes of this row (cells outside the grid are masked to 0)
#pragma unroll
    for (int k = 0; k < 8; k++) c[k] &= vmask;
    uint32_t w[8];
    slices_to_codes(c, w);
    if (has_vertices) {
        // the block's vertices: 32 independent count lookups per lane (byte j
        // of seg = the row's cells 8j .. 8j+7, at most 96), one warp
        // reduction (inactive cells have codes 0 or 255, count 0)
        uint32_t seg = 0;
#pragma unroll
        for (int i = 0; i < 32; i++) seg += (uint32_t)s_cnt[(w[i >> 2] >> (8 * (i & 3))) & 0xffu] << (8 * (i >> 3));
        const uint32_t vs = (seg & 0xffu) + ((seg >> 8) & 0xffu) + ((seg >> 16) & 0xffu) + (seg >> 24);
        const uint32_t total = __reduce_add_sync(0xffffffffu, vs);
        if (lane == 0) V.levels[V.level_off[kBlockLevel] + b] = total;
        // codes in Morton order: word q of the slot = quad (qx, qy), cells
        // (2qx,2qy), (2qx+1,2qy), (2qx,2qy+1), (2qx+1,2qy+1) from rows 2qy
        // (even lane) and 2qy+1 (odd lane); even lanes store qx 0..7, odd
        // lanes qx 8..15, each pairing its row with its neighbour's
        uint32_t p[8];
#pragma unroll
        for (int i = 0; i < 8; i++) p[i] = __shfl_xor_sync(0xffffffffu, w[i], 1);
        const bool odd = lane & 1;
        const uint32_t qy = (uint32_t)lane >> 1;
        const long long slot = ((long long)z * V.nfy + fy) * V.nfx + fx;
        uint32_t* dst = V.arena + slot * kSlotWords;
        // Morton index of quad (qx, qy), qx = (odd ? 8 : 0) + i: the bits of i
        // (compile-time) and of the lane's part are disjoint
        const uint32_t qys = (qy & 1u) | ((qy & 2u) << 1) | ((qy & 4u) << 2) | ((qy & 8u) << 3);
        const uint32_t qbase = (odd ? 0x40u : 0u) | (qys << 1);
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const uint32_t wi = odd ? w[4 + (i >> 1)] : w[i >> 1];  // this lane's word with cells 2qx, 2qx+1
            const uint32_t pi = odd ? p[4 + (i >> 1)] : p[i >> 1];
            const uint32_t upper = odd ? wi : pi;  // row 2qy+1
            const uint32_t lower = odd ? pi : wi;  // row 2qy
            const uint32_t word = __byte_perm(lower, upper, (i & 1) ? 0x7632 : 0x5410);
            const uint32_t ispread = (uint32_t)((i & 1) | ((i & 2) << 1) | ((i & 4) << 2));
            dst[qbase | ispread] = word;
        }
        // Morton tile q = lane (cells 32q .. 32q+31, an 8x4 tile at rows
        // ty .. ty+3, columns tx .. tx+7; Morton bits x0 y0 x1 y1 x2 | y2 x3
        // y3 x4 y4): its active mask gathered from four rows in Morton order
        // and its vertices from the rows' segment counts
        const uint32_t q = (uint32_t)lane;
        const int ty = 4 * (int)((q & 1u) | ((q >> 1) & 2u) | ((q >> 2) & 4u));
        const uint32_t tx = 8u * (((q >> 1) & 1u) | ((q >> 2) & 2u));
        uint32_t r[4], tcnt = 0;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            r[i] = (__shfl_sync(0xffffffffu, active, ty + i) >> tx) & 0xffu;
            tcnt += (__shfl_sync(0xffffffffu, seg, ty + i) >> tx) & 0xffu;
        }
        // rows 0/2 on Morton bit 3 = 0/1 with bit 1 = 0; rows 1/3 shifted by 2 (bit 1 = 1)
        const uint32_t tmask = spread16(r[0] | (r[2] << 8)) | (spread16(r[1] | (r[3] << 8)) << 2);
        reinterpret_cast<uint2*>(dst + kSlotTileWord)[lane] = make_uint2(tmask, tcnt);
    }
    if (V.codes_out) {
        const int y = fy * 32 + lane;
        if (y < V.cells[1]) {
            uint8_t* row = V.codes_out + ((long long)z * V.cells[1] + y) * V.cells[0] + fx * 32;
            const int nx = min(32, V.cells[0] - fx * 32);
#pragma unroll
            for (int i = 0; i < 32; i++)
                if (i < nx) row[i] = (uint8_t)(w[i >> 2] >> (8 * (i & 3)));
        }
    }
}

}  // namespace

// Shared memory of a column classifier CTA.  Bit rows are kept for the last
// kRowBuffers sample layers (indexed by a running layer counter mod
// kRowBuffers): while a slow warp still classifies the slices of box p
// (layers 8p-1 .. 8p+7) other warps already convert box p+1 (layers 8p+8 ..
// 8p+15), so the buffers of the two boxes must not alias.
constexpr int kRowBuffers = 32;

template <int FT>
struct ColumnGeom {
    using T = typename std::conditional<FT == kFieldF32, float, uint8_t>::type;
    static constexpr int BXE = (FT == kFieldF32) ? 36 : 48;  // box width (16-byte multiple)
    static constexpr int LAYER = BXE * 33;                    // elements of one sample layer
    static constexpr int STAGE_BYTES = LAYER * kLayersPerBox * (int)sizeof(T);
    static constexpr int STAGE_STRIDE = (STAGE_BYTES + 127) & ~127;
};

struct ColumnSmem {
    // 16-byte aligned: warps store 4 rows at a time (uint4), whatever the
    // number of ring stages before it
    alignas(16) uint32_t rows[kRowBuffers][36];  // bit x = sample (x0 + x, y0 + r) below iso; [32] = row 32
    uint64_t col[kRowBuffers];                   // bit r = sample (x0 + 32, y0 + r) below iso; bit 32 = corner
    uint64_t bar[kRingStages];
    uint8_t cnt[256];
    // level-5 index of block (0, 0) of slice z, z < kSliceTable: a footprint's
    // block is that OR its own Morton part (the footprint's bits lie below
    // the tile's), so a slice costs one load instead of two bit spreads
    uint32_t zbase[1024];
};
constexpr int kSliceTable = 1024;
static_assert(offsetof(ColumnSmem, rows) % 16 == 0 && (36 * 4) % 16 == 0, "uint4 row stores need 16-byte alignment");

// Bit rows of the nl layers of one box (stage st), layer l stored at
// running index gl0 + l.  Warp w converts rows 4w .. 4w+3 of every layer;
// row 32 and column x0+32 of layer g go to warp (g + 3) mod 8.
static_assert(kWarps == 8 && kLayersPerBox <= kWarps, "a box's layers and slices map onto the 8 warps mod 8");
static_assert(kRowBuffers % kLayersPerBox == 0, "a box's bit-row buffers never wrap");

template <int FT>
__device__ __forceinline__ void convert_box(const typename ColumnGeom<FT>::T* st, int nl, uint32_t gl0, float iso,
                                            int u8_thr, int warp, int lane, ColumnSmem& C) {
    using G = ColumnGeom<FT>;
    using T = typename G::T;
    // Every sample first, then the ballots and stores: the compiler cannot
    // tell the bit-row stores from the ring stage, so loads issued after a
    // store would wait for it.  A stage always holds kLayersPerBox layers
    // (copies past the volume read zeros), so all of them are read; layers
    // past nl are not stored.
    T v[kLayersPerBox][4];
    const T* row = st + 4 * warp * G::BXE + lane;
#pragma unroll
    for (int l = 0; l < kLayersPerBox; l++)
#pragma unroll
        for (int i = 0; i < 4; i++) v[l][i] = row[l * G::LAYER + i * G::BXE];
    const int le = (int)(((uint32_t)warp - gl0 - 3u) & 7u);  // the layer whose row 32 and column 32 this warp takes
    const T* layer = st + (le < kLayersPerBox ? le : 0) * G::LAYER;  // inside the stage for any box depth
    const T e_row = layer[32 * G::BXE + lane], e_col = layer[lane * G::BXE + 32], e_corner = layer[32 * G::BXE + 32];
    // gl0 is a multiple of kLayersPerBox and kRowBuffers of that, so a box's
    // buffers are g0 .. g0 + kLayersPerBox - 1 without wrapping
    const uint32_t g0 = gl0 & (kRowBuffers - 1);
    uint4* const rows_w = reinterpret_cast<uint4*>(&C.rows[g0][4 * warp]);
#pragma unroll
    for (int l = 0; l < kLayersPerBox; l++) {
        const uint32_t b0 = __ballot_sync(0xffffffffu, below<FT>(v[l][0], iso, u8_thr));
        const uint32_t b1 = __ballot_sync(0xffffffffu, below<FT>(v[l][1], iso, u8_thr));
        const uint32_t b2 = __ballot_sync(0xffffffffu, below<FT>(v[l][2], iso, u8_thr));
        const uint32_t b3 = __ballot_sync(0xffffffffu, below<FT>(v[l][3], iso, u8_thr));
        if (l < nl && lane == 0) rows_w[l * (36 / 4)] = make_uint4(b0, b1, b2, b3);
    }
    const uint32_t r32 = __ballot_sync(0xffffffffu, below<FT>(e_row, iso, u8_thr));
    const uint32_t col = __ballot_sync(0xffffffffu, below<FT>(e_col, iso, u8_thr));
    const bool corner = below<FT>(e_corner, iso, u8_thr);
    if (le < nl && lane == 0) {
        const uint32_t buf = g0 + (uint32_t)le;
        C.rows[buf][32] = r32;
        C.col[buf] = (uint64_t)col | ((uint64_t)corner << 32);
    }
}

// Morton part of footprint (fx, fy) in a block index.
__device__ __forceinline__ uint32_t footprint_morton(int fx, int fy) {
    return morton_spread16((uint32_t)fx) | (morton_spread16((uint32_t)fy) << 1);
}

// The slice table for slices 0 .. min(cells, kSliceTable)-1 (all threads).
__device__ __forceinline__ void fill_slice_table(const Volume& V, ColumnSmem& C) {
    const int n = min(V.cells[2], kSliceTable);
    for (int z = threadIdx.x; z < n; z += blockDim.x) C.zbase[z] = (uint32_t)column_block_index(V, z, 0, 0);
}

__device__ __forceinline__ uint32_t slice_block(const Volume& V, const ColumnSmem& C, int z, uint32_t fm) {
    return (z < kSliceTable ? C.zbase[z] : (uint32_t)column_block_index(V, z, 0, 0)) | fm;
}

// After the box barrier: the slices whose upper layer arrived in this box
// (column-relative slices lb-1 .. lb+nl-2), warp (glu + slice) mod 8 each, so
// the work rotates over the warps from box to box.  glu = running index of
// the column's layer 0.
__device__ __forceinline__ void classify_box_slices(const Volume& V, int z0, int fx, int fy, uint32_t fm, int lb,
                                                    int nl, uint32_t glu, int warp, int lane, uint32_t vmask,
                                                    bool full, ColumnSmem& C) {
    // the slice of this warp, if any.  glu + lb is the running index of the
    // box's first layer, a multiple of kLayersPerBox: with 8-layer boxes the
    // warp's offset in the box is the same in every box
    const uint32_t w1 = kLayersPerBox == 8 ? (uint32_t)(warp + 1) & 7u
                                           : ((uint32_t)warp - (glu + (uint32_t)lb - 1u)) & 7u;
    const int sl = lb - 1 + (int)w1;
    if (sl >= 0 && sl <= lb + nl - 2) {
        const uint32_t g = glu + (uint32_t)sl;
        const uint32_t bb = g & (kRowBuffers - 1), bt = (g + 1u) & (kRowBuffers - 1);
        const int z = z0 + sl;
        classify_slice_warp(V, z, fx, fy, slice_block(V, C, z, fm), lane, vmask, full, C.rows[bb], C.col[bb],
                            C.rows[bt], C.col[bt], C.cnt);
    }
}

// Cells of row `lane` of footprint (x0, y0) inside the grid (masked codes are
// 0, shadergen.cpp:112-125).
__device__ __forceinline__ uint32_t row_mask(const Volume& V, int x0, int y0, int lane) {
    const int xv = V.cells[0] - x0;
    const uint32_t xmask = xv >= 32 ? 0xffffffffu : ((1u << xv) - 1u);
    return (y0 + lane < V.cells[1]) ? xmask : 0u;
}

template <int FT>
__device__ __forceinline__ uint8_t* ring_base() {
    extern __shared__ __align__(128) uint8_t s_dyn[];
    // TMA destinations must be 128-byte aligned: align the ring explicitly
    // (the launch reserves 128 spare bytes)
    return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(s_dyn) + 127) & ~uintptr_t(127));
}

// Column CTA body (one column per CTA): footprint (fx, fy) of the slice
// tiles, slices zc*column_slices .. +column_slices-1, field boxes from `tmap`.
template <int FT>
__device__ __forceinline__ void classify_column_body(const CUtensorMap* tmap, const Volume& V, int fx, int fy,
                                                     int zc) {
    using G = ColumnGeom<FT>;
    uint8_t* const s_ring = ring_base<FT>();
    __shared__ __align__(16) ColumnSmem C;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int x0 = fx * 32, y0 = fy * 32;
    const int z0 = zc * V.column_slices;
    const int z1 = min(V.cells[2], z0 + V.column_slices);
    const int nlayers = z1 - z0 + 1;
    const int nbox = (nlayers + kLayersPerBox - 1) / kLayersPerBox;
    const float iso = V.binary ? 0.5f : V.iso;
    const int u8_thr = V.u8_thr;

    C.cnt[tid] = c_vertex_count[tid];
    fill_slice_table(V, C);
    const uint32_t fm = footprint_morton(fx, fy);
    if (tid == 0) {
        for (int s = 0; s < kRingStages; s++) mbar_init(&C.bar[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    // test hook: the first column of the volume never receives box stall_box
    const int stall = (fx == 0 && fy == 0 && zc == 0) ? V.stall_box : -1;
    const uint64_t pol = l2_evict_first_policy();  // the field is read once
    if (tid == 0) {
        for (int k = 0; k < kRingStages && k < nbox; k++) {
            if (k == stall) continue;
            mbar_arrive_expect_tx(&C.bar[k], G::STAGE_BYTES);
            tma_load_3d(s_ring + k * G::STAGE_STRIDE, tmap, x0, y0, z0 + k * kLayersPerBox, &C.bar[k], pol);
        }
    }
    const uint32_t vmask = row_mask(V, x0, y0, lane);
    const bool full = __all_sync(0xffffffffu, vmask == 0xffffffffu);

    bool timed_out = false;
    int k = 0;
    for (; k < nbox; k++) {
        const int s = k % kRingStages;
        const uint32_t parity = (uint32_t)(k / kRingStages) & 1u;
        const int lb = k * kLayersPerBox;
        const int nl = min(kLayersPerBox, nlayers - lb);
        // every warp waits on the box's mbarrier (suspended in hardware, not spinning)
        if (!mbar_wait_bounded(&C.bar[s], parity, V.wait_limit_ns, &V.ctrl->status, kStatusTimeout)) timed_out = true;
        if (!timed_out)
            convert_box<FT>(reinterpret_cast<const typename G::T*>(s_ring + s * G::STAGE_STRIDE), nl, (uint32_t)lb,
                            iso, u8_thr, warp, lane, C);
        // the only CTA barrier of a box: stage s consumed, bit rows of layers
        // lb .. lb+nl-1 ready, and a uniform decision on a timed-out wait
        if (__syncthreads_or(timed_out)) break;
        if (tid == 0 && k + kRingStages < nbox && k + kRingStages != stall) {
            mbar_arrive_expect_tx(&C.bar[s], G::STAGE_BYTES);
            tma_load_3d(s_ring + s * G::STAGE_STRIDE, tmap, x0, y0, z0 + (k + kRingStages) * kLayersPerBox,
                        &C.bar[s], pol);
        }
        classify_box_slices(V, z0, fx, fy, fm, lb, nl, 0u, warp, lane, vmask, full, C);
    }
    if (timed_out) {
        // drain the boxes still in flight (bounded) before the CTA exits
        if (tid == 0) {
            for (int l = k; l < nbox && l < k + kRingStages; l++)
                mbar_wait_bounded(&C.bar[l % kRingStages], (uint32_t)(l / kRingStages) & 1u, V.wait_limit_ns,
                                  nullptr, 0u);
            atomicOr(&V.ctrl->status, kStatusTimeout);
        }
    }
}

// Persistent column classifier (column = footprint (fx, fy) x one run of
// column_slices slices, numbered footprint-fastest so that neighbouring
// columns share halo samples in L2).  Thread 0 claims columns from a device
// queue (one atomic per column: a CTA whose columns end early takes more) and
// streams their boxes back to back through the ring, tagging every stage with
// its column and box, so the copy engine never idles between columns; after
// the last column it arrives on the next stage without a copy, tagged -1.
// The last CTA to finish resets the queue for the next launch.
template <int FT>
__global__ void __launch_bounds__(kThreads) classify_columns(const __grid_constant__ CUtensorMap tmap,
                                                             const __grid_constant__ Volume V, int ncolumns) {
    using G = ColumnGeom<FT>;
    uint8_t* const s_ring = ring_base<FT>();
    __shared__ __align__(16) ColumnSmem C;
    // per ring stage: box k | layers << 16 of its column (-1: end), footprint
    // fx | fy << 16, first slice and the footprint's Morton part -- decoded
    // once by the producer, so that the consumers start converting without
    // integer divisions after each wait
    __shared__ int4 s_tag[kRingStages];
    // per ring stage: the column's x mask and valid rows (bit 31: every row
    // valid and the mask full), so a lane's row mask is one compare
    __shared__ uint2 s_rowmask[kRingStages];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int per_slab = V.nfx * V.nfy;
    const float iso = V.binary ? 0.5f : V.iso;
    const int u8_thr = V.u8_thr;
    // column u -> footprint, first slice, layers (slices + 1)
    auto column = [&](int u, int& fx, int& fy, int& z0, int& nlayers) {
        const int zc = u / per_slab;
        const int r = u - zc * per_slab;
        fy = r / V.nfx;
        fx = r - fy * V.nfx;
        z0 = zc * V.column_slices;
        nlayers = min(V.cells[2], z0 + V.column_slices) - z0 + 1;
    };

    __shared__ int s_early;
    C.cnt[tid] = c_vertex_count[tid];
    fill_slice_table(V, C);
    if (tid == 0) {
        for (int s = 0; s < kRingStages; s++) mbar_init(&C.bar[s], 1);
        mbar_fence_init();
        // The previous grid may still be this pyramid's extraction (its
        // flag is set before it lets this launch begin and cleared by its
        // last CTA): then this CTA streams at once and waits at its end.  A
        // CTA that sees the flag clear takes the ordinary path; a stale clear
        // flag only costs the overlap.
        s_early = V.overlap && *reinterpret_cast<volatile unsigned int*>(&V.ctrl->extracting) != 0u;
    }
    __syncthreads();
    const bool early = s_early != 0;
    // Otherwise global memory (field, pyramid, control block) only after the
    // previous grid.  No early trigger: the reduce launches as these CTAs
    // exit (reduce CTAs resident and waiting through the whole build measured
    // ~2% slower).
    if (!early) wait_prior_grid();
    // producer state (thread 0): next box to issue = box pk of column pu; the
    // following column is claimed one column ahead (pnext), so the atomic's
    // round trip overlaps the current column
    int pu = -1, pk = 0, pnl = 0, pz0 = 0, pfx = 0, pfy = 0, pnext = -1;
    const uint64_t pol = l2_evict_first_policy();  // the field is read once
    bool pdone = false;
    uint32_t issued = 0;
    if (tid == 0) pnext = (int)atomicAdd(&V.ctrl->col_next, 1u);
    auto issue_next = [&]() {
        if (pdone) return;
        const int s = (int)(issued % kRingStages);
        if (pu < 0 || pk * kLayersPerBox >= pnl) {
            pu = pnext;
            if (pu < ncolumns) pnext = (int)atomicAdd(&V.ctrl->col_next, 1u);
            pk = 0;
            if (pu >= ncolumns) {
                s_tag[s] = make_int4(-1, 0, 0, 0);
                mbar_arrive(&C.bar[s]);  // completes the phase: the consumers see the end tag
                issued++;
                pdone = true;
                return;
            }
            column(pu, pfx, pfy, pz0, pnl);
        }
        s_tag[s] = make_int4(pk | (pnl << 16), pfx | (pfy << 16), pz0, (int)footprint_morton(pfx, pfy));
        {
            const int xv = V.cells[0] - pfx * 32, yv = V.cells[1] - pfy * 32;
            const uint32_t xm = xv >= 32 ? 0xffffffffu : ((1u << xv) - 1u);
            const uint32_t rows = (uint32_t)min(yv, 32);
            s_rowmask[s] = make_uint2(xm, rows | ((xm == 0xffffffffu && rows == 32u) ? 0x80000000u : 0u));
        }
        // test hook: a CTA never issues its box stall_box (its waits run out)
        if ((int)issued != V.stall_box) {
            mbar_arrive_expect_tx(&C.bar[s], G::STAGE_BYTES);
            tma_load_3d(s_ring + s * G::STAGE_STRIDE, &tmap, pfx * 32, pfy * 32, pz0 + pk * kLayersPerBox, &C.bar[s],
                        pol);
        }
        issued++;
        pk++;
    };
    if (tid == 0)
        for (int i = 0; i < kRingStages; i++) issue_next();

    bool timed_out = false;
    uint32_t pos = 0;  // running box position (ring slot, phase, row-buffer index)
    for (;; pos++) {
        const int s = (int)(pos % kRingStages);
        const uint32_t parity = (pos / kRingStages) & 1u;
        const bool ok = mbar_wait_bounded(&C.bar[s], parity, V.wait_limit_ns, &V.ctrl->status, kStatusTimeout);
        // the stage's tag was written before the producer's arrival (release) on its barrier
        const int4 tag = ok ? s_tag[s] : make_int4(-1, 0, 0, 0);
        const uint2 rm = ok ? s_rowmask[s] : make_uint2(0u, 0u);  // read before the producer refills stage s
        const int fx = tag.y & 0xffff, fy = tag.y >> 16, z0 = tag.z;
        const uint32_t fm = (uint32_t)tag.w;
        const int k = tag.x & 0xffff, nlayers = tag.x >> 16;
        const int lb = k * kLayersPerBox;
        const int nl = min(kLayersPerBox, nlayers - lb);
        if (ok && tag.x >= 0)
            convert_box<FT>(reinterpret_cast<const typename G::T*>(s_ring + s * G::STAGE_STRIDE), nl,
                            pos * kLayersPerBox, iso, u8_thr, warp, lane, C);
        // the only CTA barrier of a box (uniform decision on a timed-out wait);
        // the producer rewrites the stage and its tag only after it
        if (__syncthreads_or(!ok)) {
            timed_out = true;
            break;
        }
        if (tag.x < 0) break;        // the end tag (the same for every thread)
        if (tid == 0) issue_next();  // refill stage s
        const uint32_t vmask = (uint32_t)lane < (rm.y & 0xffu) ? rm.x : 0u;  // == row_mask(V, 32 fx, 32 fy, lane)
        const bool full = (rm.y >> 31) != 0u;
        classify_box_slices(V, z0, fx, fy, fm, lb, nl, (pos - (uint32_t)k) * kLayersPerBox, warp, lane, vmask, full,
                            C);
    }
    if (timed_out && tid == 0) {
        // drain the boxes still in flight (bounded) before the CTA exits
        for (uint32_t p = pos; p < issued; p++)
            mbar_wait_bounded(&C.bar[p % kRingStages], (p / kRingStages) & 1u, V.wait_limit_ns, nullptr, 0u);
        atomicOr(&V.ctrl->status, kStatusTimeout);
    }
    // an early CTA ends only after the extraction it overlapped, so the
    // reduce (and all later work) still follows every earlier grid
    if (early) wait_prior_grid();
    // the last CTA to finish resets the column queue for the next launch
    if (tid == 0) {
        __threadfence();
        if (atomicAdd(&V.ctrl->col_done, 1u) == gridDim.x - 1) {
            V.ctrl->col_next = 0;
            V.ctrl->col_done = 0;
            __threadfence();
        }
    }
}


// ---------------------------------------------------------------------------
// Upper reductions (shadergen.cpp:174-225 without the floor filter): level
// j+1 entry e = sum of level j entries 4e..4e+3.  CTA c reduces 1024 entries
// of level j_in (5 levels: registers, shuffles and one shared-memory
// exchange); the last CTA to finish carries on from those partial tops to
// level j_stop.  The top entry is the vertex count (hpiface.cpp:323-327).
// Level-5 entries of padding blocks (footprints past the grid) are zero: the
// levels are cleared when they are set up and only the generic classifier
// writes those entries, with zero.
constexpr int kReduceChunk = 1024;  // level entries per CTA (5 levels)
constexpr int kReduceTop = 4096;    // entries the last CTA can finish (6 levels)


__device__ void reduce_tree(const Volume& V, uint32_t* buf0, uint32_t* buf1, int& j, int j_stop, long long n,
                            long long out_base, bool& overflow) {
    // buf0 holds n entries of level j (n a power of 4); out_base = index of the
    // first entry of level j in this chunk.  Leaves the last level in buf0.
    uint32_t* src = buf0;
    uint32_t* dst = buf1;
    while (j < j_stop && n >= 4) {
        n >>= 2;
        out_base >>= 2;
        j++;
        for (long long i = threadIdx.x; i < n; i += blockDim.x) {
            const unsigned long long s =
                (unsigned long long)src[4 * i] + src[4 * i + 1] + src[4 * i + 2] + src[4 * i + 3];
            if (s > 0xffffffffull) overflow = true;
            dst[i] = (uint32_t)s;
            V.levels[V.level_off[j] + out_base + i] = (uint32_t)s;
        }
        __syncthreads();
        uint32_t* t = src;
        src = dst;
        dst = t;
    }
    if (src != buf0) {
        for (long long i = threadIdx.x; i < n; i += blockDim.x) buf0[i] = src[i];
        __syncthreads();
    }
}

// One chunk of kReduceChunk level-j_in entries (chunk `chunk` of `nchunks`).
// Returns true in the CTA that wrote the vertex count (level jtop reached).
__device__ __forceinline__ bool reduce_chunk(const Volume& V, int j_in, int j_stop, long long chunk, unsigned int nchunks, uint32_t* buf0, uint32_t* buf1,
                                             int* s_last) {
    bool overflow = false;
    const long long n_in = level_entries(V.size_l2, j_in);
    const long long base = chunk * kReduceChunk;
    const long long n = min((long long)kReduceChunk, n_in - base);  // a power of 4 (>= 4), or 1 at the top
    const int t = threadIdx.x;
    int j = j_in;
    if (n == kReduceChunk && j_stop - j_in >= 5) {
        // a full chunk, five levels without shared-memory round trips: thread
        // t's four entries make level j+1 entry t, groups of 4 and 16 lanes
        // (shuffles) levels j+2 and j+3, pairs of warps and then all eight
        // (one exchange) levels j+4 and j+5.  A chunk's sums stay below 2^32
        // (1024 entries of at most 15 * 1024 vertices each).
        const uint4 v = *reinterpret_cast<const uint4*>(V.levels + V.level_off[j_in] + base + 4 * t);
        uint32_t a = v.x + v.y + v.z + v.w;
        V.levels[V.level_off[j_in + 1] + (base >> 2) + t] = a;
        a += __shfl_xor_sync(0xffffffffu, a, 1);
        a += __shfl_xor_sync(0xffffffffu, a, 2);
        if ((t & 3) == 0) V.levels[V.level_off[j_in + 2] + (base >> 4) + (t >> 2)] = a;
        a += __shfl_xor_sync(0xffffffffu, a, 4);
        a += __shfl_xor_sync(0xffffffffu, a, 8);
        if ((t & 15) == 0) V.levels[V.level_off[j_in + 3] + (base >> 6) + (t >> 4)] = a;
        a += __shfl_xor_sync(0xffffffffu, a, 16);
        if ((t & 31) == 0) buf1[t >> 5] = a;  // the warps' sums
        __syncthreads();
        if (t < kWarps / 2) {
            const uint32_t p = buf1[2 * t] + buf1[2 * t + 1];
            V.levels[V.level_off[j_in + 4] + (base >> 8) + t] = p;
            buf1[kWarps + t] = p;
        }
        __syncthreads();
        if (t == 0) {
            const uint32_t c = buf1[kWarps] + buf1[kWarps + 1] + buf1[kWarps + 2] + buf1[kWarps + 3];
            V.levels[V.level_off[j_in + 5] + (base >> 10)] = c;
            buf0[0] = c;
        }
        __syncthreads();
        j = j_in + 5;
    } else {
        if (4 * t < n)
            *reinterpret_cast<uint4*>(&buf0[4 * t]) =
                *reinterpret_cast<const uint4*>(V.levels + V.level_off[j_in] + base + 4 * t);
        __syncthreads();
        reduce_tree(V, buf0, buf1, j, j_stop, n, base, overflow);
    }
    if (j < j_stop) {
        // levels remain above this chunk's top: the last CTA to finish continues
        __threadfence();
        if (threadIdx.x == 0) *s_last = (atomicAdd(&V.ctrl->reduce_done, 1u) == nchunks - 1);
        __syncthreads();
        if (!*s_last) {
            if (overflow) atomicOr(&V.ctrl->status, kStatusOverflow);
            return false;
        }
        __threadfence();
        const long long m = level_entries(V.size_l2, j);  // == nchunks entries, <= kReduceTop
        for (long long i = threadIdx.x; i < m; i += blockDim.x) buf0[i] = __ldcg(&V.levels[V.level_off[j] + i]);
        __syncthreads();
        reduce_tree(V, buf0, buf1, j, j_stop, m, 0, overflow);
        if (threadIdx.x == 0) V.ctrl->reduce_done = 0;
    }
    if (overflow) atomicOr(&V.ctrl->status, kStatusOverflow);
    if (j == V.jtop && threadIdx.x == 0) V.ctrl->total = buf0[0];
    return j == V.jtop;
}

__global__ void __launch_bounds__(kThreads) reduce_levels(const __grid_constant__ Volume V, int j_in, int j_stop) {
    __shared__ __align__(16) uint32_t buf0[kReduceTop];
    __shared__ uint32_t buf1[kReduceTop / 4];
    __shared__ int s_last;
    wait_prior_grid();
    allow_next_grid();
    reduce_chunk(V, j_in, j_stop, blockIdx.x, gridDim.x, buf0, buf1, &s_last);
}

// Top entry when the whole pyramid is one block (no reduction launch needed).
__global__ void copy_total(const __grid_constant__ Volume V) {
    wait_prior_grid();
    allow_next_grid();
    if (threadIdx.x == 0) V.ctrl->total = V.levels[V.level_off[V.jtop]];
}

// ---------------------------------------------------------------------------
// Batched build.  One classify launch covers the column bricks of every
// volume (CTA = one brick, its volume found in the brick prefix array); one
// reduce launch covers the reduction chunks of every volume (each volume's
// pyramid finished by its own last CTA), and the CTA that completes the last
// volume scans the per-volume counts into output offsets and traversal work
// items.  Volume descriptors are copied into shared memory per CTA.
template <int FT>
__global__ void __launch_bounds__(kThreads) classify_batch_tma(const __grid_constant__ BatchDev B) {
    __shared__ __align__(16) Volume sV;
    const int v = find_segment(B.brick_start, B.nvol, blockIdx.x);
    copy_volume(&sV, B.vols + v, threadIdx.x, blockDim.x);
    __syncthreads();
    const uint32_t lb = blockIdx.x - __ldg(B.brick_start + v);
    const uint32_t per_slab = (uint32_t)sV.nfx * (uint32_t)sV.nfy;
    const int zc = (int)(lb / per_slab);
    const uint32_t r = lb - (uint32_t)zc * per_slab;
    const int fy = (int)(r / (uint32_t)sV.nfx);
    const int fx = (int)(r - (uint32_t)fy * (uint32_t)sV.nfx);
    classify_column_body<FT>(B.tmaps + v, sV, fx, fy, zc);
}

namespace {

// Block-wide exclusive scan (kThreads threads); `total` receives the sum.
template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T x, T* s_warp, T& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    T off = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < kWarps; w++) {
        const T s = s_warp[w];
        if (w < warp) off += s;
        tot += s;
    }
    __syncthreads();
    total = tot;
    return off + inc - x;
}

// Output offsets (exclusive scan of the vertex counts) and traversal work
// items (vertices that fit the output, in items of 32 * rounds).
__device__ void batch_scan(const BatchDev& B) {
    __shared__ unsigned long long s_w64[kWarps];
    __shared__ uint32_t s_w32[kWarps];
    const uint32_t VW = 32u * (uint32_t)B.rounds;
    unsigned long long carry = 0;
    uint32_t ccarry = 0;
    for (int base = 0; base < B.nvol; base += kThreads) {
        const int v = base + (int)threadIdx.x;
        unsigned long long tot = 0;
        if (v < B.nvol) {
            const Ctrl* c = B.vols[v].ctrl;
            tot = __ldcg(&c->total);
        }
        unsigned long long sum64;
        const unsigned long long vb = carry + block_exclusive_scan<unsigned long long>(tot, s_w64, sum64);
        const unsigned long long room = B.capacity > vb ? B.capacity - vb : 0ull;
        const unsigned long long nw = tot < room ? tot : room;
        const uint32_t items = (uint32_t)((nw + VW - 1) / VW);
        uint32_t sum32;
        const uint32_t cs = ccarry + block_exclusive_scan<uint32_t>(items, s_w32, sum32);
        if (v < B.nvol) {
            B.vbase[v] = vb;
            B.chunk_start[v] = cs;
        }
        carry += sum64;
        ccarry += sum32;
    }
    if (threadIdx.x == 0) {
        B.vbase[B.nvol] = carry;
        B.chunk_start[B.nvol] = ccarry;
        B.ctrl->total = carry;
        if (carry > B.capacity) atomicOr(&B.ctrl->status, kStatusCapacity);
        B.ctrl->reduce_done = 0;
        __threadfence();
    }
}

}  // namespace

__global__ void __launch_bounds__(kThreads) reduce_batch(const __grid_constant__ BatchDev B) {
    __shared__ __align__(16) uint32_t buf0[kReduceTop];
    __shared__ uint32_t buf1[kReduceTop / 4];
    __shared__ __align__(16) Volume sV;
    __shared__ int s_last, s_all;
    const int v = find_segment(B.reduce_start, B.nvol, blockIdx.x);
    copy_volume(&sV, B.vols + v, threadIdx.x, blockDim.x);
    __syncthreads();
    const uint32_t c0 = __ldg(B.reduce_start + v);
    const uint32_t nchunks = __ldg(B.reduce_start + v + 1) - c0;
    // every batch volume reaches its top in this launch (jtop - 5 <= 11)
    const bool finished =
        reduce_chunk(sV, kBlockLevel, sV.jtop, (long long)(blockIdx.x - c0), nchunks, buf0, buf1, &s_last);
    if (!finished) return;  // uniform across the CTA
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();  // this volume's total before the batch counter
        s_all = (atomicAdd(&B.ctrl->reduce_done, 1u) == (unsigned)B.nvol - 1u);
    }
    __syncthreads();
    if (s_all) {
        __threadfence();
        batch_scan(B);
    }
}

// ---------------------------------------------------------------------------
// Host launchers
constexpr int kRingBytesF32 = kRingStages * ((36 * 33 * 4 * kLayersPerBox + 127) & ~127) + 128;
constexpr int kRingBytesU8 = kRingStages * ((48 * 33 * kLayersPerBox + 127) & ~127) + 128;

// Resident column-classifier CTAs per SM (shared-memory bound).
static int column_ctas_per_sm() {
    static int n = 0;
    if (n == 0) {
        column_smem_ok();
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, classify_columns<kFieldF32>, kThreads,
                                                          kRingBytesF32) !=
                cudaSuccess ||
            n < 1)
            n = 1;
    }
    return n;
}

cudaError_t launch_classify(const Volume& V, const CUtensorMap* tmap, int max_ctas, cudaStream_t st) {
    if (V.column_layout && tmap) {
        const int nz = (V.cells[2] + V.column_slices - 1) / V.column_slices;
        const int ncolumns = V.nfx * V.nfy * nz;
        // persistent: every resident CTA slot (max_ctas = 16 per SM)
        const int slots = (max_ctas / 16) * column_ctas_per_sm();
        const int grid = ncolumns < slots ? ncolumns : slots;
        if (V.ftype == kFieldF32)
            return launch_dependent(classify_columns<kFieldF32>, grid, kThreads, kRingBytesF32, st, *tmap, V, ncolumns);
        else if (V.ftype == kFieldU8)
            return launch_dependent(classify_columns<kFieldU8>, grid, kThreads, kRingBytesU8, st, *tmap, V, ncolumns);
        else
            return launch_dependent(classify_columns<kFieldUNorm8>, grid, kThreads, kRingBytesU8, st, *tmap, V,
                                    ncolumns);
    } else {
        const long long nb = V.nblocks;
        const int grid = (int)(nb < (long long)max_ctas ? nb : (long long)max_ctas);
        switch (V.ftype) {
            case kFieldF32: classify_blocks<kFieldF32><<<grid, kThreads, 0, st>>>(V); break;
            case kFieldU8: classify_blocks<kFieldU8><<<grid, kThreads, 0, st>>>(V); break;
            case kFieldUNorm8: classify_blocks<kFieldUNorm8><<<grid, kThreads, 0, st>>>(V); break;
            case kFieldF32X4: classify_blocks<kFieldF32X4><<<grid, kThreads, 0, st>>>(V); break;
            default: classify_blocks<kFieldFunctor><<<grid, kThreads, 0, st>>>(V); break;
        }
    }
    return cudaGetLastError();
}

cudaError_t launch_reduce(const Volume& V, cudaStream_t st) {
    if (V.jtop == kBlockLevel) return launch_dependent(copy_total, 1, 32, 0, st, V);
    int j_in = kBlockLevel;
    while (j_in < V.jtop) {
        // one launch reduces 5 levels per CTA plus up to 6 more in the last CTA
        const int j_stop = (V.jtop - j_in <= 11) ? V.jtop : j_in + 5;
        const long long n_in = level_entries(V.size_l2, j_in);
        const long long grid = (n_in + kReduceChunk - 1) / kReduceChunk;
        cudaError_t e = launch_dependent(reduce_levels, (unsigned)grid, kThreads, 0, st, V, j_in, j_stop);
        if (e != cudaSuccess) return e;
        j_in = j_stop;
    }
    return cudaSuccess;
}

cudaError_t launch_classify_batch(const BatchDev& B, int ftype, unsigned int bricks, cudaStream_t st) {
    if (!bricks) return cudaSuccess;
    if (ftype == kFieldF32)
        classify_batch_tma<kFieldF32><<<bricks, kThreads, kRingBytesF32, st>>>(B);
    else if (ftype == kFieldU8)
        classify_batch_tma<kFieldU8><<<bricks, kThreads, kRingBytesU8, st>>>(B);
    else if (ftype == kFieldUNorm8)
        classify_batch_tma<kFieldUNorm8><<<bricks, kThreads, kRingBytesU8, st>>>(B);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_reduce_batch(const BatchDev& B, unsigned int chunks, cudaStream_t st) {
    reduce_batch<<<chunks, kThreads, 0, st>>>(B);
    return cudaGetLastError();
}

bool column_smem_ok() {
    static int configured = 0;
    if (!configured) {
        cudaFuncSetAttribute(classify_columns<kFieldF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRingBytesF32);
        cudaFuncSetAttribute(classify_columns<kFieldU8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRingBytesU8);
        cudaFuncSetAttribute(classify_columns<kFieldUNorm8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kRingBytesU8);
        cudaFuncSetAttribute(classify_batch_tma<kFieldF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRingBytesF32);
        cudaFuncSetAttribute(classify_batch_tma<kFieldU8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRingBytesU8);
        cudaFuncSetAttribute(classify_batch_tma<kFieldUNorm8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kRingBytesU8);
        configured = 1;
    }
    return true;
}

}  // namespace hpmc
