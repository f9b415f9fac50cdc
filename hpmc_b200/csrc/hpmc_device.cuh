// hpmc_device.cuh -- device-side data model of the B200 HistoPyramid extractor.
//
// The reference keeps its pyramid as one square RGBA32F mip chain whose base
// level tiles the z-slices in 2-D (hpmc/src/init.cpp:105-130,
// hpmc/src/texfbosetup.cpp:72-92).  Every cell (x,y,z) gets a virtual 2-D
// cell coordinate X = 2*tile_x*(z mod layout_x) + x, Y = 2*tile_y*(z div layout_x) + y
// (shadergen.cpp:103-104, 497-503) and the pyramid's child order
// r,g,b,a = (0,0),(1,0),(0,1),(1,1) (shadergen.cpp:148-153, 215-218) makes the
// vertex order the Morton order of (X, Y), X on the even bits.
//
// Here the same key space is stored compactly:
//   * a "block" is an aligned Morton range of 4^5 = 1024 keys (a 32x32 square
//     of virtual cells);
//   * dense level j (j >= 5) holds, per aligned range of 4^j keys, its vertex
//     count as uint32 -- level j equals the reference's mip level j flattened
//     channel by channel (level j texel t, channel c <-> entry 4*morton(t)+c);
//   * below block level nothing is stored densely: each block with a non-zero
//     count gets an "arena" slot holding its 1024 MC codes in Morton order.
//     A traversal warp that enters the block turns them into the block's
//     active-cell list in its own shared memory -- the cells with vertices,
//     in Morton (= vertex) order, each with its MC code and the
//     block-relative index of its first vertex.  Levels 0..4 of the reference
//     are thus implied by the codes: the count of a Morton range of cells is
//     the difference of two list starts.  Cells of empty blocks are all
//     inside or all outside and are not needed.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "hpmc_config.h"

namespace hpmc {

constexpr int kBlockLevel = 5;       // 4^5 keys per block
constexpr int kBlockKeys = 1024;
constexpr int kMaxLevels = 40;

// Arena slot of a non-empty block: its codes in Morton order, four per word
// (cell 4i + c in byte c of word i), then per Morton tile t of 32 cells
// (t = 0..31) the pair {active-cell mask (bit i = cell 32t + i), vertices} at
// words kSlotTileWord + 2t, +1.
constexpr int kSlotTileWord = kBlockKeys / 4;
constexpr int kSlotWords = kSlotTileWord + 64;
constexpr size_t kSlotBytes = sizeof(uint32_t) * (size_t)kSlotWords;

// Active-cell list of one block (a traversal warp's shared memory): one word
// per cell with vertices, in Morton order,
//     start << 18 | code << 10 | cell
// start = block-relative index of the cell's first vertex (< 15 * 1024),
// code = MC case, cell = Morton index of the cell in the block.  The last
// entry is followed by kListSentinels words of all ones (start 16383, past
// any vertex), so a warp may read the 32 entries after any list position
// without knowing the list's length.
constexpr int kListSentinels = 32;
constexpr int kListWords = kBlockKeys + kListSentinels;
constexpr uint32_t kListSentinel = 0xffffffffu;
constexpr int kListStartShift = 18;

enum FieldType : int {
    kFieldF32 = 0,      // float
    kFieldU8 = 1,       // uint8 read as float(b)
    kFieldUNorm8 = 2,   // uint8 read as b/255 (GL_ALPHA UNSIGNED_BYTE texture)
    kFieldFunctor = 3,  // registered device functor evaluated at texel centres
    kFieldF32X4 = 4,    // float4 (gradient x, y, z, value): a GL RGBA float texture
    kFieldUser = 5,     // a caller's functor type (include/hpmc_functor.cuh), a template argument
};

// Template argument of the kernels when the field is not a caller's functor.
struct NoUserField {};

enum NormalMode : int {
    kNormalsForward = 0,  // reference default: iso - lerp(f(a+e), f(b+e), t)
    kNormalsCentral = 1,  // -lerp(central difference at a, at b, t)
};

// Device control block of one pyramid (one volume).
struct Ctrl {
    unsigned long long total;    // vertex count (top of the pyramid)
    unsigned int reduce_done;    // last-block-done counter of the reduce kernel
    unsigned int status;         // sticky error bits (kStatus*)
    unsigned int written;        // vertices written by the last extraction
    unsigned int work_next;      // traversal work queue: next chunk to hand out
    unsigned int work_done;      // traversal CTAs finished (the last one resets the queue)
    unsigned int col_next;       // column classifier's work queue: next column to claim
    unsigned int col_done;       // column classifier CTAs finished (the last one resets the queue)
    unsigned int extracting;     // nonzero while an extraction of this pyramid runs (traverse_kernel)
    unsigned int pad[3];
};

enum : unsigned int {
    kStatusOverflow = 1u,      // vertex count does not fit the level type
    kStatusCapacity = 2u,      // output buffer smaller than the vertex count
    kStatusTimeout = 8u,       // a bounded wait gave up
};

// Parameters of a registered field functor (custom fetch).
struct FunctorParams {
    int id;          // functor id (hpmc_functors.cuh)
    int count;       // number of meaningful floats in p
    float p[kFunctorMaxParams];
};

// Everything a kernel needs to know about one volume.
struct Volume {
    // field
    const void* field;
    long long row_pitch;     // elements
    long long slice_pitch;   // elements
    int idx32;               // every element index (+ one slice) fits in int32
    int ftype;
    int lattice[3];
    int cells[3];
    float iso;
    int binary;
    int gradient;            // gradient normals: a functor's analytic gradient (HPMC_fetchGrad) or the
                             // .xyz of an RGBA field (shadergen.cpp:260-266, 539-551); scalar
                             // fields read a zero gradient there, as GL's alpha textures do
    float scale[3];          // extent / cells
    double dscale[3];        // extent / cells in FP64 (geometry)
    // layout (init.cpp:72-149); all sizes are powers of two
    int tile_x, tile_y;      // texels per tile (cells per tile = 2x)
    int layout_x, layout_y;
    int size_l2;
    int wx_l2, wy_l2;        // log2 of the cells per tile (2 tile_x, 2 tile_y)
    int lx_l2;               // log2 of layout_x
    int u8_thr;              // uint8 fields: sample below iso  <=>  byte < u8_thr
    // compact pyramid
    int jtop;                          // top dense level: max(5, size_l2 + 1)
    uint32_t* levels;                  // dense levels, top level first
    long long level_off[kMaxLevels];   // entry offset of dense level j (index j), multiple of 4
    long long nblocks;                 // entries of level 5
    int top_cached;                    // leading entries of `levels` the traversal caches in smem
    // Arena slot of a block.  Column layout (every 32x32 block lies inside
    // one slice tile): slot = (z * nfy + fy) * nfx + fx over the real
    // footprints, so only real blocks take memory.  Otherwise slot = block.
    int column_layout;
    int nfx, nfy;                      // 32-cell footprints per slice in x, y
    int column_slices;                 // slices per column CTA
    uint32_t* arena;                   // kSlotWords words (one block's codes) per slot
    long long arena_slots;             // capacity of the arena
    Ctrl* ctrl;
    // optional capture of every cell's code, [cz][cy][cx] (inspection)
    uint8_t* codes_out;
    // custom field
    FunctorParams functor;
    unsigned long long vertex_base;    // first output index of this volume (batched)
    // bounded waits of the column classifier (kWaitLimitNs unless a test lowers it)
    unsigned long long wait_limit_ns;
    // Test hook (failure detection without a fault): the column classifier's
    // producer never issues box `stall_box` of its first column (no expect_tx,
    // no copy), so the consumers' bounded waits run out and the build reports
    // kStatusTimeout.  -1: off.
    int stall_box;
    // The column classifier may start streaming while the previous grid on
    // the stream is still this pyramid's extraction (ctrl->extracting set):
    // the levels and arena it writes are not the ones that extraction reads
    // (two alternating sets) and the field is none of that extraction's
    // outputs.  0: every CTA waits for the previous grid first.
    int overlap;
};

// --- Morton helpers (X on even bits) ---------------------------------------
__host__ __device__ __forceinline__ uint32_t morton_compact(uint64_t v) {
    v &= 0x5555555555555555ull;
    v = (v | (v >> 1)) & 0x3333333333333333ull;
    v = (v | (v >> 2)) & 0x0f0f0f0f0f0f0f0full;
    v = (v | (v >> 4)) & 0x00ff00ff00ff00ffull;
    v = (v | (v >> 8)) & 0x0000ffff0000ffffull;
    v = (v | (v >> 16)) & 0x00000000ffffffffull;
    return (uint32_t)v;
}
// 16-bit value -> even bits of a 32-bit word
__host__ __device__ __forceinline__ uint32_t morton_spread16(uint32_t v) {
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}
// 10-bit Morton index inside a block -> (cx, cy) in 0..31
__host__ __device__ __forceinline__ void morton10(uint32_t m, int& cx, int& cy) {
    uint32_t x = m & 0x155u, y = (m >> 1) & 0x155u;
    x = (x | (x >> 1)) & 0x133u; x = (x | (x >> 2)) & 0x10fu; x = (x | (x >> 4)) & 0x1fu;
    y = (y | (y >> 1)) & 0x133u; y = (y | (y >> 2)) & 0x10fu; y = (y | (y >> 4)) & 0x1fu;
    cx = (int)x;
    cy = (int)y;
}

// Virtual cell (X, Y) -> lattice cell; false for padding (shadergen.cpp:497-503).
__host__ __device__ __forceinline__ bool virtual_to_cell(const Volume& V, uint32_t X, uint32_t Y,
                                                         int& x, int& y, int& z) {
    const uint32_t tu = X >> V.wx_l2, tv = Y >> V.wy_l2;
    x = (int)(X & ((1u << V.wx_l2) - 1u));
    y = (int)(Y & ((1u << V.wy_l2) - 1u));
    if (tu >= (uint32_t)V.layout_x || tv >= (uint32_t)V.layout_y) return false;
    z = (int)((tv << V.lx_l2) | tu);
    return x < V.cells[0] && y < V.cells[1] && z < V.cells[2];
}

__host__ __device__ __forceinline__ long long level_entries(int size_l2, int j) {
    int e = size_l2 + 1 - j;
    return e <= 0 ? 1ll : (1ll << (2 * e));
}

// Column layout: block b -> (slice z, footprint fx, fy); false for padding.
__host__ __device__ __forceinline__ bool column_block(const Volume& V, uint64_t b, int& z, int& fx,
                                                      int& fy) {
    const uint32_t X0 = morton_compact(b) << 5, Y0 = morton_compact(b >> 1) << 5;
    int x0, y0;
    const bool ok = virtual_to_cell(V, X0, Y0, x0, y0, z);
    fx = x0 >> 5;
    fy = y0 >> 5;
    return ok;
}

__host__ __device__ __forceinline__ long long block_slot(const Volume& V, uint64_t b) {
    if (!V.column_layout) return (long long)b;
    int z, fx, fy;
    column_block(V, b, z, fx, fy);
    return ((long long)z * V.nfy + fy) * V.nfx + fx;
}

// Block index of footprint (fx, fy) of slice z (column layout).
__host__ __device__ __forceinline__ uint64_t column_block_index(const Volume& V, int z, int fx, int fy) {
    const uint32_t tu = (uint32_t)z & ((1u << V.lx_l2) - 1u), tv = (uint32_t)z >> V.lx_l2;
    const uint32_t X0 = (tu << V.wx_l2) + 32u * (uint32_t)fx;
    const uint32_t Y0 = (tv << V.wy_l2) + 32u * (uint32_t)fy;
    return (uint64_t)(morton_spread16(X0 >> 5) | (morton_spread16(Y0 >> 5) << 1));
}

// Programmatic dependent launch.  The step's kernels (classify, reduce,
// traverse) are launched with programmatic stream serialization, so a
// kernel's CTAs may become resident while the previous kernel on the stream
// is still running.  Every thread calls wait_prior_grid() before it reads or
// writes global memory that earlier stream work may touch; it returns once
// the previous grid has completed and its writes are visible (at once when
// the launch had no such attribute).  allow_next_grid() lets the next kernel
// launch its CTAs early; they wait in their own wait_prior_grid().  The one
// exception is the column classifier after its own pyramid's extraction
// (Volume::overlap): it touches nothing that extraction reads or writes, so
// its CTAs stream the field at once and wait only before they exit (which
// keeps the completion order of the stream's grids).
__device__ __forceinline__ void wait_prior_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allow_next_grid() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

#ifdef __CUDACC__
// Host: launch `kernel` on `st` with programmatic stream serialization.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                                    const Args&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}
#endif

}  // namespace hpmc
