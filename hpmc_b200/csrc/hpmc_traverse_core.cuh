// hpmc_traverse_core.cuh -- the per-vertex HistoPyramid traversal on sm_100a:
// shared-memory layout, case tables, the descent, the active-cell list lookup
// and the extraction kernel template.
//
// Reference: the traversal vertex shader extractVertex (shadergen.cpp:436-565,
// GL3+ path) driven by HPMCextractVertices (triface.cpp:332-457), one
// invocation per output vertex in batches of 3000 (constants.cpp:198).
//
// Included by kernels_traverse.cu (the library's field types) and by
// include/hpmc_functor.cuh (a caller's functor types, instantiated in the
// caller's own translation unit).  Every translation unit gets its own copy
// of the tables in its own device module.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "hpmc_device.cuh"
#include "hpmc_fetch.cuh"
#include "hpmc_geometry.cuh"
#include "hpmc_kernels.h"
#include "_gen/hpmc_case_tables.h"

namespace hpmc {

// Case tables of this translation unit's device module (HPMC's, generated at
// build time from its tables.cpp; see gen_tables.py).
static __constant__ uint8_t c_vertex_count_t[256] = HPMC_GEN_VERTEX_COUNT;
static __constant__ uint64_t c_edge_nibbles[256] = HPMC_GEN_EDGE_NIBBLES;
static __device__ const float g_binary_normals[256 * 16 * 3] = HPMC_GEN_BINARY_NORMALS;
constexpr uint64_t kEdgeGeometry = HPMC_GEN_EDGE_GEOMETRY;

enum { kModeForward = kGeomForward, kModeCentral = kGeomCentral, kModeBinary = kGeomBinary };

namespace {

struct TraverseSmem {
    uint32_t list[kWarps][kListWords];  // per warp: the active-cell list of the block it is in
    uint64_t edge[256];
    uint32_t top[kTopCacheEntries];
    uint16_t morton[kBlockKeys];  // cell Morton index in a block -> cx | cy << 8
    uint8_t cnt[256];
};

constexpr size_t kTraverseSmem = sizeof(TraverseSmem);
constexpr size_t kBatchVolOffset = (sizeof(TraverseSmem) + 15) & ~size_t(15);
constexpr size_t kBatchSmem = kBatchVolOffset + kWarps * sizeof(Volume);

// The block a warp is working in: its key-space origin and, for the column
// layout, the lattice cell of its first key (every cell of such a block lies
// in the same slice tile); its active-cell list (the warp's shared-memory
// area) and the list entry of the cell holding the next block-relative
// vertex the warp expects (knext).
struct WarpBlock {
    uint32_t b, base, count;
    uint32_t X0, Y0;
    int ox, oy, oz;
    uint32_t* list;
    uint32_t cur, knext;
    bool have;
};

// List entry j of a block (clamped to the list area: consistent data never
// reads past the sentinels that follow the last entry).
__device__ __forceinline__ uint32_t list_entry(const uint32_t* list, uint32_t j) {
    return list[j < (uint32_t)kListWords ? j : (uint32_t)(kListWords - 1)];
}

// One warp: block b's active-cell list into `list` from its arena slot (1024
// codes in Morton order, one slot word per quad, and per Morton tile of 32
// cells its active mask and vertices).  Lane l takes tile l: its codes (two
// 16-byte loads) and its mask and vertices (one 8-byte load); one warp scan
// of (cells << 16 | vertices) gives every lane its first list entry and first
// vertex, and the lane writes its active cells in order.  32 sentinels follow
// the last entry.
__device__ __forceinline__ void load_block(const Volume& V, const uint8_t* s_cnt, uint32_t* list, int lane,
                                           uint32_t b) {
    long long slot = block_slot(V, b);
    slot = slot < V.arena_slots ? slot : V.arena_slots - 1;  // in range for consistent data
    const uint32_t* sw = V.arena + slot * kSlotWords;
    const uint4* src = reinterpret_cast<const uint4*>(sw) + 2 * lane;
    const uint4 w0 = __ldg(src), w1 = __ldg(src + 1);
    const uint2 tile = __ldg(reinterpret_cast<const uint2*>(sw + kSlotTileWord) + lane);
    const uint32_t w[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
    const uint32_t amask = tile.x;
    // block totals < 2^16 each
    const uint32_t mine = (tile.y & 0xffffu) | ((uint32_t)__popc(amask) << 16);
    uint32_t scan = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, scan, o);
        if (lane >= o) scan += t;
    }
    const uint32_t excl = scan - mine;
    uint32_t vpos = excl & 0xffffu, apos = excl >> 16;
    __syncwarp();  // every lane is done with the previous list
#pragma unroll
    for (int k = 0; k < 8; k++) {
        uint32_t am = (amask >> (4 * k)) & 0xfu;
        while (am) {
            const int j = __ffs(am) - 1;
            am &= am - 1u;
            const uint32_t code = (w[k] >> (8 * j)) & 0xffu;
            list[apos++] = (vpos << kListStartShift) | (code << 10) | (uint32_t)(32 * lane + 4 * k + j);
            vpos += s_cnt[code];
        }
    }
    list[(__shfl_sync(0xffffffffu, scan, 31) >> 16) + (uint32_t)lane] = kListSentinel;
    __syncwarp();  // the list is visible to the warp
}

__device__ __forceinline__ uint32_t compact32(uint32_t v) {
    v &= 0x55555555u;
    v = (v | (v >> 1)) & 0x33333333u;
    v = (v | (v >> 2)) & 0x0f0f0f0fu;
    v = (v | (v >> 4)) & 0x00ff00ffu;
    v = (v | (v >> 8)) & 0x0000ffffu;
    return v;
}

// Case tables and the block Morton table (no barrier).
__device__ __forceinline__ void load_base_tables(TraverseSmem& S) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        S.cnt[i] = c_vertex_count_t[i];
        S.edge[i] = c_edge_nibbles[i];
    }
    for (int i = threadIdx.x; i < kBlockKeys; i += blockDim.x) {
        int cx, cy;
        morton10((uint32_t)i, cx, cy);
        S.morton[i] = (uint16_t)(cx | (cy << 8));
    }
}

__device__ __forceinline__ void load_tables(const Volume& V, TraverseSmem& S) {
    load_base_tables(S);
    // the pyramid and the control block only after the previous grid (the
    // build)
    wait_prior_grid();
    for (int i = threadIdx.x; i < V.top_cached; i += blockDim.x) S.top[i] = V.levels[i];
    __syncthreads();
}

// Descent through the dense levels (jtop-1 .. 5) for vertex key `key`
// (warp-uniform: every lane passes the same key).
__device__ __forceinline__ void descend(const Volume& V, const TraverseSmem& S, uint32_t key, uint32_t& block,
                                        uint32_t& base, uint32_t& count) {
    uint32_t node = 0;
    base = 0;
    count = V.top_cached ? S.top[0] : V.levels[V.level_off[V.jtop]];
    for (int j = V.jtop - 1; j >= kBlockLevel; j--) {
        const uint32_t idx = (uint32_t)V.level_off[j] + 4u * node;
        const uint4 s = (idx + 4u <= (uint32_t)V.top_cached)
                            ? *reinterpret_cast<const uint4*>(&S.top[idx])
                            : __ldg(reinterpret_cast<const uint4*>(V.levels + idx));
        const uint32_t s0 = s.x, s1 = s0 + s.y, s2 = s1 + s.z;
        const uint32_t c = (uint32_t)(key >= s0) + (uint32_t)(key >= s1) + (uint32_t)(key >= s2);
        const uint32_t skip = c == 0 ? 0u : c == 1 ? s0 : c == 2 ? s1 : s2;
        count = c == 0 ? s.x : c == 1 ? s.y : c == 2 ? s.z : s.w;
        key -= skip;
        base += skip;
        node = 4u * node + c;
    }
    block = node;
}

// Warp-uniform: index of the active cell holding block-relative vertex k
// (the last entry whose start is <= k; the sentinels end the search), 32
// entries per vote.
__device__ __forceinline__ uint32_t find_active(const uint32_t* list, uint32_t k, int lane) {
    for (uint32_t q = 0; q < (uint32_t)kBlockKeys; q += 32) {
        const bool le = (list_entry(list, q + (uint32_t)lane) >> kListStartShift) <= k;
        const uint32_t bal = __ballot_sync(0xffffffffu, le);
        if (bal != 0xffffffffu) return q + (uint32_t)__popc(bal) - 1u;
    }
    return (uint32_t)kBlockKeys - 1u;
}

// Resolved vertex: cell, code, vertex index inside the cell.
struct VertexCell {
    int x, y, z;
    int code;
    int k;
};

// Block B.b with base B.base and count B.count found: its active-cell list
// and the warp's position at block-relative vertex key - B.base.
__device__ __forceinline__ void open_block(const Volume& V, const TraverseSmem& S, int lane, uint32_t key,
                                           WarpBlock& B) {
    load_block(V, S.cnt, B.list, lane, B.b);
    B.X0 = compact32(B.b) << 5;
    B.Y0 = compact32(B.b >> 1) << 5;
    virtual_to_cell(V, B.X0, B.Y0, B.ox, B.oy, B.oz);
    B.have = true;
    const uint32_t k = key - B.base;
    B.cur = k == 0 ? 0u : find_active(B.list, k, lane);
    B.knext = k;
}

__device__ __forceinline__ void enter_block(const Volume& V, const TraverseSmem& S, int lane, uint32_t key,
                                            WarpBlock& B) {
    descend(V, S, key, B.b, B.base, B.count);  // uniform across the warp
    open_block(V, S, lane, key, B);
}

// A warp walking forward out of block B.b: the next block with vertices, if
// it lies among the next 32 level-5 entries (one coalesced load instead of a
// descent through dependent loads).  The blocks in between hold no vertices,
// so the next block's first vertex is B.base + B.count.  Entries of padding
// blocks are zero: every level buffer is cleared when it is allocated and
// only the generic classifier writes those entries (with zero).
__device__ __forceinline__ bool next_sibling(const Volume& V, int lane, WarpBlock& B) {
    const unsigned long long e = (unsigned long long)B.b + 1ull + (unsigned long long)lane;
    const uint32_t c = e < (unsigned long long)V.nblocks ? __ldg(V.levels + V.level_off[kBlockLevel] + e) : 0u;
    const uint32_t m = __ballot_sync(0xffffffffu, c != 0u);
    if (m == 0u) return false;
    const int i = __ffs(m) - 1;
    B.base += B.count;
    B.b += 1u + (uint32_t)i;
    B.count = __shfl_sync(0xffffffffu, c, i);
    return true;
}

// Steps 1-2 for one round of consecutive vertices (lane l holds vertex v,
// lanes with `act` form a prefix of the warp).  Per pass over the lanes that
// lie in the current block, lane j reads list entry cur+1+j; the cells that
// start inside the pass's window of 32 vertices set one bit each, and a
// lane's cell is cur + (starts at or before its offset) -- one popcount
// instead of a search.  Returns `act`.
__device__ __forceinline__ bool resolve_vertex(const Volume& V, const TraverseSmem& S, int lane, uint32_t v,
                                               bool act, WarpBlock& B, VertexCell& out) {
    unsigned int pending = __ballot_sync(0xffffffffu, act);
    while (pending) {
        const int leader = __ffs(pending) - 1;
        const uint32_t vl = __shfl_sync(0xffffffffu, v, leader);
        if (!B.have || vl < B.base || vl - B.base >= B.count) {
            if (B.have && vl - B.base == B.count && next_sibling(V, lane, B))
                open_block(V, S, lane, vl, B);
            else
                enter_block(V, S, lane, vl, B);
        } else if (vl - B.base != B.knext) {
            B.cur = find_active(B.list, vl - B.base, lane);
            B.knext = vl - B.base;
        }
        const uint32_t k0 = B.knext;
        const uint32_t npend = (uint32_t)__popc(pending);
        const uint32_t left = B.count - k0;
        const uint32_t nm = npend < left ? npend : left;  // lanes leader .. leader+nm-1
        const int d = lane - leader;
        const bool mine = d >= 0 && (uint32_t)d < nm;
        // entries after the current one (sentinels: start 16383, never in the window)
        const uint32_t pos = (list_entry(B.list, B.cur + 1u + (uint32_t)lane) >> kListStartShift) - k0;  // >= 1
        const uint32_t starts = __reduce_or_sync(0xffffffffu, pos < 32u ? (1u << pos) : 0u);
        if (mine) {
            const uint32_t idx = B.cur + (uint32_t)__popc(starts & ((2u << d) - 1u));
            const uint32_t e = list_entry(B.list, idx);
            out.code = (int)((e >> 10) & 0xffu);
            out.k = (int)(k0 + (uint32_t)d - (e >> kListStartShift));
            out.k = min(max(out.k, 0), 15);  // in range for consistent data; keeps table reads in bounds
            const uint32_t m = S.morton[e & 0x3ffu];
            const int cx = (int)(m & 0xffu), cy = (int)(m >> 8);
            if (V.column_layout) {
                out.x = B.ox + cx;
                out.y = B.oy + cy;
                out.z = B.oz;
            } else {
                virtual_to_cell(V, B.X0 + (uint32_t)cx, B.Y0 + (uint32_t)cy, out.x, out.y, out.z);
            }
        }
        // the active cell of vertex k0 + nm: the last cell of the pass, or the
        // next one if it starts exactly there
        const bool next_starts = __any_sync(0xffffffffu, pos == nm);
        B.cur += (uint32_t)__popc(starts & ((2u << (nm - 1u)) - 1u)) + (next_starts ? 1u : 0u);
        B.knext = k0 + nm;
        pending &= ~(nm >= 32u ? 0xffffffffu : (((1u << nm) - 1u) << leader));
    }
    return act;
}

struct EdgeGeom {
    int a[3];
    int axis;
    int edge;
};

// Rounds of 32 vertices per work item: one item per warp of the (resident,
// persistent) grid, i.e. a contiguous vertex range per warp.  Every item
// starts with a descent through dependent loads of the upper levels; after
// that the warp walks from block to block, so fewer, longer items are faster
// (measured: one item per warp beats two or four per warp), and per-vertex
// work is uniform enough that the ranges stay balanced.
__device__ __forceinline__ uint32_t item_rounds(uint32_t N, uint32_t ctas) {
    const uint32_t warps = ctas * (uint32_t)kWarps;
    const uint32_t r = (N + 32u * warps - 1u) / (32u * warps);
    return r < 1u ? 1u : r;
}

// Dynamic work queue over vertex chunks (balances the persistent grid):
// lane 0 takes the next chunk for its warp.
__device__ __forceinline__ uint32_t next_chunk(const Volume& V, int lane) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(&V.ctrl->work_next, 1u);
    return __shfl_sync(0xffffffffu, c, 0);
}

// The last CTA to finish resets the queue for the next launch on the stream
// (and, after an extraction, clears the pyramid's extraction flag).
__device__ __forceinline__ void finish_queue(const Volume& V, bool extraction = false) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&V.ctrl->work_done, 1u) == gridDim.x - 1) {
            V.ctrl->work_next = 0;
            V.ctrl->work_done = 0;
            if (extraction) V.ctrl->extracting = 0;
            __threadfence();
        }
    }
}

__device__ __forceinline__ uint32_t next_chunk_batch(const BatchDev& Bt, int lane) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(&Bt.ctrl->work_next, 1u);
    return __shfl_sync(0xffffffffu, c, 0);
}

__device__ __forceinline__ void finish_queue_batch(const BatchDev& Bt) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&Bt.ctrl->work_done, 1u) == gridDim.x - 1) {
            Bt.ctrl->work_next = 0;
            Bt.ctrl->work_done = 0;
            __threadfence();
        }
    }
}

__device__ __forceinline__ EdgeGeom edge_of(const TraverseSmem& S, const VertexCell& c) {
    EdgeGeom g;
    g.edge = (int)((S.edge[c.code] >> (4 * c.k)) & 15ull);
    const uint32_t e = (uint32_t)(kEdgeGeometry >> (5 * g.edge)) & 31u;
    g.a[0] = c.x + (int)(e & 1u);
    g.a[1] = c.y + (int)((e >> 1) & 1u);
    g.a[2] = c.z + (int)((e >> 2) & 1u);
    g.axis = (int)(e >> 3);
    return g;
}

}  // namespace

// ---------------------------------------------------------------------------
// The extraction: every vertex of the last build (up to the outputs'
// capacity), in the reference's vertex order.  UF: a caller's functor type
// when FT == kFieldUser (include/hpmc_functor.cuh).  EXTRA: the interleaved
// feedback and inspection outputs may be set (false: positions and normals
// only, without their per-vertex tests).
template <int FT, int MODE, class UF = NoUserField, bool EXTRA = true>
__global__ void __launch_bounds__(kThreads, 4) traverse_kernel(const __grid_constant__ Volume V,
                                                               const __grid_constant__ TraverseOut O) {
    extern __shared__ __align__(16) uint8_t s_traverse[];
    TraverseSmem& S = *reinterpret_cast<TraverseSmem*>(s_traverse);
    load_tables(V, S);
    // The next grid (normally the next build) may launch now.  The flag,
    // written before any CTA of this one lets it launch, tells that build's
    // column classifier that the previous grid is this extraction, which
    // neither writes the field nor reads the set of levels and arena that the
    // build writes next; the last CTA clears it.
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        V.ctrl->extracting = 1u;
        __threadfence();
    }
    __syncthreads();
    allow_next_grid();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned long long total = V.ctrl->total;
    const uint32_t N = (uint32_t)(total < O.capacity ? total : O.capacity);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (total > O.capacity) atomicOr(&V.ctrl->status, kStatusCapacity);
        V.ctrl->written = N;
    }
    const uint32_t rounds = item_rounds(N, gridDim.x);
    const uint32_t VW = 32u * rounds;
    const uint32_t nchunks = (N + VW - 1) / VW;
    WarpBlock B;
    B.have = false;
    B.list = S.list[warp];
    for (uint32_t chunk = next_chunk(V, lane); chunk < nchunks; chunk = next_chunk(V, lane)) {
#pragma unroll 1
        for (uint32_t r = 0; r < rounds; r++) {
            const uint32_t v = chunk * VW + 32u * r + lane;
            const bool act = v < N;
            if (!__any_sync(0xffffffffu, act)) break;
            VertexCell c;
            if (!resolve_vertex(V, S, lane, v, act, B, c)) continue;
            const EdgeGeom g = edge_of(S, c);
            float p[3], n[3], t;
            edge_vertex<FT, MODE, UF>(V, g.a, g.axis, c.x, c.y, c.z, g_binary_normals + 3 * (16 * c.code + c.k), p,
                                      n, t);
            const unsigned long long o = V.vertex_base + v;
            if (O.pos) __stcs(O.pos + o, make_float4(p[0], p[1], p[2], 1.0f));
            if (O.nrm) __stcs(O.nrm + o, make_float4(n[0], n[1], n[2], 0.0f));
            if (EXTRA && O.feedback) {
                float2* fb = reinterpret_cast<float2*>(O.feedback + 6ull * o);
                __stcs(fb + 0, make_float2(n[0], n[1]));
                __stcs(fb + 1, make_float2(n[2], p[0]));
                __stcs(fb + 2, make_float2(p[1], p[2]));
            }
            if (EXTRA && O.dbg_cell) O.dbg_cell[o] = make_int4(c.x, c.y, c.z, c.code | (c.k << 8) | (g.edge << 16));
            if (EXTRA && O.dbg_t) O.dbg_t[o] = t;
        }
    }
    finish_queue(V, true);
}

}  // namespace hpmc
