// kernels_traverse.cu -- per-vertex HistoPyramid traversal, geometry and the
// adjoint, on sm_100a.
//
// Reference: the traversal vertex shader extractVertex (shadergen.cpp:436-565,
// GL3+ path) driven by HPMCextractVertices (triface.cpp:332-457), one
// invocation per output vertex in batches of 3000 (constants.cpp:198).
//
// Here one persistent grid walks the vertex range; a warp owns 32 consecutive
// vertices per round:
//   1. descent (warp-cooperative): the warp descends the dense levels for the
//      first vertex not covered by its cached block, from the top (cached in
//      shared memory) to the 1024-key block, taking the first child whose
//      running sum exceeds the key exactly as shadergen.cpp:448-467 does.  All
//      lanes walk the same path, so every load is one broadcast transaction;
//      consecutive vertices reuse the block and skip the descent, and a warp
//      that walks out of its block takes the next non-empty one from the
//      following 32 level-5 entries (one coalesced load) when it lies there.
//   2. in-block lookup (warp-cooperative; replaces the base-level steps of
//      shadergen.cpp:469-495): on entering a block the warp turns its 1024
//      codes into the list of active cells (count > 0) with their first
//      vertex, in vertex order; per round a lane's cell is found from the
//      list with one OR-reduction of the cell starts that fall in the
//      round's window and a popcount (no per-vertex search).
//   3. geometry (shadergen.cpp:497-563): edge from the case table, crossing
//      parameter t, position and normal; FP32 arithmetic with a float-float
//      fallback for ill-conditioned normals; coalesced streaming float4
//      stores.
#include <cuda_runtime.h>
#include <cstdint>

#include "hpmc_batch.cuh"
#include "hpmc_device.cuh"
#include "hpmc_fetch.cuh"
#include "hpmc_geometry.cuh"
#include "hpmc_kernels.h"
#include "_gen/hpmc_case_tables.h"

namespace hpmc {

__constant__ uint8_t c_vertex_count_t[256] = HPMC_GEN_VERTEX_COUNT;
__constant__ uint64_t c_edge_nibbles[256] = HPMC_GEN_EDGE_NIBBLES;
__device__ const float g_binary_normals[256 * 16 * 3] = HPMC_GEN_BINARY_NORMALS;
constexpr uint64_t kEdgeGeometry = HPMC_GEN_EDGE_GEOMETRY;

enum { kModeForward = kGeomForward, kModeCentral = kGeomCentral, kModeBinary = kGeomBinary };

namespace {

struct TraverseSmem {
    uint64_t edge[256];
    // active cells (vertex count > 0) of each warp's block, in vertex order:
    // start << 18 | code << 10 | cell (start = first block-relative vertex of
    // the cell, <= 15 * 1024; cell = Morton index of the cell in the block)
    uint32_t act[kWarps][kBlockKeys];
    uint32_t top[kTopCacheEntries];
    uint16_t morton[kBlockKeys];  // cell Morton index in a block -> cx | cy << 8
    uint8_t cnt[256];
};

constexpr size_t kTraverseSmem = sizeof(TraverseSmem);
constexpr size_t kBatchVolOffset = (sizeof(TraverseSmem) + 15) & ~size_t(15);
constexpr size_t kBatchSmem = kBatchVolOffset + kWarps * sizeof(Volume);

// The block a warp is working in: its key-space origin and, for the column
// layout, the lattice cell of its first key (every cell of such a block lies
// in the same slice tile); its active-cell count and the active cell holding
// the next block-relative vertex the warp expects (knext).
struct WarpBlock {
    uint32_t b, base, count;
    uint32_t X0, Y0;
    int ox, oy, oz;
    uint32_t nact, cur, knext;
    bool have;
};

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
    // build).  No early trigger: the next build launches as these CTAs exit.
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

// Warp-cooperative: the active-cell list of block b (S.act[warp]); returns
// its length.  Lane l turns the block's codes 32l .. 32l+31 (Morton order)
// into counts; one warp scan gives every lane its first vertex and first
// list slot.
__device__ __forceinline__ uint32_t load_block(const Volume& V, TraverseSmem& S, int warp, int lane, uint32_t b) {
    const long long slot = block_slot(V, b);
    const uint4* src = reinterpret_cast<const uint4*>(V.arena + slot * kBlockWords) + 2 * lane;
    const uint4 w0 = __ldg(src), w1 = __ldg(src + 1);
    const uint32_t w[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
    uint32_t vsum = 0, amask = 0;
#pragma unroll
    for (int i = 0; i < 32; i++) {
        const uint32_t c = S.cnt[(w[i >> 2] >> (8 * (i & 3))) & 0xffu];
        vsum += c;
        if (c) amask |= 1u << i;
    }
    // one scan of (active cells << 16 | vertices); block totals < 2^16 each
    const uint32_t mine = vsum | ((uint32_t)__popc(amask) << 16);
    uint32_t scan = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, scan, o);
        if (lane >= o) scan += t;
    }
    const uint32_t excl = scan - mine;
    uint32_t vpos = excl & 0xffffu, apos = excl >> 16;
    uint32_t* act = S.act[warp];
    __syncwarp();  // every lane is done with the previous list
#pragma unroll
    for (int k = 0; k < 8; k++) {
        uint32_t am = (amask >> (4 * k)) & 0xfu;
        while (am) {
            const int j = __ffs(am) - 1;
            am &= am - 1u;
            const uint32_t code = (w[k] >> (8 * j)) & 0xffu;
            act[apos++] = (vpos << 18) | (code << 10) | (uint32_t)(32 * lane + 4 * k + j);
            vpos += S.cnt[code];
        }
    }
    __syncwarp();
    return __shfl_sync(0xffffffffu, scan, 31) >> 16;
}

// Warp-uniform: index of the active cell holding block-relative vertex k
// (the last entry whose start is <= k), 32 entries per vote.
__device__ __forceinline__ uint32_t find_active(const uint32_t* act, uint32_t nact, uint32_t k, int lane) {
    for (uint32_t q = 0; q <= nact; q += 32) {
        const uint32_t j = q + (uint32_t)lane;
        const bool le = j < nact && (act[j] >> 18) <= k;
        const uint32_t bal = __ballot_sync(0xffffffffu, le);
        if (bal != 0xffffffffu) return q + (uint32_t)__popc(bal) - 1u;
    }
    return nact - 1u;
}

// Resolved vertex: cell, code, vertex index inside the cell.
struct VertexCell {
    int x, y, z;
    int code;
    int k;
};

// Block B.b with base B.base and count B.count found: load its active-cell
// list and position the warp at block-relative vertex key - B.base.
__device__ __forceinline__ void open_block(const Volume& V, TraverseSmem& S, int warp, int lane, uint32_t key,
                                           WarpBlock& B) {
    B.nact = load_block(V, S, warp, lane, B.b);
    B.X0 = compact32(B.b) << 5;
    B.Y0 = compact32(B.b >> 1) << 5;
    virtual_to_cell(V, B.X0, B.Y0, B.ox, B.oy, B.oz);
    B.have = true;
    const uint32_t k = key - B.base;
    B.cur = k == 0 ? 0u : find_active(S.act[warp], B.nact, k, lane);
    B.knext = k;
}

__device__ __forceinline__ void enter_block(const Volume& V, TraverseSmem& S, int warp, int lane, uint32_t key,
                                            WarpBlock& B) {
    descend(V, S, key, B.b, B.base, B.count);  // uniform across the warp
    open_block(V, S, warp, lane, key, B);
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
__device__ __forceinline__ bool resolve_vertex(const Volume& V, TraverseSmem& S, int warp, int lane, uint32_t v,
                                               bool act, WarpBlock& B, VertexCell& out) {
    unsigned int pending = __ballot_sync(0xffffffffu, act);
    const uint32_t* list = S.act[warp];
    while (pending) {
        const int leader = __ffs(pending) - 1;
        const uint32_t vl = __shfl_sync(0xffffffffu, v, leader);
        if (!B.have || vl < B.base || vl - B.base >= B.count) {
            if (B.have && vl - B.base == B.count && next_sibling(V, lane, B))
                open_block(V, S, warp, lane, vl, B);
            else
                enter_block(V, S, warp, lane, vl, B);
        } else if (vl - B.base != B.knext) {
            B.cur = find_active(list, B.nact, vl - B.base, lane);
            B.knext = vl - B.base;
        }
        const uint32_t k0 = B.knext;
        const uint32_t npend = (uint32_t)__popc(pending);
        const uint32_t left = B.count - k0;
        const uint32_t nm = npend < left ? npend : left;  // lanes leader .. leader+nm-1
        const int d = lane - leader;
        const bool mine = d >= 0 && (uint32_t)d < nm;
        const uint32_t j = B.cur + 1u + (uint32_t)lane;
        const uint32_t pos = (j < B.nact) ? (list[j] >> 18) - k0 : 0xffffffffu;  // >= 1
        const uint32_t starts = __reduce_or_sync(0xffffffffu, pos < 32u ? (1u << pos) : 0u);
        if (mine) {
            const uint32_t idx = B.cur + (uint32_t)__popc(starts & ((2u << d) - 1u));
            const uint32_t e = list[idx];
            out.code = (int)((e >> 10) & 0xffu);
            out.k = (int)(k0 + (uint32_t)d - (e >> 18));
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

// The last CTA to finish resets the queue for the next launch on the stream.
__device__ __forceinline__ void finish_queue(const Volume& V) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&V.ctrl->work_done, 1u) == gridDim.x - 1) {
            V.ctrl->work_next = 0;
            V.ctrl->work_done = 0;
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
template <int FT, int MODE>
__global__ void __launch_bounds__(kThreads, 4) traverse_kernel(const __grid_constant__ Volume V,
                                                               const __grid_constant__ TraverseOut O) {
    extern __shared__ __align__(16) uint8_t s_traverse[];
    TraverseSmem& S = *reinterpret_cast<TraverseSmem*>(s_traverse);
    load_tables(V, S);
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
    for (uint32_t chunk = next_chunk(V, lane); chunk < nchunks; chunk = next_chunk(V, lane)) {
#pragma unroll 1
        for (uint32_t r = 0; r < rounds; r++) {
            const uint32_t v = chunk * VW + 32u * r + lane;
            const bool act = v < N;
            if (!__any_sync(0xffffffffu, act)) break;
            VertexCell c;
            if (!resolve_vertex(V, S, warp, lane, v, act, B, c)) continue;
            const EdgeGeom g = edge_of(S, c);
            float p[3], n[3], t;
            edge_vertex<FT, MODE>(V, g.a, g.axis, c.x, c.y, c.z, g_binary_normals + 3 * (16 * c.code + c.k), p, n,
                                  t);
            const unsigned long long o = V.vertex_base + v;
            if (O.pos) __stcs(O.pos + o, make_float4(p[0], p[1], p[2], 1.0f));
            if (O.nrm) __stcs(O.nrm + o, make_float4(n[0], n[1], n[2], 0.0f));
            if (O.feedback) {
                float2* fb = reinterpret_cast<float2*>(O.feedback + 6ull * o);
                __stcs(fb + 0, make_float2(n[0], n[1]));
                __stcs(fb + 1, make_float2(n[2], p[0]));
                __stcs(fb + 2, make_float2(p[1], p[2]));
            }
            if (O.dbg_cell) O.dbg_cell[o] = make_int4(c.x, c.y, c.z, c.code | (c.k << 8) | (g.edge << 16));
            if (O.dbg_t) O.dbg_t[o] = t;
        }
    }
    finish_queue(V);
}

// ---------------------------------------------------------------------------
// Adjoint: recompute the traversal of each vertex and scatter
// dL/dp . dp/df + dL/dn . dn/df onto the field samples the vertex read.
//   t = (f_a - iso)/(f_a - f_b):  dt/df_a = (iso - f_b)/(f_a - f_b)^2,
//                                 dt/df_b = (f_a - iso)/(f_a - f_b)^2
//   p_axis = (a_axis + t) s_axis
//   forward: n_i = ((1-t)(iso - f(a+e_i)) + t(iso - f(b+e_i))) s_i
//   central: n_i = -1/2((1-t)(f(a+e_i) - f(a-e_i)) + t(f(b+e_i) - f(b-e_i))) s_i
// Clamped samples scatter to the sample that was read.
namespace {
__device__ __forceinline__ void scatter(const Volume& V, float* dfield, const int* a, int dx, int dy, int dz,
                                        float g) {
    const int x = min(max(a[0] + dx, 0), V.lattice[0] - 1);
    const int y = min(max(a[1] + dy, 0), V.lattice[1] - 1);
    const int z = min(max(a[2] + dz, 0), V.lattice[2] - 1);
    atomicAdd(dfield + (long long)z * V.slice_pitch + (long long)y * V.row_pitch + x, g);
}
}  // namespace

template <int FT, int MODE>
__global__ void __launch_bounds__(kThreads, 4) adjoint_kernel(const __grid_constant__ Volume V,
                                                              const __grid_constant__ AdjointIO A) {
    extern __shared__ __align__(16) uint8_t s_traverse[];
    TraverseSmem& S = *reinterpret_cast<TraverseSmem*>(s_traverse);
    __shared__ float S_agg[kWarps][32][6];  // cotangents of lanes sharing an edge
    load_tables(V, S);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned long long total = V.ctrl->total;
    const uint32_t N = (uint32_t)(total < A.count ? total : A.count);
    const float iso = V.iso;
    const uint32_t rounds = item_rounds(N, gridDim.x);
    const uint32_t VW = 32u * rounds;
    const uint32_t nchunks = (N + VW - 1) / VW;
    WarpBlock B;
    B.have = false;
    for (uint32_t chunk = next_chunk(V, lane); chunk < nchunks; chunk = next_chunk(V, lane)) {
#pragma unroll 1
        for (uint32_t r = 0; r < rounds; r++) {
            const uint32_t v = chunk * VW + 32u * r + lane;
            const bool act = v < N;
            if (!__any_sync(0xffffffffu, act)) break;
            VertexCell c;
            const bool have = resolve_vertex(V, S, warp, lane, v, act, B, c);
            // Warp aggregation: vertices on the same edge (a, axis) -- the same
            // crossing emitted by neighbouring triangles -- have the same
            // Jacobian, so their cotangents are summed first and one lane (the
            // lowest of the group) scatters once for all of them.
            EdgeGeom g{};
            float4 dp = make_float4(0.f, 0.f, 0.f, 0.f), dn = dp;
            unsigned long long key = ~0ull - (unsigned long long)lane;  // unique for lanes without a vertex
            if (have) {
                g = edge_of(S, c);
                const unsigned long long o = V.vertex_base + v;
                if (A.dpos) dp = __ldg(A.dpos + o);
                if (A.dnrm) dn = __ldg(A.dnrm + o);
                key = ((((unsigned long long)g.a[2] * (unsigned long long)V.lattice[1] + (unsigned long long)g.a[1]) *
                            (unsigned long long)V.lattice[0] + (unsigned long long)g.a[0]) << 2) | (unsigned)g.axis;
            }
            const unsigned int peers = __match_any_sync(0xffffffffu, key);
            const bool leader = have && (__ffs(peers) - 1 == lane);
            if (__popc(peers) > 1) {
                float* slot = S_agg[warp][lane];
                slot[0] = dp.x; slot[1] = dp.y; slot[2] = dp.z;
                slot[3] = dn.x; slot[4] = dn.y; slot[5] = dn.z;
            }
            __syncwarp();
            if (leader && __popc(peers) > 1) {
                unsigned int rest = peers & (peers - 1u);  // the other lanes of the group
                while (rest) {
                    const float* q = S_agg[warp][__ffs(rest) - 1];
                    dp.x += q[0]; dp.y += q[1]; dp.z += q[2];
                    dn.x += q[3]; dn.y += q[4]; dn.z += q[5];
                    rest &= rest - 1u;
                }
            }
            __syncwarp();
            if (!leader) continue;
            const int ax = g.axis;
            const int ex = ax == 0, ey = ax == 1, ez = ax == 2;
            EdgeField F;
            gather_edge<FT, MODE == kModeCentral>(V, g.a, ax, c.x, c.y, c.z, F);
            const float dpv[3] = {dp.x, dp.y, dp.z};
            const float dnv[3] = {dn.x * V.scale[0], dn.y * V.scale[1], dn.z * V.scale[2]};
            const float va = F.va, vb = F.vb;
            const float den = va - vb;
            const FF tf = ff_ratio_of_diffs(va, iso, va, vb);
            const float t = tf.hi + tf.lo;
            const float omt = 1.0f - t;
            float dLdt = dpv[ax] * V.scale[ax];
            float ga = 0.0f, gb = 0.0f;  // direct contributions to samples a and b
#pragma unroll
            for (int i = 0; i < 3; i++) {
                const int dx = i == 0, dy = i == 1, dz = i == 2;
                const float fa_p = F.ap[i];
                const float fb_p = F.bp[i];
                if (MODE == kModeForward) {
                    dLdt += dnv[i] * (fa_p - fb_p);
                    const float wa = -omt * dnv[i], wb = -t * dnv[i];
                    if (i == ax) gb += wa; else scatter(V, A.dfield, g.a, dx, dy, dz, wa);
                    scatter(V, A.dfield, g.a, ex + dx, ey + dy, ez + dz, wb);
                } else {
                    const float fa_m = F.am[i];
                    const float fb_m = F.bm[i];
                    dLdt += -0.5f * dnv[i] * ((fb_p - fb_m) - (fa_p - fa_m));
                    const float wa = -0.5f * omt * dnv[i], wb = -0.5f * t * dnv[i];
                    if (i == ax) gb += wa; else scatter(V, A.dfield, g.a, dx, dy, dz, wa);
                    scatter(V, A.dfield, g.a, -dx, -dy, -dz, -wa);
                    scatter(V, A.dfield, g.a, ex + dx, ey + dy, ez + dz, wb);
                    if (i == ax) ga -= wb; else scatter(V, A.dfield, g.a, ex - dx, ey - dy, ez - dz, -wb);
                }
            }
            const float inv = 1.0f / (den * den);
            ga += dLdt * (iso - vb) * inv;
            gb += dLdt * (va - iso) * inv;
            scatter(V, A.dfield, g.a, 0, 0, 0, ga);
            scatter(V, A.dfield, g.a, ex, ey, ez, gb);
        }
    }
    finish_queue(V);
}

// ---------------------------------------------------------------------------
// Batched traversal: one persistent grid over the work items of every volume
// (chunk_start, written by the batched reduction).  A warp that takes an item
// of another volume copies that volume's descriptor into its own shared slot;
// the descriptors have top_cached = 0, so the descent reads the dense levels
// through L1 instead of a per-CTA cache.
template <int FT, int MODE>
__global__ void __launch_bounds__(kThreads, 4) traverse_batch(const __grid_constant__ BatchDev Bt,
                                                              const __grid_constant__ TraverseOut O) {
    // dynamic: TraverseSmem, then one volume descriptor per warp
    extern __shared__ __align__(16) uint8_t s_traverse[];
    TraverseSmem& S = *reinterpret_cast<TraverseSmem*>(s_traverse);
    Volume* s_vol = reinterpret_cast<Volume*>(s_traverse + kBatchVolOffset);
    load_base_tables(S);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t VW = 32u * (uint32_t)Bt.rounds;
    const uint32_t nitems = __ldcg(Bt.chunk_start + Bt.nvol);
    const Volume& V = s_vol[warp];
    int cur = -1;
    uint32_t c0 = 0, c1 = 0, N = 0;
    unsigned long long vb = 0;
    WarpBlock B;
    B.have = false;
    for (uint32_t item = next_chunk_batch(Bt, lane); item < nitems; item = next_chunk_batch(Bt, lane)) {
        if (cur < 0 || item < c0 || item >= c1) {
            const int v = find_segment(Bt.chunk_start, Bt.nvol, item);
            __syncwarp();
            copy_volume(&s_vol[warp], Bt.vols + v, lane, 32);
            __syncwarp();
            cur = v;
            c0 = __ldcg(Bt.chunk_start + v);
            c1 = __ldcg(Bt.chunk_start + v + 1);
            vb = __ldcg(Bt.vbase + v);
            const unsigned long long total = __ldcg(&V.ctrl->total);
            const unsigned long long room = Bt.capacity > vb ? Bt.capacity - vb : 0ull;
            N = (uint32_t)(total < room ? total : room);
            B.have = false;
        }
        const uint32_t first = (item - c0) * VW;
#pragma unroll 1
        for (int r = 0; r < Bt.rounds; r++) {
            const uint32_t v = first + 32u * r + lane;
            const bool act = v < N;
            if (!__any_sync(0xffffffffu, act)) break;
            VertexCell c;
            if (!resolve_vertex(V, S, warp, lane, v, act, B, c)) continue;
            const EdgeGeom g = edge_of(S, c);
            float p[3], n[3], t;
            edge_vertex<FT, MODE>(V, g.a, g.axis, c.x, c.y, c.z, g_binary_normals + 3 * (16 * c.code + c.k), p, n,
                                  t);
            const unsigned long long o = vb + v;
            if (O.pos) __stcs(O.pos + o, make_float4(p[0], p[1], p[2], 1.0f));
            if (O.nrm) __stcs(O.nrm + o, make_float4(n[0], n[1], n[2], 0.0f));
        }
    }
    finish_queue_batch(Bt);
}

// ---------------------------------------------------------------------------
// Indexed (welded) output.  No counterpart in the reference, which emits
// triangle soup only.  Every soup vertex lies on a lattice edge (a, axis);
// welding keeps one vertex per edge, numbered in order of first occurrence
// in the soup, and an index per soup vertex (three per triangle, the soup's
// triangle order).
//   mesh_keys   traversal without geometry: the edge key of every soup vertex
//               (and its case / vertex-in-cell, for binary-field normals);
//   mesh_insert open-addressing table key -> smallest soup index (atomicCAS
//               on the key, atomicMin on the index);
//   mesh_first  per soup vertex: that smallest index, and a flag "first";
//   mesh_scan_* exclusive scan of the flags = unique vertex numbers;
//   mesh_emit   indices, and the geometry of each unique vertex computed once
//               from its edge (bit-identical to the soup vertex's).
__device__ __forceinline__ unsigned long long edge_key(const Volume& V, const int a[3], int axis) {
    return ((((unsigned long long)a[2] * (unsigned long long)V.lattice[1]) + (unsigned long long)a[1]) *
                (unsigned long long)V.lattice[0] + (unsigned long long)a[0]) * 3ull + (unsigned long long)axis;
}

__global__ void __launch_bounds__(kThreads, 4) mesh_keys(const __grid_constant__ Volume V, unsigned long long* keys,
                                                         uint16_t* meta, uint32_t count) {
    extern __shared__ __align__(16) uint8_t s_traverse[];
    TraverseSmem& S = *reinterpret_cast<TraverseSmem*>(s_traverse);
    load_tables(V, S);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned long long total = V.ctrl->total;
    const uint32_t N = (uint32_t)(total < count ? total : count);
    const uint32_t rounds = item_rounds(N, gridDim.x);
    const uint32_t VW = 32u * rounds;
    const uint32_t nchunks = (N + VW - 1) / VW;
    WarpBlock B;
    B.have = false;
    for (uint32_t chunk = next_chunk(V, lane); chunk < nchunks; chunk = next_chunk(V, lane)) {
#pragma unroll 1
        for (uint32_t r = 0; r < rounds; r++) {
            const uint32_t v = chunk * VW + 32u * r + lane;
            const bool act = v < N;
            if (!__any_sync(0xffffffffu, act)) break;
            VertexCell c;
            if (!resolve_vertex(V, S, warp, lane, v, act, B, c)) continue;
            const EdgeGeom g = edge_of(S, c);
            keys[v] = edge_key(V, g.a, g.axis);
            meta[v] = (uint16_t)(c.code | (c.k << 8));
        }
    }
    finish_queue(V);
}

constexpr unsigned long long kEmptyKey = ~0ull;

__device__ __forceinline__ uint32_t key_hash(unsigned long long k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    return (uint32_t)k;
}

__global__ void mesh_insert(const unsigned long long* keys, uint32_t n, unsigned long long* tkeys, uint32_t* tvals,
                            uint32_t mask, unsigned int* status) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long key = keys[i];
        uint32_t h = key_hash(key) & mask;
        bool done = false;
        for (uint32_t probe = 0; probe <= mask; probe++) {  // the table has >= 2n slots: ends long before
            const unsigned long long prev = atomicCAS(&tkeys[h], kEmptyKey, key);
            if (prev == kEmptyKey || prev == key) {
                atomicMin(&tvals[h], i);
                done = true;
                break;
            }
            h = (h + 1u) & mask;
        }
        if (!done) atomicOr(status, kStatusCapacity);
    }
}

__device__ __forceinline__ uint32_t table_find(const unsigned long long* tkeys, const uint32_t* tvals, uint32_t mask,
                                               unsigned long long key) {
    uint32_t h = key_hash(key) & mask;
    for (uint32_t probe = 0; probe <= mask; probe++) {
        const unsigned long long k = tkeys[h];
        if (k == key) return tvals[h];
        if (k == kEmptyKey) break;
        h = (h + 1u) & mask;
    }
    return 0xffffffffu;
}

constexpr int kScanItems = 8;                        // per thread
constexpr uint32_t kScanTile = kThreads * kScanItems; // per CTA

__global__ void __launch_bounds__(kThreads) mesh_first(const unsigned long long* keys, uint32_t n,
                                                       const unsigned long long* tkeys, const uint32_t* tvals,
                                                       uint32_t mask, uint32_t* first, uint32_t* scan,
                                                       uint32_t* tile_sums) {
    // first[i] = smallest soup index of i's edge; scan[i] = exclusive count of
    // firsts within the tile; tile_sums[tile] = firsts in the tile
    __shared__ uint32_t s_warp[kWarps];
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t f[kScanItems], sum = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const uint32_t i = base + j;
        uint32_t fi = 0u;
        if (i < n) {
            const uint32_t m = table_find(tkeys, tvals, mask, keys[i]);
            first[i] = m;
            fi = (m == i) ? 1u : 0u;
        }
        f[j] = fi;
        sum += fi;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    uint32_t off = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < kWarps; w++) {
        if (w < warp) off += s_warp[w];
        tot += s_warp[w];
    }
    uint32_t run = off + inc - sum;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const uint32_t i = base + j;
        if (i < n) scan[i] = run;
        run += f[j];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// One CTA: exclusive scan of the tile sums in place; total into *unique.
__global__ void __launch_bounds__(kThreads) mesh_scan_tiles(uint32_t* tile_sums, uint32_t ntiles,
                                                            unsigned long long* unique) {
    __shared__ uint32_t s_warp[kWarps];
    uint32_t carry = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t b = 0; b < ntiles; b += kThreads) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t x = i < ntiles ? tile_sums[i] : 0u;
        uint32_t inc = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        uint32_t off = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < kWarps; w++) {
            if (w < warp) off += s_warp[w];
            tot += s_warp[w];
        }
        if (i < ntiles) tile_sums[i] = carry + off + inc - x;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *unique = carry;
}

template <int FT, int MODE>
__global__ void __launch_bounds__(kThreads) mesh_emit(const __grid_constant__ Volume V, const unsigned long long* keys,
                                                      const uint16_t* meta, uint32_t n, const uint32_t* first,
                                                      const uint32_t* scan, const uint32_t* tile_sums, float4* pos,
                                                      float4* nrm, unsigned long long vcap, uint32_t* indices,
                                                      unsigned long long icap) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t j = first[i];
        if (j >= n) continue;  // not found: the insert reported it
        const uint32_t u = scan[j] + tile_sums[j / kScanTile];
        if (indices && i < icap) indices[i] = u;
        if (j != i || u >= vcap) continue;
        // the unique vertex: geometry from its edge
        const unsigned long long key = keys[i];
        const int axis = (int)(key % 3ull);
        unsigned long long r = key / 3ull;
        int a[3];
        a[0] = (int)(r % (unsigned long long)V.lattice[0]);
        r /= (unsigned long long)V.lattice[0];
        a[1] = (int)(r % (unsigned long long)V.lattice[1]);
        a[2] = (int)(r / (unsigned long long)V.lattice[1]);
        const uint16_t m = meta[i];
        const int code = m & 0xff, k = (m >> 8) & 15;
        float p[3], nn[3], t;
        edge_vertex<FT, MODE>(V, a, axis, a[0], a[1], a[2], g_binary_normals + 3 * (16 * code + k), p, nn, t);
        if (pos) pos[u] = make_float4(p[0], p[1], p[2], 1.0f);
        if (nrm) nrm[u] = make_float4(nn[0], nn[1], nn[2], 0.0f);
    }
}

cudaError_t launch_mesh(const Volume& V, const MeshIO& M, int normal_mode, int traverse_grid, int grid,
                        cudaStream_t st) {
    const uint32_t n = M.count;
    mesh_keys<<<traverse_grid, kThreads, kTraverseSmem, st>>>(V, M.keys, M.meta, n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || n == 0) return e;
    if ((e = cudaMemsetAsync(M.table_keys, 0xff, sizeof(unsigned long long) * (M.table_mask + 1ull), st)) !=
            cudaSuccess ||
        (e = cudaMemsetAsync(M.table_vals, 0xff, sizeof(uint32_t) * (M.table_mask + 1ull), st)) != cudaSuccess)
        return e;
    mesh_insert<<<grid, kThreads, 0, st>>>(M.keys, n, M.table_keys, M.table_vals, M.table_mask, &V.ctrl->status);
    const uint32_t ntiles = (n + kScanTile - 1) / kScanTile;
    mesh_first<<<ntiles, kThreads, 0, st>>>(M.keys, n, M.table_keys, M.table_vals, M.table_mask, M.first, M.scan,
                                            M.tile_sums);
    mesh_scan_tiles<<<1, kThreads, 0, st>>>(M.tile_sums, ntiles, M.unique);
    const int mode = V.binary ? kModeBinary : (normal_mode == kNormalsCentral ? kModeCentral : kModeForward);
#define HPMC_MESH_EMIT(FT_, MODE_)                                                                             \
    mesh_emit<FT_, MODE_><<<grid, kThreads, 0, st>>>(V, M.keys, M.meta, n, M.first, M.scan, M.tile_sums, M.pos,  \
                                                     M.nrm, M.vcap, M.indices, M.icap)
#define HPMC_MESH_CASE(FT_)                                                                                    \
    case FT_:                                                                                                  \
        if (mode == kModeBinary) HPMC_MESH_EMIT(FT_, kModeBinary);                                             \
        else if (mode == kModeCentral) HPMC_MESH_EMIT(FT_, kModeCentral);                                      \
        else HPMC_MESH_EMIT(FT_, kModeForward);                                                                \
        break;
    switch (V.ftype) {
        HPMC_MESH_CASE(kFieldF32)
        HPMC_MESH_CASE(kFieldU8)
        HPMC_MESH_CASE(kFieldUNorm8)
        HPMC_MESH_CASE(kFieldFunctor)
        default: return cudaErrorInvalidValue;
    }
#undef HPMC_MESH_CASE
#undef HPMC_MESH_EMIT
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
cudaError_t launch_traverse(const Volume& V, const TraverseOut& O, int normal_mode, int grid,
                            cudaStream_t st) {
    const int mode = V.binary ? kModeBinary : (normal_mode == kNormalsCentral ? kModeCentral : kModeForward);
#define HPMC_TRAVERSE_CASE(FT_)                                                                              \
    case FT_:                                                                                                \
        if (mode == kModeBinary)                                                                             \
            return launch_dependent(traverse_kernel<FT_, kModeBinary>, grid, kThreads, kTraverseSmem, st, V, O);  \
        if (mode == kModeCentral)                                                                            \
            return launch_dependent(traverse_kernel<FT_, kModeCentral>, grid, kThreads, kTraverseSmem, st, V, O); \
        return launch_dependent(traverse_kernel<FT_, kModeForward>, grid, kThreads, kTraverseSmem, st, V, O);
    switch (V.ftype) {
        HPMC_TRAVERSE_CASE(kFieldF32)
        HPMC_TRAVERSE_CASE(kFieldU8)
        HPMC_TRAVERSE_CASE(kFieldUNorm8)
        HPMC_TRAVERSE_CASE(kFieldFunctor)
        default: return cudaErrorInvalidValue;
    }
#undef HPMC_TRAVERSE_CASE
}

cudaError_t launch_adjoint(const Volume& V, const AdjointIO& A, int normal_mode, int grid, cudaStream_t st) {
    const bool central = normal_mode == kNormalsCentral;
    switch (V.ftype) {
        case kFieldF32:
            if (central) adjoint_kernel<kFieldF32, kModeCentral><<<grid, kThreads, kTraverseSmem, st>>>(V, A);
            else adjoint_kernel<kFieldF32, kModeForward><<<grid, kThreads, kTraverseSmem, st>>>(V, A);
            break;
        case kFieldU8:
            if (central) adjoint_kernel<kFieldU8, kModeCentral><<<grid, kThreads, kTraverseSmem, st>>>(V, A);
            else adjoint_kernel<kFieldU8, kModeForward><<<grid, kThreads, kTraverseSmem, st>>>(V, A);
            break;
        case kFieldUNorm8:
            if (central) adjoint_kernel<kFieldUNorm8, kModeCentral><<<grid, kThreads, kTraverseSmem, st>>>(V, A);
            else adjoint_kernel<kFieldUNorm8, kModeForward><<<grid, kThreads, kTraverseSmem, st>>>(V, A);
            break;
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// The batched traversal needs more than the default 48 KB of dynamic shared memory.
static void configure_batch_smem() {
    static bool done = false;
    if (done) return;
    done = true;
    const int bytes = (int)kBatchSmem;
    cudaFuncSetAttribute(traverse_batch<kFieldF32, kModeCentral>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(traverse_batch<kFieldF32, kModeForward>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(traverse_batch<kFieldU8, kModeCentral>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(traverse_batch<kFieldU8, kModeForward>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(traverse_batch<kFieldUNorm8, kModeCentral>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         bytes);
    cudaFuncSetAttribute(traverse_batch<kFieldUNorm8, kModeForward>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         bytes);
}

cudaError_t launch_traverse_batch(const BatchDev& B, const TraverseOut& O, int ftype, int normal_mode, int grid,
                                  cudaStream_t st) {
    configure_batch_smem();  // set before any capture: the first call comes from traverse_batch_blocks_per_sm
    const bool central = normal_mode == kNormalsCentral;
    switch (ftype) {
        case kFieldF32:
            if (central) traverse_batch<kFieldF32, kModeCentral><<<grid, kThreads, kBatchSmem, st>>>(B, O);
            else traverse_batch<kFieldF32, kModeForward><<<grid, kThreads, kBatchSmem, st>>>(B, O);
            break;
        case kFieldU8:
            if (central) traverse_batch<kFieldU8, kModeCentral><<<grid, kThreads, kBatchSmem, st>>>(B, O);
            else traverse_batch<kFieldU8, kModeForward><<<grid, kThreads, kBatchSmem, st>>>(B, O);
            break;
        case kFieldUNorm8:
            if (central) traverse_batch<kFieldUNorm8, kModeCentral><<<grid, kThreads, kBatchSmem, st>>>(B, O);
            else traverse_batch<kFieldUNorm8, kModeForward><<<grid, kThreads, kBatchSmem, st>>>(B, O);
            break;
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int traverse_batch_blocks_per_sm() {
    configure_batch_smem();
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, traverse_batch<kFieldF32, kModeCentral>, kThreads,
                                                      kBatchSmem) !=
            cudaSuccess ||
        n < 1)
        n = 1;
    return n;
}

int traverse_blocks_per_sm() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, traverse_kernel<kFieldF32, kModeCentral>, kThreads,
                                                      kTraverseSmem) !=
            cudaSuccess ||
        n < 1)
        n = 1;
    return n;
}

}  // namespace hpmc

