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
//      shadergen.cpp:469-495): the classifier left every non-empty block's
//      1024 codes in Morton order and, per 32-cell Morton tile, its active
//      mask and vertex count in the block's arena slot; a warp entering the
//      block turns them into the block's active-cell list (cells with their
//      first vertex, in vertex order) in its shared memory with one scan, and
//      per round a lane's cell is found from that list with one OR-reduction
//      of the cell starts that fall in the round's window and a popcount (no
//      per-vertex search).
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
#include "hpmc_traverse_core.cuh"

namespace hpmc {

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
    B.list = S.list[warp];
    for (uint32_t chunk = next_chunk(V, lane); chunk < nchunks; chunk = next_chunk(V, lane)) {
#pragma unroll 1
        for (uint32_t r = 0; r < rounds; r++) {
            const uint32_t v = chunk * VW + 32u * r + lane;
            const bool act = v < N;
            if (!__any_sync(0xffffffffu, act)) break;
            VertexCell c;
            const bool have = resolve_vertex(V, S, lane, v, act, B, c);
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
    B.list = S.list[warp];
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
            if (!resolve_vertex(V, S, lane, v, act, B, c)) continue;
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
        HPMC_MESH_CASE(kFieldF32X4)
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
    const bool extra = O.feedback || O.dbg_cell || O.dbg_t;
#define HPMC_TRAVERSE_LAUNCH(FT_, MODE_)                                                                          \
    return extra ? launch_dependent(traverse_kernel<FT_, MODE_, NoUserField, true>, grid, kThreads, kTraverseSmem, \
                                    st, V, O)                                                                     \
                 : launch_dependent(traverse_kernel<FT_, MODE_, NoUserField, false>, grid, kThreads, kTraverseSmem, \
                                    st, V, O);
#define HPMC_TRAVERSE_CASE(FT_)                                             \
    case FT_:                                                               \
        if (mode == kModeBinary) HPMC_TRAVERSE_LAUNCH(FT_, kModeBinary)     \
        if (mode == kModeCentral) HPMC_TRAVERSE_LAUNCH(FT_, kModeCentral)   \
        HPMC_TRAVERSE_LAUNCH(FT_, kModeForward)
    switch (V.ftype) {
        HPMC_TRAVERSE_CASE(kFieldF32)
        HPMC_TRAVERSE_CASE(kFieldU8)
        HPMC_TRAVERSE_CASE(kFieldUNorm8)
        HPMC_TRAVERSE_CASE(kFieldFunctor)
        HPMC_TRAVERSE_CASE(kFieldF32X4)
        default: return cudaErrorInvalidValue;
    }
#undef HPMC_TRAVERSE_CASE
#undef HPMC_TRAVERSE_LAUNCH
}

cudaError_t launch_adjoint(const Volume& V, const AdjointIO& A, int normal_mode, int grid, cudaStream_t st) {
    const bool central = normal_mode == kNormalsCentral;
    // the adjoint's static cotangent buffer plus the traversal's dynamic
    // shared memory pass the 48 KB a launch gets without opting in
    static const bool opted_in = [] {
        const int bytes = (int)kTraverseSmem;
        cudaFuncSetAttribute(adjoint_kernel<kFieldF32, kModeCentral>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        cudaFuncSetAttribute(adjoint_kernel<kFieldF32, kModeForward>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        cudaFuncSetAttribute(adjoint_kernel<kFieldU8, kModeCentral>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        cudaFuncSetAttribute(adjoint_kernel<kFieldU8, kModeForward>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        cudaFuncSetAttribute(adjoint_kernel<kFieldUNorm8, kModeCentral>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             bytes);
        cudaFuncSetAttribute(adjoint_kernel<kFieldUNorm8, kModeForward>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             bytes);
        return true;
    }();
    (void)opted_in;
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

