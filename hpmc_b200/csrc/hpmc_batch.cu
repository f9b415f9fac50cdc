// hpmc_batch.cu -- batched extraction: many volumes of uneven lattices and
// iso-values built, counted and traversed by three launches captured in one
// CUDA graph.  No counterpart in the reference (it extracts one volume per
// HistoPyramid handle, hpmc/include/hpmc.h:330-469); per volume the results
// equal the handle path's (same layout, same kernels' arithmetic).
//
// Device memory of a batch (one allocation):
//   batch control block | per-volume control blocks | descriptors |
//   tensor maps | brick, reduce-chunk and work-item prefix arrays |
//   output offsets | dense levels of every volume | block-code arenas
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "hpmc.h"
#include "hpmc_device.cuh"
#include "hpmc_host.h"
#include "hpmc_kernels.h"

using hpmc::BatchCtrl;
using hpmc::BatchDev;
using hpmc::Ctrl;
using hpmc::Volume;

namespace {

constexpr uint32_t kMagicBatch = 0x48504231u;  // "HPB1"

// Tuning choices (autotuner search space).
constexpr int kRoundChoices[5] = {4, 8, 16, 32, 64};
constexpr int kTraverseCtaChoices[3] = {2, 3, 4};

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Autotuner choices of this process per batch signature (scalar type, normal
// mode, SM count and every volume's lattice): a later batch of the same shape
// takes the choice without timing the 72 candidates again.
std::mutex g_tune_mu;
std::map<std::vector<long long>, std::array<int, 3>> g_tune_cache;

}  // namespace

struct HPMCBatch {
    uint32_t magic = kMagicBatch;
    HPMCConstants* constants = nullptr;
    int nvol = 0;
    int ftype = hpmc::kFieldF32;
    int normal_mode = HPMC_NORMALS_FORWARD;
    std::vector<HPMCBatchVolume> src;
    std::vector<Volume> hv;            // descriptors (device pointers filled in)
    std::vector<uint8_t> column;       // volume uses the TMA column classifier
    std::vector<CUtensorMap> tmaps;
    std::vector<uint32_t> brick_start, reduce_start;
    unsigned int bricks = 0, reduce_chunks = 0;
    // device
    unsigned char* d_base = nullptr;
    BatchCtrl* d_bctrl = nullptr;
    Ctrl* d_ctrls = nullptr;
    Volume* d_vols = nullptr;
    CUtensorMap* d_tmaps = nullptr;
    uint32_t* d_brick_start = nullptr;
    uint32_t* d_reduce_start = nullptr;
    uint32_t* d_chunk_start = nullptr;
    unsigned long long* d_vbase = nullptr;
    // tuning (column_slices 0 = automatic)
    int column_slices = 0;
    int traverse_ctas_per_sm = 0;
    int rounds = hpmc::kTraverseRounds;
    bool upload = true;  // descriptors / prefix arrays changed since the last upload
    // captured graph and what it was captured for
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    struct Key {
        float* pos;
        float* nrm;
        size_t cap;
        int mode, zc, ctas, rounds;
    } key{};
    bool have_graph = false;
    cudaStream_t last_stream = nullptr;
};

namespace {

bool valid(const HPMCBatch* b) { return b && b->magic == kMagicBatch; }

void release(HPMCBatch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    b->have_graph = false;
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
    b->capture_stream = nullptr;
    cudaFree(b->d_base);
    b->d_base = nullptr;
}

// Column depth of every volume and the brick prefix array.
void apply_column_slices(HPMCBatch* b) {
    int zc = b->column_slices;
    if (zc == 0) {
        // the longest column that still gives ~12 CTAs per SM over the batch
        const long long target = 12ll * b->constants->num_sms;
        zc = hpmc::kColumnSliceChoices[3];
        for (int c : hpmc::kColumnSliceChoices) {
            long long n = 0;
            for (int v = 0; v < b->nvol; v++)
                if (b->column[v]) n += (long long)b->hv[v].nfx * b->hv[v].nfy * ((b->hv[v].cells[2] + c - 1) / c);
            if (n >= target) {
                zc = c;
                break;
            }
        }
    }
    uint32_t acc = 0;
    for (int v = 0; v < b->nvol; v++) {
        Volume& V = b->hv[v];
        V.column_slices = zc;
        b->brick_start[v] = acc;
        if (b->column[v]) acc += (uint32_t)(V.nfx * V.nfy * ((V.cells[2] + zc - 1) / zc));
    }
    b->brick_start[b->nvol] = acc;
    b->bricks = acc;
    b->upload = true;
}

int max_traverse_ctas() {
    static int n = 0;
    if (n == 0) n = hpmc::traverse_batch_blocks_per_sm();
    return n;
}

int effective_ctas(const HPMCBatch* b) {
    const int maxc = max_traverse_ctas();
    const int c = b->traverse_ctas_per_sm > 0 ? b->traverse_ctas_per_sm : maxc;
    return std::max(1, std::min(c, maxc));
}

BatchDev device_view(const HPMCBatch* b, size_t cap) {
    BatchDev B{};
    B.vols = b->d_vols;
    B.tmaps = b->d_tmaps;
    B.brick_start = b->d_brick_start;
    B.reduce_start = b->d_reduce_start;
    B.vbase = b->d_vbase;
    B.chunk_start = b->d_chunk_start;
    B.ctrl = b->d_bctrl;
    B.capacity = cap;
    B.nvol = b->nvol;
    B.rounds = b->rounds;
    return B;
}

// The launches of one batched extraction, on `st` (captured into the graph).
cudaError_t issue(HPMCBatch* b, float* pos, float* nrm, size_t cap, int traverse_grid, cudaStream_t st) {
    const BatchDev B = device_view(b, cap);
    const int num_sms = b->constants->num_sms;
    cudaError_t e = cudaSuccess;
    for (int v = 0; v < b->nvol && e == cudaSuccess; v++)
        if (!b->column[v]) e = hpmc::launch_classify(b->hv[v], nullptr, num_sms * 16, st);
    if (e == cudaSuccess) e = hpmc::launch_classify_batch(B, b->ftype, b->bricks, st);
    if (e == cudaSuccess) e = hpmc::launch_reduce_batch(B, b->reduce_chunks, st);
    if (e == cudaSuccess) {
        hpmc::TraverseOut O{};
        O.pos = reinterpret_cast<float4*>(pos);
        O.nrm = reinterpret_cast<float4*>(nrm);
        O.capacity = cap;
        e = hpmc::launch_traverse_batch(B, O, b->ftype, b->normal_mode, traverse_grid, st);
    }
    return e;
}

int upload(HPMCBatch* b, cudaStream_t st) {
    if (!b->upload) return HPMC_OK;
    const size_t n1 = sizeof(uint32_t) * (b->nvol + 1);
    if (cudaMemcpyAsync(b->d_vols, b->hv.data(), sizeof(Volume) * b->nvol, cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaMemcpyAsync(b->d_tmaps, b->tmaps.data(), sizeof(CUtensorMap) * b->nvol, cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaMemcpyAsync(b->d_brick_start, b->brick_start.data(), n1, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(b->d_reduce_start, b->reduce_start.data(), n1, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        cudaGetLastError();
        return HPMC_ERR_CUDA;
    }
    b->upload = false;
    return HPMC_OK;
}

int ensure_graph(HPMCBatch* b, float* pos, float* nrm, size_t cap) {
    const HPMCBatch::Key k{pos, nrm, cap, b->normal_mode, b->hv.empty() ? 0 : b->hv[0].column_slices,
                           effective_ctas(b), b->rounds};
    if (b->have_graph && std::memcmp(&k, &b->key, sizeof k) == 0) return HPMC_OK;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    b->have_graph = false;
    cudaGraph_t g = nullptr;
    const int grid = b->constants->num_sms * k.ctas;  // queried before the capture starts
    if (cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return HPMC_ERR_CUDA;
    }
    const cudaError_t e = issue(b, pos, nrm, cap, grid, b->capture_stream);
    const cudaError_t e2 = cudaStreamEndCapture(b->capture_stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return HPMC_ERR_CUDA;
    }
    const cudaError_t e3 = cudaGraphInstantiate(&b->exec, g, 0);
    cudaGraphDestroy(g);
    if (e3 != cudaSuccess) {
        cudaGetLastError();
        b->exec = nullptr;
        return HPMC_ERR_CUDA;
    }
    std::memcpy(&b->key, &k, sizeof k);
    b->have_graph = true;
    return HPMC_OK;
}

int run(HPMCBatch* b, float* pos, float* nrm, size_t cap, cudaStream_t st) {
    int s = upload(b, st);
    if (s == HPMC_OK) s = ensure_graph(b, pos, nrm, cap);
    if (s != HPMC_OK) return s;
    if (cudaGraphLaunch(b->exec, st) != cudaSuccess) {
        cudaGetLastError();
        return HPMC_ERR_CUDA;
    }
    b->last_stream = st;
    return HPMC_OK;
}

}  // namespace

extern "C" {

int HPMCcreateBatch(HPMCConstants* c, const HPMCBatchVolume* volumes, int count, HPMCBatch** out) {
    if (!out) return HPMC_ERR_INVALID_VALUE;
    *out = nullptr;
    if (!hpmc::host::valid_constants(c)) return HPMC_ERR_INVALID_HANDLE;
    if (!volumes || count < 1 || count > (1 << 20)) return HPMC_ERR_INVALID_VALUE;
    const int stype = volumes[0].scalar_type;
    if (stype < HPMC_SCALAR_F32 || stype > HPMC_SCALAR_UNORM8) return HPMC_ERR_INVALID_VALUE;

    auto* b = new (std::nothrow) HPMCBatch;
    if (!b) return HPMC_ERR_OUT_OF_MEMORY;
    b->constants = c;
    b->nvol = count;
    b->ftype = stype == HPMC_SCALAR_F32 ? hpmc::kFieldF32 : stype == HPMC_SCALAR_U8 ? hpmc::kFieldU8
                                                                                     : hpmc::kFieldUNorm8;
    b->src.assign(volumes, volumes + count);
    b->hv.assign(count, Volume{});
    b->column.assign(count, 0);
    b->tmaps.assign(count, CUtensorMap{});
    b->brick_start.assign(count + 1, 0);
    b->reduce_start.assign(count + 1, 0);

    // per-volume layouts and sizes
    std::vector<long long> lev_off(count), arena_off(count);
    long long lev_total = 0, arena_total = 0;
    uint32_t chunks = 0;
    for (int v = 0; v < count; v++) {
        const HPMCBatchVolume& s = volumes[v];
        if (!s.field || s.scalar_type != stype) {
            delete b;
            return HPMC_ERR_INVALID_VALUE;  // one scalar type per batch
        }
        const int lattice[3] = {s.size[0], s.size[1], s.size[2]};
        const int cells[3] = {s.size[0] - 1, s.size[1] - 1, s.size[2] - 1};
        int L[6];
        if (!hpmc::host::determine_layout(lattice, cells, L)) {
            delete b;
            return HPMC_ERR_LAYOUT;
        }
        float ext[3];
        const bool zero_ext = s.extent[0] == 0.f && s.extent[1] == 0.f && s.extent[2] == 0.f;
        for (int i = 0; i < 3; i++) ext[i] = zero_ext ? 1.0f : s.extent[i];
        Volume& V = b->hv[v];
        long long lev = 0, slots = 0;
        hpmc::host::volume_layout(V, lattice, cells, ext, L, &lev, &slots);
        // every volume's pyramid is completed by one reduction launch
        if (V.jtop - hpmc::kBlockLevel > 11) {
            delete b;
            return HPMC_ERR_TOO_LARGE;
        }
        V.top_cached = 0;  // the batched traversal has no per-volume shared cache
        const size_t es = hpmc::host::elem_size(stype);
        const size_t rp = s.row_pitch_bytes ? s.row_pitch_bytes : (size_t)lattice[0] * es;
        const size_t sp = s.slice_pitch_bytes ? s.slice_pitch_bytes : rp * (size_t)lattice[1];
        if (rp % es || sp % es || rp < (size_t)lattice[0] * es || sp < rp * (size_t)lattice[1]) {
            delete b;
            return HPMC_ERR_INVALID_VALUE;
        }
        V.field = s.field;
        V.ftype = b->ftype;
        V.row_pitch = (long long)(rp / es);
        V.slice_pitch = (long long)(sp / es);
        V.idx32 = (V.slice_pitch * ((long long)lattice[2] + 1) < (1ll << 31)) ? 1 : 0;
        V.iso = s.iso;
        V.binary = 0;
        V.u8_thr = hpmc::host::u8_threshold(V.ftype, s.iso);
        if (V.column_layout && ((uintptr_t)s.field % 16 == 0) && rp % 16 == 0 && sp % 16 == 0)
            b->column[v] = hpmc::host::encode_column_map(&b->tmaps[v], s.field, stype, lattice, rp, sp) ? 1 : 0;
        lev_off[v] = lev_total;
        lev_total += lev;  // a multiple of 4 entries: every volume's levels stay 16-byte aligned
        arena_off[v] = arena_total;
        arena_total += slots;
        b->reduce_start[v] = chunks;
        const long long n5 = hpmc::level_entries(V.size_l2, hpmc::kBlockLevel);
        chunks += (uint32_t)std::max(1ll, (n5 + 1023) / 1024);
    }
    b->reduce_start[count] = chunks;
    b->reduce_chunks = chunks;

    // one allocation
    size_t off = 0;
    const size_t o_bctrl = off;
    off = align_up(off + sizeof(BatchCtrl), 256);
    const size_t o_ctrls = off;
    off = align_up(off + sizeof(Ctrl) * count, 256);
    const size_t o_levels = off;
    off = align_up(off + sizeof(uint32_t) * (size_t)lev_total, 256);
    const size_t zero_bytes = off;  // control blocks and levels start at zero
    const size_t o_vols = off;
    off = align_up(off + sizeof(Volume) * count, 256);
    const size_t o_tmaps = off;
    off = align_up(off + sizeof(CUtensorMap) * count, 256);
    const size_t o_brick = off;
    off = align_up(off + sizeof(uint32_t) * (count + 1), 256);
    const size_t o_red = off;
    off = align_up(off + sizeof(uint32_t) * (count + 1), 256);
    const size_t o_chunk = off;
    off = align_up(off + sizeof(uint32_t) * (count + 1), 256);
    const size_t o_vbase = off;
    off = align_up(off + sizeof(unsigned long long) * (count + 1), 256);
    const size_t o_arena = off;
    off += hpmc::kSlotBytes * (size_t)arena_total;
    if (cudaMalloc(&b->d_base, off) != cudaSuccess) {
        cudaGetLastError();
        delete b;
        return HPMC_ERR_OUT_OF_MEMORY;
    }
    if (cudaMemset(b->d_base, 0, zero_bytes) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        release(b);
        delete b;
        return HPMC_ERR_CUDA;
    }
    b->d_bctrl = reinterpret_cast<BatchCtrl*>(b->d_base + o_bctrl);
    b->d_ctrls = reinterpret_cast<Ctrl*>(b->d_base + o_ctrls);
    uint32_t* d_levels = reinterpret_cast<uint32_t*>(b->d_base + o_levels);
    b->d_vols = reinterpret_cast<Volume*>(b->d_base + o_vols);
    b->d_tmaps = reinterpret_cast<CUtensorMap*>(b->d_base + o_tmaps);
    b->d_brick_start = reinterpret_cast<uint32_t*>(b->d_base + o_brick);
    b->d_reduce_start = reinterpret_cast<uint32_t*>(b->d_base + o_red);
    b->d_chunk_start = reinterpret_cast<uint32_t*>(b->d_base + o_chunk);
    b->d_vbase = reinterpret_cast<unsigned long long*>(b->d_base + o_vbase);
    uint32_t* d_arena = reinterpret_cast<uint32_t*>(b->d_base + o_arena);
    for (int v = 0; v < count; v++) {
        Volume& V = b->hv[v];
        V.levels = d_levels + lev_off[v];
        V.arena = d_arena + (size_t)hpmc::kSlotWords * (size_t)arena_off[v];
        V.arena_slots = (v + 1 < count ? arena_off[v + 1] : arena_total) - arena_off[v];
        V.ctrl = b->d_ctrls + v;
    }
    apply_column_slices(b);
    *out = b;
    return HPMC_OK;
}

void HPMCdestroyBatch(HPMCBatch* b) {
    if (!valid(b)) return;
    cudaDeviceSynchronize();
    release(b);
    b->magic = 0;
    delete b;
}

int HPMCbatchSetIsoValues(HPMCBatch* b, const GLfloat* iso) {
    if (!valid(b)) return HPMC_ERR_INVALID_HANDLE;
    if (!iso) return HPMC_ERR_INVALID_VALUE;
    for (int v = 0; v < b->nvol; v++) {
        b->hv[v].iso = iso[v];
        b->hv[v].u8_thr = hpmc::host::u8_threshold(b->hv[v].ftype, iso[v]);
        b->src[v].iso = iso[v];
    }
    b->upload = true;
    return HPMC_OK;
}

int HPMCbatchSetNormalMode(HPMCBatch* b, int mode) {
    if (!valid(b)) return HPMC_ERR_INVALID_HANDLE;
    if (mode != HPMC_NORMALS_FORWARD && mode != HPMC_NORMALS_CENTRAL) return HPMC_ERR_INVALID_VALUE;
    b->normal_mode = mode;
    return HPMC_OK;
}

int HPMCbatchSetTuning(HPMCBatch* b, int column_slices, int traverse_ctas_per_sm, int rounds) {
    if (!valid(b)) return HPMC_ERR_INVALID_HANDLE;
    const bool zc_ok = column_slices == 0 || std::find(std::begin(hpmc::kColumnSliceChoices),
                                                       std::end(hpmc::kColumnSliceChoices),
                                                       column_slices) != std::end(hpmc::kColumnSliceChoices);
    if (!zc_ok || traverse_ctas_per_sm < 0 || rounds < 0 || rounds > 64) return HPMC_ERR_INVALID_VALUE;
    b->column_slices = column_slices;
    b->traverse_ctas_per_sm = traverse_ctas_per_sm;
    b->rounds = rounds ? rounds : hpmc::kTraverseRounds;
    apply_column_slices(b);
    return HPMC_OK;
}

int HPMCbatchGetTuning(HPMCBatch* b, int out[3]) {
    if (!valid(b)) return HPMC_ERR_INVALID_HANDLE;
    if (!out) return HPMC_ERR_INVALID_VALUE;
    out[0] = b->hv[0].column_slices;
    out[1] = effective_ctas(b);
    out[2] = b->rounds;
    return HPMC_OK;
}

int HPMCbatchSetTestStall(HPMCBatch* b, int volume, int box, unsigned int wait_limit_us) {
    if (!valid(b)) return HPMC_ERR_INVALID_HANDLE;
    if (volume < 0 || volume >= b->nvol) return HPMC_ERR_INVALID_VALUE;
    for (int v = 0; v < b->nvol; v++) {
        b->hv[v].stall_box = (v == volume && box >= 0) ? box : -1;
        b->hv[v].wait_limit_ns = wait_limit_us ? 1000ull * wait_limit_us : hpmc::kWaitLimitNs;
    }
    b->upload = true;
    return HPMC_OK;
}

int HPMCbatchExtract(HPMCBatch* b, float* positions, float* normals, size_t capacity_vertices, void* cuda_stream) {
    if (!valid(b)) return HPMC_ERR_INVALID_HANDLE;
    if ((positions && (uintptr_t)positions % 16) || (normals && (uintptr_t)normals % 16))
        return HPMC_ERR_INVALID_VALUE;
    return run(b, positions, normals, capacity_vertices, static_cast<cudaStream_t>(cuda_stream));
}

int HPMCbatchGetDeviceOffsets(HPMCBatch* b, const unsigned long long** device_offsets) {
    if (!valid(b)) return HPMC_ERR_INVALID_HANDLE;
    if (!device_offsets) return HPMC_ERR_INVALID_VALUE;
    *device_offsets = b->d_vbase;
    return HPMC_OK;
}

int HPMCbatchGetOffsets(HPMCBatch* b, unsigned long long* host_offsets) {
    if (!valid(b)) return HPMC_ERR_INVALID_HANDLE;
    if (!host_offsets) return HPMC_ERR_INVALID_VALUE;
    BatchCtrl bc;
    if (cudaStreamSynchronize(b->last_stream) != cudaSuccess ||
        cudaMemcpy(host_offsets, b->d_vbase, sizeof(unsigned long long) * (b->nvol + 1), cudaMemcpyDeviceToHost) !=
            cudaSuccess ||
        cudaMemcpy(&bc, b->d_bctrl, sizeof bc, cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return HPMC_ERR_CUDA;
    }
    // timeouts of the column classifier and overflows are recorded per volume
    std::vector<Ctrl> cs(b->nvol);
    if (cudaMemcpy(cs.data(), b->d_ctrls, sizeof(Ctrl) * b->nvol, cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return HPMC_ERR_CUDA;
    }
    unsigned int st = bc.status;
    for (const Ctrl& c : cs) st |= c.status;
    if (st) {
        // every status bit is reported once: clear them for the next extraction
        const unsigned int clear = 0;
        cudaMemcpy(&b->d_bctrl->status, &clear, sizeof clear, cudaMemcpyHostToDevice);
        for (int v = 0; v < b->nvol; v++)
            if (cs[v].status) cudaMemcpy(&b->d_ctrls[v].status, &clear, sizeof clear, cudaMemcpyHostToDevice);
    }
    if (st & hpmc::kStatusTimeout) return HPMC_ERR_TIMEOUT;
    if (st & hpmc::kStatusOverflow) return HPMC_ERR_OVERFLOW;
    if (st & hpmc::kStatusCapacity) return HPMC_ERR_CAPACITY;
    return HPMC_OK;
}

int HPMCbatchAutotune(HPMCBatch* b, float* positions, float* normals, size_t capacity_vertices, void* cuda_stream,
                      int chosen[3]) {
    if (!valid(b)) return HPMC_ERR_INVALID_HANDLE;
    std::vector<long long> key{b->ftype, b->normal_mode, b->constants->num_sms, b->nvol};
    for (const HPMCBatchVolume& v : b->src) key.insert(key.end(), {v.size[0], v.size[1], v.size[2]});
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            b->column_slices = it->second[0];
            b->traverse_ctas_per_sm = it->second[1];
            b->rounds = it->second[2];
            apply_column_slices(b);
            if (chosen) std::memcpy(chosen, it->second.data(), sizeof(int) * 3);
            return HPMC_OK;
        }
    }
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError();
        return HPMC_ERR_CUDA;
    }
    const int maxc = max_traverse_ctas();
    float best = 1e30f;
    int bz = 0, bc = 0, br = hpmc::kTraverseRounds;
    int status = HPMC_OK;
    for (int zc : hpmc::kColumnSliceChoices) {
        for (int ctas : kTraverseCtaChoices) {
            if (ctas > maxc) continue;
            for (int r : kRoundChoices) {
                b->column_slices = zc;
                b->traverse_ctas_per_sm = ctas;
                b->rounds = r;
                apply_column_slices(b);
                status = run(b, positions, normals, capacity_vertices, st);  // warm-up (and capture)
                if (status != HPMC_OK) break;
                constexpr int kReps = 3;
                cudaEventRecord(e0, st);
                for (int i = 0; i < kReps && status == HPMC_OK; i++)
                    status = run(b, positions, normals, capacity_vertices, st);
                cudaEventRecord(e1, st);
                float ms = 0.f;
                if (status != HPMC_OK || cudaEventSynchronize(e1) != cudaSuccess ||
                    cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                    if (status == HPMC_OK) status = HPMC_ERR_CUDA;
                    break;
                }
                if (ms < best) {
                    best = ms;
                    bz = zc;
                    bc = ctas;
                    br = r;
                }
            }
            if (status != HPMC_OK) break;
        }
        if (status != HPMC_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaGetLastError();
    b->column_slices = bz;
    b->traverse_ctas_per_sm = bc;
    b->rounds = br;
    apply_column_slices(b);
    if (status != HPMC_OK) return status;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = {bz, bc, br};
    }
    if (chosen) {
        chosen[0] = bz;
        chosen[1] = bc;
        chosen[2] = br;
    }
    return HPMC_OK;
}

}  // extern "C"
