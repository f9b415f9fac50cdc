// hpmc_host.cu -- host-side helpers shared by the handle and batch runtimes.
#include "hpmc_host.h"

#include <algorithm>
#include <cmath>

namespace hpmc {
namespace host {

bool determine_layout(const int lattice[3], const int cells[3], int out[6]) {
    for (int i = 0; i < 3; i++) {
        if (lattice[i] < 2 || lattice[i] > 16384) return false;  // init.cpp:82-90
        if (lattice[i] <= cells[i]) return false;                // init.cpp:98-103
        if (cells[i] < 1) return false;
    }
    // For a 1-cell axis the reference shifts by -1 (undefined); the exponent
    // is clamped at 0 here.
    auto tile_exp = [](int c) {
        int e = (int)ceilf(log2f(static_cast<float>(c) / 2.0f));  // init.cpp:106-111
        return e < 0 ? 0 : e;
    };
    const int tx = 1 << tile_exp(cells[0]);
    const int ty = 1 << tile_exp(cells[1]);
    const float aspect = static_cast<float>(tx) / static_cast<float>(ty);
    const float lxe = std::max(0.0f, ceilf(log2f(sqrtf(static_cast<float>(cells[2]) / aspect))));
    const int lx = 1 << static_cast<int>(lxe);                     // init.cpp:116-119
    const int ly = (cells[2] + lx - 1) / lx;                       // init.cpp:120-121
    const int l2 = static_cast<int>(ceilf(log2f(static_cast<float>(std::max(tx * lx, ty * ly)))));
    const int size = 1 << l2;                                      // init.cpp:123-128
    out[0] = tx;
    out[1] = ty;
    out[2] = size / tx;                                            // init.cpp:129-130
    out[3] = size / ty;
    out[4] = l2;
    out[5] = size;
    return true;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

void volume_layout(Volume& V, const int lattice[3], const int cells[3], const float extent[3], const int L[6],
                   long long* level_entries_total, long long* arena_slots) {
    for (int i = 0; i < 3; i++) {
        V.lattice[i] = lattice[i];
        V.cells[i] = cells[i];
        V.scale[i] = extent[i] / (float)cells[i];
        V.dscale[i] = (double)extent[i] / (double)cells[i];
    }
    V.tile_x = L[0];
    V.tile_y = L[1];
    V.layout_x = L[2];
    V.layout_y = L[3];
    V.size_l2 = L[4];
    auto ilog2 = [](int v) {
        int e = 0;
        while ((1 << e) < v) e++;
        return e;
    };
    V.wx_l2 = ilog2(2 * L[0]);
    V.wy_l2 = ilog2(2 * L[1]);
    V.lx_l2 = ilog2(L[2]);
    V.jtop = std::max(kBlockLevel, V.size_l2 + 1);
    // dense levels, top first, each padded to a multiple of 4 entries
    long long off = 0;
    for (int j = V.jtop; j >= kBlockLevel; j--) {
        V.level_off[j] = off;
        off += (level_entries(V.size_l2, j) + 3) & ~3ll;
    }
    V.nblocks = level_entries(V.size_l2, kBlockLevel);
    V.top_cached = 0;
    for (int j = V.jtop; j >= kBlockLevel; j--) {
        const long long end = V.level_off[j] + ((level_entries(V.size_l2, j) + 3) & ~3ll);
        if (end > kTopCacheEntries) break;
        V.top_cached = (int)end;
    }
    V.column_layout = (2 * V.tile_x >= 32 && 2 * V.tile_y >= 32) ? 1 : 0;
    V.nfx = (V.cells[0] + 31) / 32;
    V.nfy = (V.cells[1] + 31) / 32;
    V.column_slices = kColumnSliceChoices[3];
    V.wait_limit_ns = kWaitLimitNs;
    V.stall_box = -1;
    *level_entries_total = off;
    *arena_slots = V.column_layout ? (long long)V.nfx * V.nfy * V.cells[2] : V.nblocks;
}

int default_column_slices(const Volume& V, int num_sms) {
    const long long target = (long long)kColumnsPerSm * num_sms;
    for (int zc : kColumnSliceChoices)
        if ((long long)V.nfx * V.nfy * ((V.cells[2] + zc - 1) / zc) >= target) return zc;
    return kColumnSliceChoices[3];
}

bool encode_column_map(CUtensorMap* map, const void* ptr, int scalar_type, const int lattice[3], size_t rp,
                       size_t sp) {
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)lattice[0], (cuuint64_t)lattice[1], (cuuint64_t)lattice[2]};
    const cuuint64_t strides[2] = {(cuuint64_t)rp, (cuuint64_t)sp};
    const bool f32 = scalar_type == HPMC_SCALAR_F32;
    // one ring stage of the column kernel: 32+1 columns padded to a 16-byte
    // row, 32+1 rows, kLayersPerBox layers.  No L2 promotion: a box row is
    // 144 (f32) or 48 (u8) bytes, and wider fills fetch the neighbouring
    // column's samples, which (read with an evict-first policy) rarely stay
    // until that column is classified (measured at 512^3: 1.4 us per step
    // faster than 256-byte promotion, the same as 128-byte)
    const cuuint32_t box[3] = {f32 ? 36u : 48u, 33u, (cuuint32_t)kLayersPerBox};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(map, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(ptr),
               dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int u8_threshold(int field_type, float iso) {
    // host float division is IEEE, the same rounding as the device's
    int n = 0;
    for (int b = 0; b < 256; b++) {
        const float f = (field_type == kFieldUNorm8) ? (float)b / 255.0f : (float)b;
        if (f < iso) n = b + 1;
    }
    return n;
}

}  // namespace host
}  // namespace hpmc
