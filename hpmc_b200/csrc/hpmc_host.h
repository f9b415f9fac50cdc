// hpmc_host.h -- host-side helpers shared by the handle runtime (hpmc_api.cu)
// and the batched runtime (hpmc_batch.cu).
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "hpmc.h"
#include "hpmc_device.cuh"

// HPMCConstants (hpmc/include/hpmc_internal.h:67-80 of the reference holds
// GL limits and shared tables; here: the device and its launch geometry).
struct HPMCConstants {
    uint32_t magic;
    int device;
    int num_sms;
    int traverse_ctas_per_sm;
};

namespace hpmc {
namespace host {

constexpr uint32_t kMagicConstants = 0x48504331u;  // "HPC1"

inline bool valid_constants(const HPMCConstants* c) { return c && c->magic == kMagicConstants; }

// init.cpp:72-149 -- layout of the tiled base level: out = {tile_x, tile_y,
// layout_x, layout_y, log2 size, size}.  False for lattices the reference
// rejects.
bool determine_layout(const int lattice[3], const int cells[3], int out[6]);

// cuTensorMapEncodeTiled through the runtime's driver entry point (null if
// the driver does not provide it).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

inline size_t elem_size(int type) {
    return type == HPMC_SCALAR_F32 ? 4 : type == HPMC_SCALAR_F32X4 ? 16 : 1;
}

// Kernel field type of an HPMCScalarType.
inline int field_type(int scalar_type) {
    return scalar_type == HPMC_SCALAR_F32    ? kFieldF32
           : scalar_type == HPMC_SCALAR_U8   ? kFieldU8
           : scalar_type == HPMC_SCALAR_F32X4 ? kFieldF32X4
                                              : kFieldUNorm8;
}

// Geometry and compact-pyramid members of V from the lattice, the grid and
// the layout L (everything except the field, the device pointers and iso).
// Returns the dense-level entries and the arena slots the volume needs.
void volume_layout(Volume& V, const int lattice[3], const int cells[3], const float extent[3], const int L[6],
                   long long* level_entries_total, long long* arena_slots);

// Slices per column of the persistent column classifier (the single-volume
// paths: the pyramid handle and HPMCextractStatic): the longest column that
// still gives kColumnsPerSm columns per SM for this volume.
int default_column_slices(const Volume& V, int num_sms);

// Tensor map of the column classifier (box 36x33xkLayersPerBox f32 or
// 48x33xkLayersPerBox uint8).  False if the driver refuses it.
bool encode_column_map(CUtensorMap* map, const void* ptr, int scalar_type, const int lattice[3], size_t row_pitch,
                       size_t slice_pitch);

// uint8 fields: the largest byte value below `iso` plus one (f(b) < iso
// <=>  b < threshold, f monotonic).
int u8_threshold(int field_type, float iso);

}  // namespace host
}  // namespace hpmc
