// hpmc_kernels.h -- host-side launch interface of the sm_100a kernels.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "hpmc_device.cuh"

namespace hpmc {

// Output streams of one extraction.
struct TraverseOut {
    float4* pos;                   // x, y, z, 1 per vertex (may be null)
    float4* nrm;                   // nx, ny, nz, 0 per vertex (may be null)
    float* feedback;               // interleaved N3F_V3F, 6 floats per vertex (may be null)
    unsigned long long capacity;   // vertices the outputs can hold
    int4* dbg_cell;                // optional: x, y, z, code | k << 8 | edge << 16
    float* dbg_t;                  // optional: edge parameter t
};

// Adjoint inputs/outputs: dL/dp and dL/dn per vertex (float4, w ignored) and
// dL/df accumulated into a float lattice of the field's shape (dense, pitch
// = the field's pitches).
struct AdjointIO {
    const float4* dpos;
    const float4* dnrm;
    float* dfield;
    unsigned long long count;      // vertices to differentiate (<= vertex count)
};

// Batch-wide control block (device).
struct BatchCtrl {
    unsigned int reduce_done;     // volumes whose pyramid is complete (the last one scans)
    unsigned int work_next;       // traversal work queue: next item to hand out
    unsigned int work_done;       // traversal CTAs finished (the last one resets the queue)
    unsigned int status;          // sticky kStatus* bits of the batch
    unsigned long long total;     // vertices of all volumes
};

// Kernel view of a batch (all arrays in device memory).
struct BatchDev {
    const Volume* vols;            // per-volume descriptors (top_cached = 0)
    const CUtensorMap* tmaps;      // per-volume column tensor maps (64-byte aligned)
    const uint32_t* brick_start;   // nvol + 1: column bricks before volume v
    const uint32_t* reduce_start;  // nvol + 1: reduction chunks before volume v
    unsigned long long* vbase;     // nvol + 1: first output vertex of volume v (written by the reduction)
    uint32_t* chunk_start;         // nvol + 1: traversal work items before volume v (written by the reduction)
    BatchCtrl* ctrl;
    unsigned long long capacity;   // vertices the outputs can hold
    int nvol;
    int rounds;                    // traversal rounds of 32 vertices per work item
};

// Indexed-mesh extraction: scratch and outputs (device).
struct MeshIO {
    uint32_t count;                  // soup vertices (the vertex count of the build)
    unsigned long long* keys;        // count: edge key per soup vertex
    uint16_t* meta;                  // count: case | vertex-in-cell << 8
    unsigned long long* table_keys;  // table_mask + 1 (>= 2 count, power of two)
    uint32_t* table_vals;
    uint32_t table_mask;
    uint32_t* first;                 // count
    uint32_t* scan;                  // count
    uint32_t* tile_sums;             // count / 2048 + 1
    unsigned long long* unique;      // 1: unique vertices
    float4* pos;                     // unique vertices (may be null)
    float4* nrm;
    unsigned long long vcap;
    uint32_t* indices;               // one per soup vertex (may be null)
    unsigned long long icap;
};

cudaError_t launch_mesh(const Volume& V, const MeshIO& M, int normal_mode, int traverse_grid, int grid,
                        cudaStream_t st);
cudaError_t launch_classify(const Volume& V, const CUtensorMap* tmap, int max_ctas, cudaStream_t st);
cudaError_t launch_classify_batch(const BatchDev& B, int ftype, unsigned int bricks, cudaStream_t st);
cudaError_t launch_reduce_batch(const BatchDev& B, unsigned int chunks, cudaStream_t st);
cudaError_t launch_traverse_batch(const BatchDev& B, const TraverseOut& O, int ftype, int normal_mode, int grid,
                                  cudaStream_t st);
int traverse_batch_blocks_per_sm();
cudaError_t launch_reduce(const Volume& V, cudaStream_t st);
cudaError_t launch_traverse(const Volume& V, const TraverseOut& O, int normal_mode, int grid,
                            cudaStream_t st);
cudaError_t launch_adjoint(const Volume& V, const AdjointIO& A, int normal_mode, int grid, cudaStream_t st);
bool column_smem_ok();
int traverse_blocks_per_sm();

}  // namespace hpmc
