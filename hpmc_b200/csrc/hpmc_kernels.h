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

cudaError_t launch_classify(const Volume& V, const CUtensorMap* tmap, int max_ctas, cudaStream_t st);
cudaError_t launch_reduce(const Volume& V, cudaStream_t st);
cudaError_t launch_traverse(const Volume& V, const TraverseOut& O, int normal_mode, int grid,
                            cudaStream_t st);
cudaError_t launch_adjoint(const Volume& V, const AdjointIO& A, int normal_mode, int grid, cudaStream_t st);
bool column_smem_ok();
int traverse_blocks_per_sm();

}  // namespace hpmc
