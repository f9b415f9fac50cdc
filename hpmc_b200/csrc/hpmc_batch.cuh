// hpmc_batch.cuh -- device helpers of the batched extractor: many volumes of
// different lattices and iso-values in one classify, one reduce and one
// traversal launch.
//
// Every volume keeps its own reference layout, dense levels, arena and
// control block (a segmented pyramid: per-volume pointers into shared
// allocations).  Work lists are prefix arrays over the volumes: CTA or work
// item i belongs to the last volume v with start[v] <= i.
#pragma once
#include <cstdint>

#include "hpmc_device.cuh"
#include "hpmc_kernels.h"

namespace hpmc {

// Last v in [0, n) with start[v] <= i (start is non-decreasing, start[0] = 0).
__device__ __forceinline__ int find_segment(const uint32_t* start, int n, uint32_t i) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(start + mid) <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Copy of a volume descriptor into shared memory by `nthreads` threads
// numbered `t` (a CTA or a warp).
__device__ __forceinline__ void copy_volume(Volume* dst, const Volume* src, int t, int nthreads) {
    static_assert(sizeof(Volume) % 8 == 0, "Volume is copied in 8-byte words");
    const uint2* s = reinterpret_cast<const uint2*>(src);
    uint2* d = reinterpret_cast<uint2*>(dst);
    for (int i = t; i < (int)(sizeof(Volume) / 8); i += nthreads) d[i] = __ldg(s + i);
}

}  // namespace hpmc
