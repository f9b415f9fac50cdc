// hpmc_config.h -- compile-time limits shared by host and device code.
#pragma once

namespace hpmc {

// Floats of user parameters a registered field functor can take
// (the HPMCgetBuilderProgram / uniform analogue): 32 metaballs x 4 + 8.
constexpr int kFunctorMaxParams = 136;

// Threads per CTA of the classify and traverse kernels.
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// Classification: sample layers per TMA box (one ring stage), ring depth, and
// the slices per column CTA (chosen per volume from kColumnSliceChoices so
// that slices + 1 layers fill whole boxes and the grid covers the GPU).
constexpr int kLayersPerBox = 8;
constexpr int kRingStages = 2;
constexpr int kColumnSliceChoices[4] = {63, 31, 15, 7};
// Columns per SM the single-volume column classifier aims for when it picks
// the column depth: 2 resident CTAs per SM with ~12 columns each, so that
// the persistent CTAs end evenly (fewer, longer columns measured slower).
constexpr int kColumnsPerSm = 24;

// Traversal: top pyramid entries cached in shared memory per CTA
// (levels with <= 1024 entries: 1 + 4 + ... + 1024, each padded to 4).
constexpr int kTopCacheEntries = 1368;
// Vertices per warp work item (R rounds of 32) of the batched traversal (its
// default; the autotuner chooses) and of the host's grid sizing; the
// single-volume traversal gives each warp one contiguous range instead.
constexpr int kTraverseRounds = 8;

// Bounded waits: an mbarrier poll gives up after this long (a TMA box lands
// in microseconds; only a fault in the copy path gets near it).
constexpr unsigned long long kWaitLimitNs = 2000000000ull;

}  // namespace hpmc
