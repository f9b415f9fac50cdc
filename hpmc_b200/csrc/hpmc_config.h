// hpmc_config.h -- compile-time limits shared by host and device code.
#pragma once

namespace hpmc {

// Floats of user parameters a registered field functor can take
// (the HPMCgetBuilderProgram / uniform analogue): 32 metaballs x 4 + 8.
constexpr int kFunctorMaxParams = 136;

// Threads per CTA of the classify and traverse kernels.
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// Classification: slices per column CTA and TMA ring depth.
constexpr int kColumnSlices = 32;
constexpr int kRingStages = 6;

// Traversal: top pyramid entries cached in shared memory per CTA
// (levels with <= 1024 entries: 1 + 4 + ... + 1024, each padded to 4).
constexpr int kTopCacheEntries = 1368;
// Vertices per warp work item (R rounds of 32).
constexpr int kTraverseRounds = 4;

// Bounded waits: iterations of an mbarrier poll before giving up.
constexpr unsigned int kSpinLimit = 1u << 26;

}  // namespace hpmc
