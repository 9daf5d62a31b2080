// workspace.h -- reduction scratch (per-block partial sums, ticket counter, results).
#pragma once

#include "common.cuh"

namespace qcub {

constexpr int kScratchBlocks = 4096;   // >= SMs x resident blocks of any reducing kernel

struct Scratch {
    double2* partials = nullptr;   // [kScratchBlocks][3][kMaxRhs]
    unsigned* counter = nullptr;   // one ticket counter, zero between launches
    double2* result = nullptr;     // [3][kMaxRhs]
    int max_blocks = 0;
};

// Allocate / free one scratch set (device memory; counter zeroed).
int scratch_alloc(Scratch* s);
void scratch_free(Scratch* s);

// Shared scratch of the current device for the standalone BLAS entry points.
// Calls that use it on different streams at the same time race.
int device_scratch(const Scratch** out);

}  // namespace qcub
