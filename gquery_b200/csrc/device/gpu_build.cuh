// Binary BVH built on the device (gpu_build.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../../include/gq.h"
#include "../layout.h"

namespace gqd {

struct GpuBuildResult {
    int32_t root_ref = 0;
    float root_lo[3] = {0.f, 0.f, 0.f}, root_hi[3] = {0.f, 0.f, 0.f};
    int32_t max_depth = 0;  // internal ancestors of the deepest leaf
};

// verts [nv][dim], index [n_prims][dim] on the device (indices already validated);
// pairs: room for max(n_prims - 1, 1) pair records, prims: n_prims primitive records.
// Synchronises `st` before returning.
cudaError_t gpu_build_bvh(int dim, const float *verts, const int32_t *index, int64_t n_prims, void *pairs,
                          void *prims, GpuBuildResult &res, cudaStream_t st);

}  // namespace gqd
