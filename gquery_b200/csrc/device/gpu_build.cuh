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

// SNCH on the device-built tree.  A triangle mesh: the unique edges (gpu_silhouette_edges
// with its face_edge and orient outputs) in, 3 n_prims silhouette records (three per
// leaf) out.  A polyline: n_verts in, 2 n_prims vertex records (two per leaf) out.
// Both: max(n_prims - 1, 1) SNCH pair records out.
struct GpuSnchBuild {
    const float *edges19 = nullptr;       // 3D: unique edges, 19 floats each
    const uint32_t *face_edge = nullptr;  // 3D: [3 n_prims] edge of half-edge 3 f + k
    const float *edge_orient = nullptr;   // 3D: [edges] +1 / -1, see gpu_silhouette_edges
    int64_t n_verts = 0;                  // 2D: vertex count
    void *spairs = nullptr;               // gq_spair3_t / gq_spair2_t
    void *sils = nullptr;                 // gq_sile_t / gq_silv_t
};

// verts [nv][dim], index [n_prims][dim] on the device (indices already validated);
// pairs: room for max(n_prims - 1, 1) pair records, prims: n_prims primitive records;
// snch (may be null): the SNCH on the same tree.  Synchronises `st` before
// returning.
cudaError_t gpu_build_bvh(int dim, const float *verts, const int32_t *index, int64_t n_prims, void *pairs,
                          void *prims, GpuBuildResult &res, cudaStream_t st, const GpuSnchBuild *snch = nullptr);

// Unique edges of a triangle mesh in the reference's flat layout (19 floats each, the
// layout of build_flat_silhouette_edges / silhouette_data()), in order of first
// appearance, on the device.  *n_edges receives the count; nothing is written unless
// `out` holds cap_edges >= *n_edges records.  *bad_input = 1 (and nothing else done)
// when a face index is outside [0, nv).  face_edge (optional, [3 nf]) receives the edge
// index of every half-edge; orient (optional, [edges]) +1 where the stored end points
// follow the winding of their last writer's face with its index pair in ascending
// order, else -1 (the faces' normals then point the other way).  Synchronises `st`.
cudaError_t gpu_silhouette_edges(const float *verts, int64_t nv, const int32_t *faces, int64_t nf, float *out,
                                 int64_t cap_edges, int64_t *n_edges, int *bad_input, cudaStream_t st,
                                 uint32_t *face_edge = nullptr, float *orient = nullptr);

}  // namespace gqd
