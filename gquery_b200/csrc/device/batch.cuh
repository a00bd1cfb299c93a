// Batched queries over many scenes in one launch (batch.cu).
#pragma once

#include "queries.cuh"

namespace gqd {

// Queries of one kind: query q belongs to scene[q] (an index into the batch's scenes).
struct BatchKind {
    gq_vecs a{};             // points / ray origins
    gq_vecs b{};             // ray directions
    const float *r_max = nullptr;
    const int32_t *scene = nullptr;
    int64_t n = 0;
    const int32_t *perm = nullptr;  // filled by batch_run: sorted order
};

#define GQ_BATCH_SKIP (-1)       // scene index of a padding slot: no traversal, outputs untouched
#define GQ_BATCH_ERR_SCENE 1    // a query named a scene outside the batch
#define GQ_BATCH_ERR_NO_SNCH 2  // a silhouette query named a scene built without SNCH

// Closest-point mode of batch_run from GQ_BATCH_* flags: 1 warp-coherent, 0 one lane
// per query in the reference order, 2 the same with queries past a visit budget
// handed to one warp each.
inline int cp_mode_of(int flags) {
    return (flags & GQ_BATCH_CP_SPLIT) ? 2 : (flags & GQ_BATCH_CP_EXACT) ? 0 : 1;
}

// Silhouette mode of batch_run from GQ_BATCH_* flags.
inline int sil_mode_of(int flags) {
    return (flags & GQ_BATCH_SIL_SPLIT) ? 3 : (flags & GQ_BATCH_SIL_EXACT) ? 0 : (flags & GQ_BATCH_SIL_WARP) ? 2 : 1;
}

// Device scratch for batch_run with at most max_n queries of each kind.
size_t batch_scratch_bytes(int64_t max_n);

// kinds[0] closest point, kinds[1] rays, kinds[2] silhouettes (n = 0 to skip a kind).
// ray_wide: rays on the quantised 8-wide BVH (every scene must have it); cp_mode:
// closest points as cp_mode_of; sil_mode: silhouettes 1 warp-coherent, 2 one query per
// warp, 0 reference order per lane, 3 the same with long traversals handed to a warp;
// grid_share in (0, 1) caps the persistent grid at that share of the GPU's resident
// blocks, so a launch on another stream can run beside it; block: threads per block of
// the batch and hand-over kernels, 128 or 32 (one warp: a launch beside one-warp
// silhouette blocks then fits in the room any one of them leaves); sort: queries in
// (scene, Morton) order, else in their given order with one small launch instead of the
// keys and the radix sort (for small steps, whose launches should need little room).
// No allocation and no host synchronisation: the call can be recorded in a CUDA graph.
cudaError_t batch_run(const DevScene *scenes_dev, int n_scenes, int dim, BatchKind kinds[3], const gq_cp_out &cp_out,
                      const gq_ray_out &ray_out, const gq_sil_out &sil_out, int ray_wide, int cp_mode,
                      int sil_mode, float grid_share, int block, bool sort, void *scratch, int64_t max_n,
                      int32_t *err, cudaStream_t st);

}  // namespace gqd
