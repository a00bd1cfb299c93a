// Host-side launchers of the query kernels (implemented in queries.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../../include/gq.h"
#include "../layout.h"

namespace gqd {

// Device view of one scene.
struct DevScene {
    int dim;
    const void *pairs;   // gq_pair2_t / gq_pair3_t
    const void *prims;   // gq_seg_t / gq_tri_t
    const gq_tsph_t *spheres;  // 3D: bounding sphere per ordered triangle
    int32_t root_ref;
    float root_lo[3], root_hi[3];
    const void *wnodes;  // gq_wnode2_t / gq_wnode3_t (may be null)
    const void *wq16 = nullptr;  // gq_wq16_2_t / gq_wq16_3_t: 16-bit bounds of the same nodes (may be null)
    int32_t wroot_ref;
    const void *spairs;  // gq_spair2_t / gq_spair3_t (may be null)
    const void *sils;    // gq_silv_t / gq_sile_t
    int64_t n_sils = 0;  // records in sils
    int32_t sroot_ref;
    const float *verts;  // original vertices [nv][D] (brute force)
    const int32_t *index;  // original primitives [np][D]
    int64_t n_prims;
    float coord_bound;   // largest |coordinate| of any vertex
    int32_t *err;        // device error word
    int32_t stack_cap = 1 << 30;  // entries a traversal stack may hold (the compiled sizes when larger); a walk
                                  // that needs more stops, its query is a miss and GQ_DEVERR_STACK is raised
};

#define GQ_DEVERR_STACK 1

// Reordering along a space-filling curve (points: Hilbert; rays by origin and direction):
// writes perm[0..n) (a permutation of 0..n-1) using `scratch`.
// Returns the scratch bytes needed when scratch == nullptr.
size_t morton_scratch_bytes(int64_t n);
// ray_mode > 0 (3D): keys from the ray origins q and directions ray_dir (see k_ray_keys).
cudaError_t morton_order(const DevScene &s, gq_vecs q, int64_t n, int32_t *perm, void *scratch, size_t scratch_bytes,
                         cudaStream_t st, int ray_mode = 0, gq_vecs ray_dir = gq_vecs{});

// Launch choices for one query kind (picked by the autotuner or the defaults).
struct Tune {
    int packet = 0;   // closest point: 1 = warp-coherent traversal
    int sorted = 1;   // warp-coherent wide nodes: 1 = children in distance order, 0 = nearest first
    int persist = 1;  // persistent warps with lane refill (per-thread traversal)
    int budget = 32;  // node visits between refills
    int block = 128;  // threads per block: 64, 128 or 256
    int stack = 0;    // warp-coherent closest point: 32 = short stack (trees that fit), 0 = full depth
};

// Index of a supported block size (64, 128, 256) for per-size launch caches; -1 otherwise.
inline int block_slot(int block) { return block == 64 ? 0 : block == 128 ? 1 : block == 256 ? 2 : -1; }

// `counter` is an 8-byte device word used by the persistent / warp-coherent kernels
// (may be null: one query per thread then).
cudaError_t launch_cp(const DevScene &s, int variant, const Tune &t, gq_vecs q, int64_t n, const int32_t *perm,
                      const gq_cp_out &o, unsigned long long *counter, cudaStream_t st);
// Rays over the quantised 8-wide BVH, one ray per group of 8 lanes (ray_group.cu).
cudaError_t launch_ray_group(const DevScene &s, gq_vecs x, gq_vecs v, const float *r_max, int64_t n,
                             const int32_t *perm, const gq_ray_out &o, unsigned long long *counter, cudaStream_t st);
cudaError_t launch_ray(const DevScene &s, int variant, const Tune &t, gq_vecs x, gq_vecs v, const float *r_max,
                       int64_t n, const int32_t *perm, const gq_ray_out &o, unsigned long long *counter,
                       cudaStream_t st);
// Warp-coherent closest point; layout 0 = binary pairs, 1 / 2 = quantised 8-wide (3D): sorted / nearest first.
cudaError_t launch_cp_packet(const DevScene &s, int layout, const Tune &t, gq_vecs q, int64_t n,
                             const int32_t *perm, const gq_cp_out &o, unsigned long long *counter, cudaStream_t st);
// Closest silhouette.  GQ_VARIANT_COHERENT (with a counter): warp-coherent traversal of
// 32 sorted queries at a time; otherwise the reference order per lane, with persistent
// lane refill when t.persist is set (t.budget steps between refills).
cudaError_t launch_sil(const DevScene &s, int variant, const Tune &t, gq_vecs x, const float *r_max, int64_t n,
                       const int32_t *perm, const gq_sil_out &o, unsigned long long *counter, cudaStream_t st);
cudaError_t launch_cp_brute(const DevScene &s, gq_vecs q, int64_t n, const gq_cp_out &o, cudaStream_t st);
// closest_silhouette_baseline over `sils` (n_sil records of the scene's silhouette
// layout, in the reference's list order) instead of the SNCH leaf lists.
cudaError_t launch_sil_brute(const DevScene &s, const void *sils, int64_t n_sil, gq_vecs x, const float *r_max,
                             int64_t n, const gq_sil_out &o, cudaStream_t st);
cudaError_t launch_ray_brute(const DevScene &s, gq_vecs x, gq_vecs v, const float *r_max, int64_t n,
                             const gq_ray_out &o, cudaStream_t st);
// Reads `bytes` (a multiple of 16) of device memory `reps` times with L2-only loads.
cudaError_t launch_read_probe(const void *buf, int64_t bytes, int reps, unsigned *sink, cudaStream_t st);
// FP64 nearest silhouette over raw records (2D: 8 floats, 3D: 16 floats each).
cudaError_t launch_sil_f64(int dim, const float *recs, int64_t n_sil, gq_vecs x, int64_t n, double *out_d,
                           int32_t *out_id, cudaStream_t st);
cudaError_t launch_brute_f64(const DevScene &s, int kind, gq_vecs a, gq_vecs b, int64_t n, double *out_d,
                             int32_t *out_id, cudaStream_t st);

}  // namespace gqd

namespace gqd {
// Allocation-free closest point (noalloc.cu): scratch in a static device array.
int64_t noalloc_max_queries();
cudaError_t noalloc_closest_point(const DevScene &s, int variant, const Tune &t, gq_vecs q, int64_t n, int sort,
                                  const gq_cp_out &o, cudaStream_t st);
}  // namespace gqd
