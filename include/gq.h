/* gq.h — C ABI of the B200 geometry-query engine (libgq.so).
 *
 * Replaces two reference interfaces:
 *   - the nanobind builder module `gquery_ext` (src/gquery.cpp:181-250): BVH, BVH3D,
 *     SNCH, SNCH3D, node_data(), primitive_data(), silhouette_data(),
 *     build_flat_silhouette_edges();
 *   - the DrJit-traced traversal methods called by Polyline / Mesh:
 *     BVH.closest_point (gquery/shapes/bvh.py:127), BVH.intersect (bvh.py:200),
 *     BVH3D.closest_point (bvh3d.py:108), BVH3D.intersect (bvh3d.py:176),
 *     SNCH.closest_silhouette (snch.py:106), SNCH3D.closest_silhouette (snch3d.py:143),
 *     and the brute-force *_baseline methods (polyline.py:138, 176, 212; mesh.py:61, 92, 124).
 *
 * Conventions
 *   - Plain pointers and sizes only.  Host pointers are marked "host"; everything a
 *     query reads or writes is device memory on the scene's device.
 *   - Every call returns a gq_status; nothing throws across the ABI.  The text of
 *     the last error on the calling thread is available from gq_last_error().
 *   - Query calls are asynchronous and ordered on the CUDA stream passed as
 *     `stream` (a cudaStream_t; NULL = legacy default stream).
 *   - Scenes are immutable after the build and may be shared by host threads and
 *     streams.
 *   - Arrays of vectors are strided: component k of element i is
 *     ptr[k * comp_stride + i * elem_stride] (SoA [D][n] -> (n, 1); AoS [n][D] -> (1, D)).
 *   - Output records are structure-of-arrays with component stride n; a NULL field
 *     pointer skips that field.  A miss writes an all-zero record (valid = 0).
 */
#ifndef GQ_H
#define GQ_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t gq_status;
#define GQ_OK 0
#define GQ_ERR_INVALID 1    /* bad argument (shape, null pointer, index out of range) */
#define GQ_ERR_CUDA 2       /* a CUDA call failed */
#define GQ_ERR_NOMEM 3      /* allocation failed */
#define GQ_ERR_DEPTH 4      /* tree deeper than the traversal stack of the requested variant */
#define GQ_ERR_DEVICE 5     /* a kernel raised its error flag (see gq_scene_device_error) */
#define GQ_ERR_UNSUPPORTED 6

/* Traversal variants */
#define GQ_VARIANT_EXACT 0    /* binary tree, gQuery's visit order: reference-identical answers */
#define GQ_VARIANT_WIDE8 1    /* 8-wide nodes, 8-bit outward-rounded child boxes */
#define GQ_VARIANT_AUTO 2     /* the scene's tuned choice for the query kind (gq_scene_set_tuning) */
#define GQ_VARIANT_COHERENT 3 /* binary tree walked once per warp of queries adjacent in the sort order (closest
                                 point, closest silhouette); rays run as EXACT */
#define GQ_VARIANT_WARP 4     /* closest silhouette only: one query per warp, its 32 lanes expanding up to
                                 32 tree nodes per step (for few, far-reaching queries) */
#define GQ_VARIANT_WIDE16 5   /* the 8-wide nodes with 16-bit outward-rounded child bounds (scenes built with
                                 build_wide = 2); closest points and rays, one lane per query */
/* All variants other than EXACT give the same answers as EXACT except at FP32 distance
 * ties (distances within 2e-6 relative). */

/* Query kinds (tuning table) */
#define GQ_KIND_CLOSEST_POINT 0
#define GQ_KIND_INTERSECT 1
#define GQ_KIND_SILHOUETTE 2

typedef struct {
    int32_t variant;  /* variant used when a query asks for GQ_VARIANT_AUTO */
    int32_t packet;   /* WIDE8 closest point (3D): 1 = warp-coherent traversal; warp-coherent closest
                         points (COHERENT, and WIDE8 with packet): 2 = the compact stack (keys rounded
                         down to FP16, one node word per warp; same answers); WIDE8 rays: 1 = one ray
                         per group of 8 lanes, one child or item per lane; WARP silhouettes: switch
                         to the coherent traversal from 2^18 queries on */
    int32_t sorted;   /* warp-coherent wide nodes: children in distance order (else nearest first) */
    int32_t persist;  /* per-thread kernels: persistent warps, finished lanes take new queries */
    int32_t budget;   /* node visits between refills */
    int32_t block;    /* threads per block of the persistent / warp-coherent kernels: 64, 128, 256 (0: 128) */
    int32_t stack;    /* warp-coherent closest point: 32 = short traversal stack when the tree fits, 0 = full */
} gq_tuning;

typedef struct gq_scene gq_scene;

typedef struct {
    int32_t max_prims_in_node; /* leaf size limit of the SAH build; gQuery's default is 10 */
    int32_t n_threads;         /* host threads for the build; 0 = all cores */
    int32_t build_snch;        /* also build silhouettes and normal cones */
    int32_t build_wide;        /* also build the quantised 8-wide BVH (8-bit child bounds); 2: and the same
                                  nodes' 16-bit child bounds (GQ_VARIANT_WIDE16) */
    int32_t device;            /* CUDA device that holds the scene */
    int32_t gpu_build;         /* build a linear BVH on the device instead (milliseconds; no SNCH, no wide
                                  nodes, no reference arrays; answers equal up to FP32 ties) */
} gq_build_opts;

typedef struct {
    int32_t dim;               /* 2 or 3 */
    int64_t n_vertices, n_prims, n_nodes, n_wide_nodes, n_silhouettes;
    int32_t max_depth;         /* deepest leaf of the binary tree (root = 0) */
    int32_t exact_stack, wide_stack;
    int64_t device_bytes;      /* HBM held by the scene */
    float bbox_lo[3], bbox_hi[3];
} gq_scene_info;

typedef struct {
    const float *ptr;
    int64_t comp_stride;
    int64_t elem_stride;
} gq_vecs;

typedef struct {
    uint8_t *valid;   /* [n] */
    float *p;         /* [D][n] closest point */
    float *n;         /* [D][n] normal */
    float *t;         /* 2D: [n] parameter on the segment; 3D: [2][n] barycentric uv */
    float *d;         /* [n] distance */
    int32_t *prim_id; /* [n] original primitive index */
} gq_cp_out;

typedef struct {
    uint8_t *valid;
    float *p;
    float *n;
    float *t;         /* 2D: [n] (gQuery stores -1 on a hit); 3D: [2][n] uv */
    float *d;         /* [n] ray parameter of the hit */
    int32_t *prim_id;
    uint8_t *on_boundary;
} gq_ray_out;

typedef struct {
    uint8_t *valid;
    float *p;         /* [D][n] closest silhouette point */
    float *d;
    int32_t *prim_id; /* silhouette id: vertex index (2D) / edge index (3D) */
} gq_sil_out;

typedef struct {
    int32_t variant;        /* GQ_VARIANT_* */
    int32_t sort;           /* 1: reorder queries along a space-filling curve before traversal (gq_query_order) */
    const int32_t *order;   /* optional device permutation from gq_query_order(); replaces `sort` */
    void *scratch;          /* optional device scratch (see gq_query_scratch_bytes); NULL = stream-ordered allocation */
    int64_t scratch_bytes;
} gq_query_opts;

/* ---- errors ---- */
/* Copies the calling thread's last error message (NUL-terminated, truncated to cap). */
void gq_last_error(char *buf, int64_t cap);
const char *gq_status_string(gq_status s);

/* ---- scene build (replaces gquery_ext.BVH / BVH3D / SNCH / SNCH3D constructors,
 *      src/gquery.cpp:184-185, 196-197, 227-228, 239-240) ----
 * vertices: host [nv][D] float32, finite; prims: host [np][D] int32 (edges in 2D, faces in
 * 3D) in [0, nv).  Other input is GQ_ERR_INVALID. */
gq_status gq_scene_build_2d(const float *vertices, int64_t nv, const int32_t *edges, int64_t ne,
                            const gq_build_opts *opts, gq_scene **out);
gq_status gq_scene_build_3d(const float *vertices, int64_t nv, const int32_t *faces, int64_t nf,
                            const gq_build_opts *opts, gq_scene **out);
gq_status gq_scene_free(gq_scene *scene);

/* Scene files (no counterpart in the reference, which rebuilds its trees whenever a
 * Mesh / Polyline is constructed): save writes the input geometry and the flattened
 * device arrays of a scene that has a device copy; load uploads them to `device` without
 * building anything.  The host trees behind gq_scene_ref_array are rebuilt on first use
 * (the build is deterministic).  The format is native-endian and versioned.  Load checks
 * the arrays on the host before uploading them (sizes, every reference inside its array
 * with at most one parent, leaf ends, finite vertices) and refuses a file that fails
 * with GQ_ERR_INVALID ("... is corrupt: ..."). */
gq_status gq_scene_save(const gq_scene *scene, const char *path);
gq_status gq_scene_load(const char *path, int32_t device, gq_scene **out);
gq_status gq_scene_get_info(const gq_scene *scene, gq_scene_info *info);

/* Launch choices per query kind (no counterpart in the reference, whose DrJit backend
 * picks its own launch shape).  gquery_b200.autotune measures the candidates and sets
 * them; the built-in defaults are the measured B200 choices for the benchmark scenes.
 * Not thread-safe against concurrent queries on the same scene. */
gq_status gq_scene_set_tuning(gq_scene *scene, int32_t kind, const gq_tuning *tuning);
gq_status gq_scene_get_tuning(const gq_scene *scene, int32_t kind, gq_tuning *tuning);

/* Reference float layouts (gquery_ext node_data / primitive_data / silhouette_data /
 * raw_silhouette_data, src/gquery.cpp:186-187, 229-231, 241-244).  Copies up to `cap`
 * floats into host `dst` and stores the full length in *len (dst may be NULL to query). */
#define GQ_ARRAY_BVH_NODES 0       /* stride 2D+3 (7 / 9) */
#define GQ_ARRAY_PRIMITIVES 1      /* stride 5 / 10 */
#define GQ_ARRAY_SNCH_NODES 2      /* stride 13 / 16 */
#define GQ_ARRAY_SILHOUETTES 3     /* ordered, per-leaf lists; stride 10 / 19 */
#define GQ_ARRAY_RAW_SILHOUETTES 4 /* one per vertex / unique edge */
#define GQ_ARRAY_WIDE_NODES 5      /* quantised 8-wide node records as raw 32-bit words (24 / 20 per node);
                                      host-only scenes (device < 0) only */
#define GQ_ARRAY_SNCH_PAIRS 6      /* SNCH pair records (gq_spair2_t / gq_spair3_t) as raw 32-bit words
                                      (20 / 40 per pair; pair 0 is the root's); host-only scenes only */
#define GQ_ARRAY_WIDE16_BOUNDS 8   /* 16-bit bounds records (gq_wq16_2_t / gq_wq16_3_t) as raw 32-bit words
                                      (20 / 28 per node); host-only scenes built with build_wide = 2 only */
#define GQ_ARRAY_SIL_RECORDS 7     /* silhouette records (gq_silv_t / gq_sile_t) as raw 32-bit words
                                      (8 / 16 per record, in leaf order); host-only scenes only */
gq_status gq_scene_ref_array(const gq_scene *scene, int32_t which, float *dst, int64_t cap, int64_t *len);

/* build_flat_silhouette_edges (src/gquery.cpp:250, src/shapes/silhouette_edge.cpp:62-71):
 * host in, host out (19 floats per unique edge). */
gq_status gq_flat_silhouette_edges(const float *vertices, int64_t nv, const int32_t *faces, int64_t nf,
                                   float *dst, int64_t cap, int64_t *len);

/* The same on the device: vertices [nv][3] float and faces [nf][3] int32 in device
 * memory of `device`, the 19-float records written to device `dst` (cap floats; with
 * dst = NULL only *len is set).  Ordered, valued and encoded exactly as
 * gq_flat_silhouette_edges; synchronises `stream`. */
gq_status gq_flat_silhouette_edges_device(const float *vertices, int64_t nv, const int32_t *faces, int64_t nf,
                                          float *dst, int64_t cap, int64_t *len, int32_t device, void *stream);

/* ---- queries ---- */
/* Device scratch a query of n items needs when opts->scratch is supplied. */
int64_t gq_query_scratch_bytes(int64_t n);

/* Order of n query points (or ray origins) along a space-filling curve over twice the
 * scene's box (a Hilbert curve, 1024 cells per axis in 3D, 32768 in 2D): writes a
 * permutation of 0..n-1 to device `order`.  `scratch` (device, gq_order_scratch_bytes(n)
 * bytes) may be NULL for a stream-ordered allocation.  Several queries on the same
 * points can share one order through gq_query_opts.order. */
int64_t gq_order_scratch_bytes(int64_t n);
gq_status gq_query_order(const gq_scene *scene, gq_vecs points, int64_t n, int32_t *order, void *scratch,
                         int64_t scratch_bytes, void *stream);
/* The same for rays (3D scenes), keyed by origin and direction so that the rays of one warp
 * also point alike: mode 0 = the origins' order of gq_query_order, 1 = direction
 * octant, then the origins' Morton code, 2 = origin cell and octahedral direction cell
 * interleaved.  No counterpart in the reference (DrJit runs rays in input order). */
gq_status gq_ray_order(const gq_scene *scene, gq_vecs origins, gq_vecs dirs, int64_t n, int32_t mode, int32_t *order,
                       void *scratch, int64_t scratch_bytes, void *stream);

/* closest_point_bvh (Polyline: polyline.py:171 -> bvh.py:127; Mesh: mesh.py:119 -> bvh3d.py:108) */
gq_status gq_closest_point(const gq_scene *scene, gq_vecs q, int64_t n, const gq_cp_out *out,
                           const gq_query_opts *opts, void *stream);

/* Closest point without any device allocation.  No counterpart in the reference: for
 * callers that cannot allocate device memory while querying (a plugin whose host
 * application owns every device allocation and hands it only input and output buffers,
 * a real-time loop that must not enter an allocator, since cudaMalloc may synchronise the
 * device and take unbounded time).  The per-call scratch (work counter and
 * sort buffers) comes from a fixed device array inside the library, which every
 * device that loads the library holds until the process exits; hence at most
 * gq_noalloc_max_queries() queries per call (larger n is rejected with GQ_ERR_INVALID).
 * Same answers as gq_closest_point with the same variant and sort flag.  All calls on a
 * device share that array: calls whose kernels may overlap on the GPU race and must be
 * ordered by the caller (one stream, or events).  The first call on a device looks up
 * the array's device address; make that first call before any stream capture.  The
 * address is kept for the process's primary context of each device: call this entry
 * point from the primary context only, and not after cudaDeviceReset (which frees the
 * array the kept address points to). */
int64_t gq_noalloc_max_queries(void);
gq_status gq_closest_point_noalloc(const gq_scene *scene, gq_vecs q, int64_t n, const gq_cp_out *out,
                                   int32_t variant, int32_t sort, void *stream);

/* intersect_bvh (polyline.py:132 -> bvh.py:200; mesh.py:86 -> bvh3d.py:176).
 * r_max: device [n] or NULL for +inf. */
gq_status gq_intersect(const gq_scene *scene, gq_vecs origin, gq_vecs dir, const float *r_max, int64_t n,
                       const gq_ray_out *out, const gq_query_opts *opts, void *stream);

/* closest_silhouette_snch (polyline.py:225 -> snch.py:106; mesh.py:137 -> snch3d.py:143).
 * r_max: device [n] or NULL for +inf.  Needs a scene built with build_snch. */
gq_status gq_closest_silhouette(const gq_scene *scene, gq_vecs x, const float *r_max, int64_t n,
                                const gq_sil_out *out, const gq_query_opts *opts, void *stream);

/* Brute-force scans over every primitive in original order (closest_point_baseline,
 * intersect_baseline: polyline.py:138-209, mesh.py:61-118).  FP32 like the reference. */
gq_status gq_closest_point_brute(const gq_scene *scene, gq_vecs q, int64_t n, const gq_cp_out *out, void *stream);
gq_status gq_intersect_brute(const gq_scene *scene, gq_vecs origin, gq_vecs dir, const float *r_max, int64_t n,
                             const gq_ray_out *out, void *stream);
/* closest_silhouette_baseline (mesh.py:124-135, polyline.py:212-223): every query scans
 * the shape's silhouette list in order (a Mesh's unique edges as build_flat_silhouette_edges
 * lists them; a Polyline's silhouette vertices as Polyline.configure_silhouette keeps them,
 * polyline.py:44-122) and keeps the first strictly nearest silhouette.  r_max: device [n]
 * or NULL for +inf.  The list is built and uploaded on the scene's first call. */
gq_status gq_closest_silhouette_brute(const gq_scene *scene, gq_vecs x, const float *r_max, int64_t n,
                                      const gq_sil_out *out, void *stream);

/* FP64 brute force used to state the error of the FP32 paths: nearest distance
 * (closest point), nearest ray parameter (ray) or nearest silhouette distance (silhouette,
 * over the SNCH's raw silhouette list; host-built scenes with build_snch), +inf when there
 * is none, and the primitive (silhouette record) it belongs to (-1 when none).  b: ray
 * directions (kind 1 only). */
gq_status gq_brute_f64(const gq_scene *scene, int32_t kind /*0 closest point, 1 ray, 2 silhouette*/, gq_vecs a,
                       gq_vecs b, int64_t n, double *out_d, int32_t *out_id, void *stream);

/* Bandwidth probe for the roofline: reads `bytes` (a multiple of 16, 16-byte aligned) of
 * device memory `reps` times in one launch with 16-byte loads that are cached in L2 only,
 * and xors what it read into the device word `sink`.  Timed on a buffer that fits in L2 it
 * gives the L2 read bandwidth, on a larger one the HBM read bandwidth.  No counterpart in
 * the reference. */
gq_status gq_read_probe(const void *buf, int64_t bytes, int32_t reps, uint32_t *sink, void *stream);

/* Reads and clears the scene's device error word (stack overflow etc.); synchronises `stream`. */
gq_status gq_scene_device_error(const gq_scene *scene, void *stream, int32_t *flags);

/* Caps the entries of this scene's traversal stacks below their compiled sizes (64 binary,
 * 96 wide / warp-coherent); 0 restores the compiled sizes.  A walk that would push past the
 * cap stops: its query comes back as a zeroed miss and GQ_DEVERR_STACK (bit 0) is raised in
 * the scene's device error word.  For bounding per-thread stack memory on trees known to be
 * shallow, and for exercising the overflow path.  Batches and servers copy the cap when they
 * are created.  No counterpart in the reference, whose 64-entry stack (bvh.py:132) has no
 * overflow check. */
gq_status gq_scene_set_stack_limit(gq_scene *scene, int32_t entries);

/* ---- batches: many scenes, all three query kinds, one launch ----
 * No counterpart in the reference, which answers one scene and one query kind per call
 * (mesh.py:86-138, polyline.py:132-226).  A batch holds device views of up to
 * thousands of scenes of one dimension on one device (the scenes must outlive it) and
 * a fixed scratch sized for max_queries queries of each kind, so gq_batch_run
 * allocates nothing and never synchronises: a step can be recorded in a CUDA graph.
 * Each query carries the index of its scene in the batch.  Results are those of the
 * single-scene calls: closest points and silhouettes follow GQ_VARIANT_COHERENT (or
 * GQ_VARIANT_EXACT with GQ_BATCH_CP_EXACT / GQ_BATCH_SIL_EXACT, GQ_VARIANT_WARP with
 * GQ_BATCH_SIL_WARP), rays GQ_VARIANT_WIDE8 when every scene has wide nodes (or
 * GQ_VARIANT_EXACT with GQ_BATCH_RAY_EXACT). */
typedef struct gq_batch gq_batch;

#define GQ_BATCH_CP_EXACT 1  /* closest point: one exact traversal per lane, reference visit order */
#define GQ_BATCH_RAY_EXACT 2 /* rays: binary BVH, reference visit order */
#define GQ_BATCH_SIL_EXACT 8 /* silhouettes: one exact traversal per lane, reference visit order */
#define GQ_BATCH_SIL_WARP 16 /* silhouettes: one query per warp (GQ_VARIANT_WARP), for sparse queries */
#define GQ_BATCH_CP_SPLIT 32 /* closest point: one lane per query in the reference order; a query past
                                1024 node visits is restarted with one warp for it (answers equal up to
                                FP32 distance ties): bounds the tail of sparse, uneven query sets */
#define GQ_BATCH_SIL_SPLIT 64 /* silhouettes: one lane per query in the reference order; a query past 2048
                                 steps is taken over by one warp from the r_max it reached (answers equal up
                                 to FP32 distance ties) */

typedef struct {
    int64_t n;             /* query count (0: none of this kind) */
    const int32_t *scene;  /* device [n]: scene index in the batch; -1 marks a padding slot
                              (skipped, its outputs left untouched) */
    gq_vecs a;             /* points / ray origins */
    gq_vecs b;             /* ray directions (rays only) */
    const float *r_max;    /* device [n] or NULL for +inf (rays, silhouettes) */
} gq_batch_queries;

gq_status gq_batch_create(gq_scene *const *scenes, int32_t n_scenes, int64_t max_queries, int32_t flags,
                          gq_batch **out);
gq_status gq_batch_free(gq_batch *batch);
/* Device bytes the batch holds besides its scenes. */
int64_t gq_batch_device_bytes(const gq_batch *batch);
/* Any of the query / output pointers may be NULL to skip that kind. */
gq_status gq_batch_run(gq_batch *batch, const gq_batch_queries *cp, const gq_cp_out *cp_out,
                       const gq_batch_queries *ray, const gq_ray_out *ray_out, const gq_batch_queries *sil,
                       const gq_sil_out *sil_out, void *stream);
/* Reads and clears the device error words of the batch and of every member scene;
 * synchronises `stream`.  Bits 0-7: the scenes' words or-ed together (bit 0 stack
 * overflow); bit 8: a query named a scene outside the batch; bit 9: a silhouette query
 * named a scene without SNCH. */
gq_status gq_batch_device_error(gq_batch *batch, void *stream, int32_t *flags);

/* ---- serving: continuous batching of requests against resident scenes ----
 * No counterpart in the reference.  A server owns a worker thread, device rings for
 * request data (inputs and results of each query kind) and pinned host mirrors of
 * them.  Requests (one scene, one query kind, n queries in host memory) may be
 * submitted from any thread at any time.  The worker admits a request when its ring
 * has room (the rings are the admission budget: their device bytes may not exceed
 * budget_bytes), copies its queries to the device at once on a copy stream while
 * earlier steps compute, and launches a step over every admitted request as soon as
 * a step slot is free: one gq_batch launch for all scenes (or, with
 * GQ_SERVER_PER_REQUEST, one single-scene call per request, the scene's tuned
 * variant).  Closest-point and ray requests share max_inflight slots; silhouette
 * requests, whose traversals are far longer, have sil_slots slots of their own on a
 * lower stream priority, taking at most sil_step_queries queries each, so the other
 * kinds never queue behind them.  Requests of at least large_queries queries form a
 * second size class with rings and slots of its own (large_slots for closest points /
 * rays and as many for silhouettes) on still lower priorities, so a small request
 * never shares a step with a large one and its blocks are placed ahead of a large
 * step's pending blocks.  Silhouette steps in the default one-query-per-warp form launch
 * one block per query that exits when its query is answered, so the blocks of
 * higher-priority steps are placed first and silhouettes fill the rest of the GPU; the
 * other silhouette forms run persistent launches that together hold at most sil_share
 * of the GPU.  Staging queries into the pinned rings and scattering results into the
 * requests' arrays run on copy_threads host threads.
 * Each slot has its own stream, so the results of one step go back to the host while
 * the next computes.  Results are those of gq_batch_run.
 * Streams: 1 + max_inflight + sil_slots + 2 * large_slots (11 by default).  CUDA maps
 * streams onto CUDA_DEVICE_MAX_CONNECTIONS hardware queues (8 unless the variable is
 * set before the CUDA context is created) and runs the work of streams that share a
 * queue in order, so a process that serves should set it to 32: otherwise a short step
 * can wait for a long one on its queue. */
typedef struct gq_server gq_server;

#define GQ_SERVER_PER_REQUEST 4 /* one single-scene launch per request instead of batched steps */

typedef struct {
    int64_t budget_bytes;     /* device bytes the request rings may hold (0: no limit) */
    int64_t ring_queries[3];  /* ring capacity in queries per kind (0: 1<<22) */
    int64_t step_queries;     /* most queries of one kind in one step, and the largest request (0: 1<<19) */
    int32_t max_inflight;     /* step slots for closest-point and ray steps (0: 3) */
    int32_t flags;            /* GQ_BATCH_*_EXACT | GQ_SERVER_PER_REQUEST */
    float sil_share;          /* share of the GPU's resident blocks all persistent silhouette steps together may hold (0: 1.5;
                                 above 1 they may oversubscribe it, each slot capped at 1) */
    int32_t sil_slots;        /* silhouette step slots (0: 3) */
    int64_t sil_step_queries; /* most silhouette queries in one small-class step, unless one request is larger (0: 1<<15) */
    int64_t large_queries;    /* requests of at least this many queries are large (0: 1<<15; negative: one class;
                                 also one class when above step_queries, with GQ_SERVER_PER_REQUEST, or when half
                                 of a kind's ring is below step_queries).  With two classes each kind's ring is
                                 split in halves, one per class */
    int32_t large_slots;      /* step slots of the large class, for closest points / rays and for silhouettes each (0: 2) */
    float large_share;        /* share of the GPU's resident blocks a large closest-point / ray step's persistent grid
                                 may hold (0: 1) */
    int32_t copy_threads;     /* host threads for staging and scattering, the worker included (0: min(8, cores / 2)) */
} gq_server_opts;

typedef struct {
    int32_t scene;       /* index into the server's scenes */
    int32_t kind;        /* GQ_KIND_* */
    int64_t n;           /* queries, 1 .. step_queries */
    const float *a;      /* host [n][D]: points / ray origins */
    const float *b;      /* host [n][D]: ray directions (rays only) */
    const float *r_max;  /* host [n] or NULL for +inf (rays, silhouettes) */
    gq_cp_out cp_out;    /* host results of a closest-point request ([D][n] fields) */
    gq_ray_out ray_out;  /* host results of a ray request */
    gq_sil_out sil_out;  /* host results of a silhouette request */
    uint64_t tag;        /* returned with the completion */
} gq_request;

typedef struct {
    uint64_t tag;
    double t_submit, t_admit, t_launch, t_done; /* seconds on gq_server_clock() */
    int64_t n;
    int32_t kind;
    int32_t step;        /* step that answered it */
    int32_t status;      /* GQ_OK, or the error of the launch that served it */
} gq_completion;

typedef struct {
    int64_t requests_done, queries_done, steps, admitted_bytes_peak, device_bytes;
    int32_t device_error; /* or-ed error words of the step slots and scenes (gq_batch_device_error bits) */
    int64_t large_queries; /* size of the smallest large request, 0 when the server keeps one class */
} gq_server_stats;

double gq_server_clock(void);
gq_status gq_server_create(gq_scene *const *scenes, int32_t n_scenes, const gq_server_opts *opts,
                           gq_server **out);
/* Stops the worker after the steps in flight; requests not yet answered are dropped. */
gq_status gq_server_free(gq_server *server);
/* Non-blocking; the request's host buffers must stay valid until its completion. */
gq_status gq_server_submit(gq_server *server, const gq_request *request);
/* Moves up to cap completions into out; *count = how many. */
gq_status gq_server_poll(gq_server *server, gq_completion *out, int64_t cap, int64_t *count);
/* Blocks until every submitted request has completed or timeout_s passed (GQ_ERR_DEVICE on timeout). */
gq_status gq_server_wait_idle(gq_server *server, double timeout_s);
gq_status gq_server_get_stats(gq_server *server, gq_server_stats *stats);
/* Open-loop driver for an otherwise idle server: submits reqs[i] at start + t_arrival[i]
 * seconds (start = now), waits for all, and writes each request's completion to out[i]
 * with t_submit set to its scheduled arrival time. */
gq_status gq_server_run_trace(gq_server *server, const gq_request *reqs, const double *t_arrival, int64_t n,
                              gq_completion *out, double timeout_s);

#ifdef __cplusplus
}
#endif

#endif /* GQ_H */
