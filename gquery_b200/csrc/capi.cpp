// C ABI of libgq.so (declared in include/gq.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/gq.h"
#include "device/batch.cuh"
#include "device/gpu_build.cuh"
#include "internal.hpp"

using namespace gqb;

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace gqi {
gq_status fail(gq_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}
gq_status fail_cuda(cudaError_t e, const char *what) {
    return fail(GQ_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace gqi

using gqi::DeviceGuard;
using gqi::fail;
using gqi::fail_cuda;

namespace {

void default_tuning(gq_scene *s);

// Linear BVH on the device (device/gpu_build.cu) straight into the traversal records.
template <int D>
gq_status build_on_device(gq_scene *s, const gq_build_opts &o) {
    if (o.device < 0) return fail(GQ_ERR_INVALID, "a device build needs a device");
    if (s->np < 1) return fail(GQ_ERR_INVALID, "a device build needs at least one primitive");
    DeviceGuard g(o.device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's CUDA device");
    gqd::DevScene &d = s->dev;
    const void *pv = nullptr, *pi = nullptr, *pe = nullptr;
    gq_status st;
    if ((st = s->upload(s->verts, &pv)) != GQ_OK) return st;
    if ((st = s->upload(s->index, &pi)) != GQ_OK) return st;
    std::vector<int32_t> zero(1, 0);
    if ((st = s->upload(zero, &pe)) != GQ_OK) return st;
    using Pair = std::conditional_t<D == 2, gq_pair2_t, gq_pair3_t>;
    using Prim = std::conditional_t<D == 2, gq_seg_t, gq_tri_t>;
    const size_t pair_bytes = sizeof(Pair) * (size_t)std::max<int64_t>(s->np - 1, 1);
    const size_t prim_bytes = sizeof(Prim) * (size_t)s->np;
    void *pairs = nullptr, *prims = nullptr;
    cudaError_t e = cudaMalloc(&pairs, pair_bytes);
    if (e == cudaSuccess) s->allocs.push_back(pairs), e = cudaMalloc(&prims, prim_bytes);
    if (e == cudaSuccess) s->allocs.push_back(prims);
    if (e != cudaSuccess) return fail(GQ_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    s->device_bytes += (int64_t)(pair_bytes + prim_bytes);
    gqd::GpuBuildResult r;
    gqd::GpuSnchBuild sb;
    const bool with_snch = o.build_snch != 0;
    std::vector<void *> tmp;  // the unique edges, freed after the build
    auto free_tmp = [&]() {
        for (void *p : tmp) cudaFree(p);
    };
    size_t spair_bytes = 0, sil_bytes = 0;
    if (with_snch) {
        using SPair = std::conditional_t<D == 2, gq_spair2_t, gq_spair3_t>;
        using Sil = std::conditional_t<D == 2, gq_silv_t, gq_sile_t>;
        const int64_t nh = 3 * s->np, n_rec = D * s->np;  // 3D: half-edges; records: D per leaf
        void *edges = nullptr, *face_edge = nullptr, *orient = nullptr, *spairs = nullptr, *sils = nullptr;
        if (D == 3) {
            e = cudaMalloc(&edges, (size_t)nh * 19 * sizeof(float));
            if (e == cudaSuccess) tmp.push_back(edges), e = cudaMalloc(&face_edge, (size_t)nh * sizeof(uint32_t));
            if (e == cudaSuccess) tmp.push_back(face_edge), e = cudaMalloc(&orient, (size_t)nh * sizeof(float));
            if (e == cudaSuccess) tmp.push_back(orient);
        }
        spair_bytes = sizeof(SPair) * (size_t)std::max<int64_t>(s->np - 1, 1);
        sil_bytes = sizeof(Sil) * (size_t)n_rec;
        if (e == cudaSuccess) e = cudaMalloc(&spairs, spair_bytes);
        if (e == cudaSuccess) s->allocs.push_back(spairs), e = cudaMalloc(&sils, sil_bytes);
        if (e == cudaSuccess) s->allocs.push_back(sils);
        if (e != cudaSuccess) {
            free_tmp();
            return fail(GQ_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
        s->device_bytes += (int64_t)(spair_bytes + sil_bytes);
        if (D == 3) {
            int64_t n_edges = 0;
            int bad = 0;
            e = gqd::gpu_silhouette_edges((const float *)pv, s->nv, (const int32_t *)pi, s->np, (float *)edges, nh,
                                          &n_edges, &bad, nullptr, (uint32_t *)face_edge, (float *)orient);
            if (e != cudaSuccess || bad) {
                free_tmp();
                if (e != cudaSuccess) return fail_cuda(e, "device silhouette edges");
                return fail(GQ_ERR_INVALID, "face index out of range");
            }
        }
        sb.edges19 = (const float *)edges;
        sb.face_edge = (const uint32_t *)face_edge;
        sb.edge_orient = (const float *)orient;
        sb.n_verts = s->nv;
        sb.spairs = spairs;
        sb.sils = sils;
    }
    e = gqd::gpu_build_bvh(D, (const float *)pv, (const int32_t *)pi, s->np, pairs, prims, r, nullptr,
                           with_snch ? &sb : nullptr);
    free_tmp();
    if (e != cudaSuccess) return fail_cuda(e, "device build");
    if (o.build_wide) {
        // the collapse into quantised 8-wide nodes runs on the host over the pair records
        using WPair = std::conditional_t<D == 2, gq_pair2_t, gq_pair3_t>;
        DeviceImage<D> wimg;
        std::vector<WPair> hp((size_t)std::max<int64_t>(s->np - 1, 0));
        if (!hp.empty()) {
            e = cudaMemcpy(hp.data(), pairs, hp.size() * sizeof(WPair), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) return fail_cuda(e, "device build: pair download");
        }
        try {
            flatten_wide_from_pairs<D>(hp, r.root_ref, r.root_lo, r.root_hi, wimg,
                                       o.n_threads > 0 ? o.n_threads : (int)std::max(1u, std::thread::hardware_concurrency()));
        } catch (const std::bad_alloc &) {
            return fail(GQ_ERR_NOMEM, "out of host memory collapsing the device-built tree");
        }
        if (!wimg.wnodes.empty() && (st = s->upload(wimg.wnodes, &d.wnodes)) != GQ_OK) return st;
        d.wroot_ref = wimg.wroot_ref;
        s->has_wide = true;
        s->wide_stack = wimg.wide_stack;
        s->n_wide = (int64_t)wimg.wnodes.size();
        s->image_bytes[3] = wimg.wnodes.size() * sizeof(wimg.wnodes[0]);
    }
    if (with_snch) {
        d.spairs = sb.spairs;
        d.sils = sb.sils;
        d.sroot_ref = s->np > 1 ? 0 : ~0;  // a single primitive: its leaf, records 0..D-1
        s->has_snch = true;
        s->n_sil = D * s->np;
        d.n_sils = s->n_sil;
        s->image_bytes[4] = s->np > 1 ? spair_bytes : 0;
        s->image_bytes[5] = sil_bytes;
    }
    d.dim = D;
    d.pairs = pairs;
    d.prims = prims;
    d.verts = (const float *)pv;
    d.index = (const int32_t *)pi;
    d.err = (int32_t *)pe;
    d.n_prims = s->np;
    d.coord_bound = 0.f;
    for (float x : s->verts) d.coord_bound = std::max(d.coord_bound, std::fabs(x));
    d.root_ref = r.root_ref;
    for (int k = 0; k < 3; ++k) d.root_lo[k] = r.root_lo[k], d.root_hi[k] = r.root_hi[k];
    s->gpu_built = true;
    s->trees_ready = false;
    s->max_prims_in_node = 1;
    s->max_depth = r.max_depth;
    s->exact_stack = r.max_depth + 1;
    s->n_nodes = 2 * s->np - 1;
    s->image_bytes[0] = s->np > 1 ? pair_bytes : 0;
    s->image_bytes[1] = prim_bytes;
    default_tuning(s);
    return GQ_OK;
}

template <int D>
gq_status build_scene(const float *vertices, int64_t nv, const int32_t *prims, int64_t np, const gq_build_opts *opts,
                      gq_scene **out) {
    if (!out) return fail(GQ_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!vertices || !prims) return fail(GQ_ERR_INVALID, "null vertex or primitive array");
    gq_build_opts o{10, 0, 1, 1, 0, 0};
    if (opts) o = *opts;
    if (o.max_prims_in_node < 1) return fail(GQ_ERR_INVALID, "max_prims_in_node must be >= 1");
    int nt = o.n_threads > 0 ? o.n_threads : (int)std::max(1u, std::thread::hardware_concurrency());

    std::unique_ptr<gq_scene> s(new (std::nothrow) gq_scene());
    if (!s) return fail(GQ_ERR_NOMEM, "out of host memory");
    s->dim = D;
    s->device = o.device;
    s->nv = nv;
    s->np = np;
    try {
        s->verts.assign(vertices, vertices + nv * D);
        s->index.assign(prims, prims + np * D);
    } catch (const std::bad_alloc &) {
        return fail(GQ_ERR_NOMEM, "out of host memory");
    }
    PrimSource<D> src{s->verts.data(), nv, s->index.data(), np};
    std::string bad = validate_source<D>(src);
    if (!bad.empty()) return fail(GQ_ERR_INVALID, bad);
    if (o.gpu_build) {
        gq_status st = build_on_device<D>(s.get(), o);
        if (st != GQ_OK) return st;
        *out = s.release();
        return GQ_OK;
    }

    DeviceImage<D> img;
    try {
        BvhTree<D> tree = build_bvh<D>(src, o.max_prims_in_node, nt);
        flatten_bvh<D>(src, tree, img);
        if (o.build_wide) {
            flatten_wide<D>(tree, img, o.build_wide >= 2);
            s->has_wide = true;
            s->has_wide16 = o.build_wide >= 2;
        }
        if (o.build_snch) {
            SnchTree<D> sn = build_snch<D>(src, tree, nt);
            flatten_snch<D>(tree, sn, img, nt);
            s->has_snch = true;
            if constexpr (D == 2)
                s->s2 = std::move(sn);
            else
                s->s3 = std::move(sn);
        }
        if constexpr (D == 2)
            s->t2 = std::move(tree);
        else
            s->t3 = std::move(tree);
    } catch (const std::bad_alloc &) {
        return fail(GQ_ERR_NOMEM, "out of host memory during the build");
    }

    s->exact_stack = img.exact_stack;
    s->wide_stack = img.wide_stack;
    s->max_prims_in_node = o.max_prims_in_node;
    s->n_nodes = D == 2 ? (int64_t)s->t2.nodes.size() : (int64_t)s->t3.nodes.size();
    s->max_depth = D == 2 ? s->t2.max_depth : s->t3.max_depth;
    s->image_bytes[0] = img.pairs.size() * sizeof(img.pairs[0]);
    s->image_bytes[1] = img.prims.size() * sizeof(img.prims[0]);
    s->image_bytes[2] = img.spheres.size() * sizeof(gq_tsph_t);
    s->image_bytes[3] = img.wnodes.size() * sizeof(img.wnodes[0]);
    s->image_bytes[4] = img.spairs.size() * sizeof(img.spairs[0]);
    s->image_bytes[5] = img.sils.size() * sizeof(img.sils[0]);
    default_tuning(s.get());
    s->n_wide = (int64_t)img.wnodes.size();
    s->n_sil = (int64_t)img.sils.size();
    s->dev.n_sils = s->n_sil;
    gqd::DevScene &d = s->dev;
    d.dim = D;
    for (int k = 0; k < 3; ++k) {
        d.root_lo[k] = k < D ? img.root_lo[k] : 0.f;
        d.root_hi[k] = k < D ? img.root_hi[k] : 0.f;
    }
    if (o.device < 0) {  // host-only scene: reference arrays, no device copy
        auto keep = [](std::vector<float> &dst, const void *src, size_t bytes) {
            dst.resize(bytes / 4);
            if (bytes) std::memcpy(dst.data(), src, bytes);
        };
        keep(s->wide_words, img.wnodes.data(), img.wnodes.size() * sizeof(img.wnodes[0]));
        keep(s->wide16_words, img.wq16.data(), img.wq16.size() * sizeof(img.wq16[0]));
        keep(s->spair_words, img.spairs.data(), img.spairs.size() * sizeof(img.spairs[0]));
        keep(s->sil_words, img.sils.data(), img.sils.size() * sizeof(img.sils[0]));
        *out = s.release();
        return GQ_OK;
    }
    DeviceGuard g(o.device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's CUDA device");
    gq_status st;
    if ((st = s->upload(img.pairs, &d.pairs)) != GQ_OK) return st;
    if ((st = s->upload(img.prims, &d.prims)) != GQ_OK) return st;
    const void *psph = nullptr;
    if ((st = s->upload(img.spheres, &psph)) != GQ_OK) return st;
    d.spheres = (const gq_tsph_t *)psph;
    if ((st = s->upload(img.wnodes, &d.wnodes)) != GQ_OK) return st;
    if ((st = s->upload(img.wq16, &d.wq16)) != GQ_OK) return st;
    if ((st = s->upload(img.spairs, &d.spairs)) != GQ_OK) return st;
    if ((st = s->upload(img.sils, &d.sils)) != GQ_OK) return st;
    const void *pv = nullptr, *pi = nullptr, *pe = nullptr;
    if ((st = s->upload(s->verts, &pv)) != GQ_OK) return st;
    if ((st = s->upload(s->index, &pi)) != GQ_OK) return st;
    std::vector<int32_t> zero(1, 0);
    if ((st = s->upload(zero, &pe)) != GQ_OK) return st;
    d.verts = (const float *)pv;
    d.index = (const int32_t *)pi;
    d.err = (int32_t *)pe;
    d.n_prims = np;
    d.coord_bound = 0.f;
    for (float x : s->verts) d.coord_bound = std::max(d.coord_bound, std::fabs(x));
    d.root_ref = img.root_ref;
    d.wroot_ref = img.wroot_ref;
    d.sroot_ref = img.sroot_ref;
    *out = s.release();
    return GQ_OK;
}

bool on_host_only(const gq_scene *s) { return s->device < 0; }

// Silhouette queries tuned to the WARP variant with `packet` set switch to the coherent
// traversal from this many queries on (measured crossover on B200: ~2^20 for the
// level-7 benchmark mesh, below it for smaller scenes).
constexpr int64_t kSilCoherentFrom = 1 << 18;

// Host trees of a loaded scene, rebuilt on first use: the build is deterministic, so
// they are the trees the saved device image was flattened from.
gq_status ensure_trees(gq_scene *s) {
    std::lock_guard<std::mutex> lk(s->tree_mu);
    if (s->trees_ready) return GQ_OK;
    const int nt = (int)std::max(1u, std::thread::hardware_concurrency());
    try {
        if (s->dim == 2) {
            PrimSource<2> src{s->verts.data(), s->nv, s->index.data(), s->np};
            s->t2 = build_bvh<2>(src, s->max_prims_in_node, nt);
            if (s->has_snch) s->s2 = build_snch<2>(src, s->t2, nt);
        } else {
            PrimSource<3> src{s->verts.data(), s->nv, s->index.data(), s->np};
            s->t3 = build_bvh<3>(src, s->max_prims_in_node, nt);
            if (s->has_snch) s->s3 = build_snch<3>(src, s->t3, nt);
        }
    } catch (const std::bad_alloc &) {
        return fail(GQ_ERR_NOMEM, "out of host memory rebuilding the trees");
    }
    s->trees_ready = true;
    return GQ_OK;
}

// Built-in launch choices (measured on B200 for the benchmark scenes).
void default_tuning(gq_scene *s) {
    for (int k = 0; k < 3; ++k) s->tune[k] = gq_tuning{GQ_VARIANT_EXACT, 0, 1, 0, 32};
    // one query per warp for few queries, warp-coherent from 2^18 on (packet = 1)
    s->tune[GQ_KIND_SILHOUETTE] = gq_tuning{GQ_VARIANT_WARP, 1, 1, 1, 32};
    if (s->dim == 3) {
        s->tune[GQ_KIND_CLOSEST_POINT] = gq_tuning{GQ_VARIANT_COHERENT, 1, 1, 0, 32};
        s->tune[GQ_KIND_INTERSECT] = gq_tuning{s->has_wide ? GQ_VARIANT_WIDE8 : GQ_VARIANT_EXACT, 0, 1, 1, 32};
    } else {
        s->tune[GQ_KIND_CLOSEST_POINT] = gq_tuning{GQ_VARIANT_COHERENT, 1, 1, 0, 32};
        s->tune[GQ_KIND_INTERSECT] = gq_tuning{s->has_wide ? GQ_VARIANT_WIDE8 : GQ_VARIANT_EXACT, 0, 1, 1, 32};
    }
}

// Launch choices of one call: the tuning entry of `kind`, with the short warp-coherent
// stack kept only when the tree fits in it (the binary walk keeps at most one entry per
// level, the 8-wide walk up to seven).
gqd::Tune to_tune(const gq_scene *s, int kind, int variant) {
    const gq_tuning &t = s->tune[kind];
    gqd::Tune r;
    r.packet = t.packet;
    r.sorted = t.sorted;
    r.persist = t.persist;
    r.budget = t.budget > 0 ? t.budget : 32;
    r.block = t.block > 0 ? t.block : 128;
    const int need = (variant == GQ_VARIANT_WIDE8 || variant == GQ_VARIANT_WIDE16) ? s->wide_stack : s->exact_stack;
    r.stack = (t.stack == 32 && need <= 32) ? 32 : 0;
    return r;
}

int resolve_variant(const gq_scene *s, const gq_query_opts *opts, int kind) {
    int v = opts ? opts->variant : GQ_VARIANT_AUTO;
    if (v == GQ_VARIANT_AUTO) {
        v = s->tune[kind].variant;
        if (v == GQ_VARIANT_WIDE8 && !s->has_wide) v = GQ_VARIANT_EXACT;
        if (v == GQ_VARIANT_WIDE16 && !s->has_wide16) v = GQ_VARIANT_EXACT;
    }
    return v;
}

gq_status check_variant(const gq_scene *s, int v) {
    if (v == GQ_VARIANT_COHERENT) {
        if (s->exact_stack > GQ_STACK_EXACT)
            return fail(GQ_ERR_DEPTH, "tree deeper than the 64-entry traversal stack");
    } else if (v == GQ_VARIANT_WIDE8 || v == GQ_VARIANT_WIDE16) {
        if (!s->has_wide) return fail(GQ_ERR_UNSUPPORTED, "scene was built without the wide BVH");
        if (v == GQ_VARIANT_WIDE16 && !s->has_wide16)
            return fail(GQ_ERR_UNSUPPORTED, "scene was built without the 16-bit child bounds (build_wide = 2)");
        if (s->wide_stack > GQ_STACK_WIDE) return fail(GQ_ERR_DEPTH, "wide tree needs a deeper stack than 96");
    } else if (v == GQ_VARIANT_EXACT) {
        if (s->exact_stack > GQ_STACK_EXACT)
            return fail(GQ_ERR_DEPTH, "tree deeper than gQuery's 64-entry traversal stack");
    } else {
        return fail(GQ_ERR_INVALID, "unknown variant");
    }
    return GQ_OK;
}

bool vecs_ok(const gq_vecs &v) { return v.ptr != nullptr; }

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kCounterBytes = 256;

// Stream-ordered scratch for the Morton permutation (caller-provided or allocated).
struct Scratch {
    void *p = nullptr;
    bool owned = false;
    cudaStream_t st = nullptr;
    ~Scratch() {
        if (owned && p) cudaFreeAsync(p, st);
    }
};

// Per-call scratch: [work counter, 256 B][permutation, n int32][Morton sort workspace].
// The counter feeds the persistent wide kernels; the rest is used when sorting.

// ray_dirs (3D rays): the rays are keyed by origin and direction (gq_ray_order mode 2),
// which keeps the rays of a warp pointing alike.
gq_status prepare_order(const gq_scene *s, gq_vecs keys_from, int64_t n, const gq_query_opts *opts,
                        cudaStream_t st, Scratch &scr, const int32_t **perm, unsigned long long **counter,
                        const gq_vecs *ray_dirs = nullptr) {
    *perm = nullptr;
    *counter = nullptr;
    const bool sorting = opts && !opts->order && opts->sort && n >= 2;
    const size_t need = sorting ? (size_t)gq_query_scratch_bytes(n) : kCounterBytes;
    if (opts && opts->scratch) {
        if ((size_t)opts->scratch_bytes < need) return fail(GQ_ERR_INVALID, "scratch buffer too small");
        scr.p = opts->scratch;
    } else {
        cudaError_t e = cudaMallocAsync(&scr.p, need, st);
        if (e != cudaSuccess) return fail(GQ_ERR_NOMEM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
        scr.owned = true;
        scr.st = st;
    }
    *counter = (unsigned long long *)scr.p;
    if (opts && opts->order) {
        *perm = opts->order;
        return GQ_OK;
    }
    if (!sorting) return GQ_OK;
    int32_t *pp = (int32_t *)((char *)scr.p + kCounterBytes);
    char *rest = (char *)pp + align256((size_t)n * 4);
    const bool ray_keys = ray_dirs && s->dim == 3;
    cudaError_t e = gqd::morton_order(s->dev, keys_from, n, pp, rest, gqd::morton_scratch_bytes(n), st,
                                      ray_keys ? 2 : 0, ray_keys ? *ray_dirs : gq_vecs{});
    if (e != cudaSuccess) return fail_cuda(e, "morton_order");
    *perm = pp;
    return GQ_OK;
}

}  // namespace


struct gq_batch {
    int dim = 0;
    int device = 0;
    int flags = 0;
    std::vector<gq_scene *> scenes;
    int64_t max_queries = 0;
    gqd::DevScene *dev_scenes = nullptr;
    void *scratch = nullptr;
    int32_t *err = nullptr;
    int64_t device_bytes = 0;

    ~gq_batch() {
        DeviceGuard g(device);
        if (dev_scenes) cudaFree(dev_scenes);
        if (scratch) cudaFree(scratch);
        if (err) cudaFree(err);
    }
};

extern "C" {

void gq_last_error(char *buf, int64_t cap) {
    if (!buf || cap <= 0) return;
    std::snprintf(buf, (size_t)cap, "%s", g_last_error.c_str());
}

const char *gq_status_string(gq_status s) {
    switch (s) {
        case GQ_OK: return "ok";
        case GQ_ERR_INVALID: return "invalid argument";
        case GQ_ERR_CUDA: return "CUDA error";
        case GQ_ERR_NOMEM: return "out of memory";
        case GQ_ERR_DEPTH: return "tree too deep for the traversal stack";
        case GQ_ERR_DEVICE: return "device error flag raised";
        case GQ_ERR_UNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}

gq_status gq_scene_build_2d(const float *vertices, int64_t nv, const int32_t *edges, int64_t ne,
                            const gq_build_opts *opts, gq_scene **out) {
    return build_scene<2>(vertices, nv, edges, ne, opts, out);
}

gq_status gq_scene_build_3d(const float *vertices, int64_t nv, const int32_t *faces, int64_t nf,
                            const gq_build_opts *opts, gq_scene **out) {
    return build_scene<3>(vertices, nv, faces, nf, opts, out);
}

gq_status gq_scene_free(gq_scene *scene) {
    delete scene;
    return GQ_OK;
}

gq_status gq_scene_set_tuning(gq_scene *s, int32_t kind, const gq_tuning *t) {
    if (!s || !t) return fail(GQ_ERR_INVALID, "null argument");
    if (kind < 0 || kind > 2) return fail(GQ_ERR_INVALID, "unknown query kind");
    if (t->variant < 0 || t->variant > 5 || t->variant == GQ_VARIANT_AUTO)
        return fail(GQ_ERR_INVALID, "tuning variant must be EXACT, WIDE8, COHERENT, WARP or WIDE16");
    if (t->variant == GQ_VARIANT_WIDE16 && (kind == GQ_KIND_SILHOUETTE || !s->has_wide16))
        return fail(GQ_ERR_UNSUPPORTED, "WIDE16 answers closest points and rays of scenes built with build_wide = 2");
    if (t->variant == GQ_VARIANT_WARP && kind != GQ_KIND_SILHOUETTE)
        return fail(GQ_ERR_INVALID, "the WARP variant answers silhouette queries only");
    if (t->variant == GQ_VARIANT_WIDE8 && !s->has_wide) return fail(GQ_ERR_UNSUPPORTED, "scene has no wide BVH");
    if (t->block != 0 && t->block != 64 && t->block != 128 && t->block != 256)
        return fail(GQ_ERR_INVALID, "block must be 0 (default), 64, 128 or 256");
    if (t->stack != 0 && t->stack != 32) return fail(GQ_ERR_INVALID, "stack must be 0 (full depth) or 32");
    if (t->budget < 0) return fail(GQ_ERR_INVALID, "budget must be >= 0");
    s->tune[kind] = *t;
    return GQ_OK;
}

gq_status gq_scene_get_tuning(const gq_scene *s, int32_t kind, gq_tuning *t) {
    if (!s || !t) return fail(GQ_ERR_INVALID, "null argument");
    if (kind < 0 || kind > 2) return fail(GQ_ERR_INVALID, "unknown query kind");
    *t = s->tune[kind];
    return GQ_OK;
}

gq_status gq_scene_get_info(const gq_scene *s, gq_scene_info *info) {
    if (!s || !info) return fail(GQ_ERR_INVALID, "null argument");
    std::memset(info, 0, sizeof *info);
    info->dim = s->dim;
    info->n_vertices = s->nv;
    info->n_prims = s->np;
    info->n_nodes = s->n_nodes;
    info->n_wide_nodes = s->n_wide;
    info->n_silhouettes = s->n_sil;
    info->max_depth = s->max_depth;
    info->exact_stack = s->exact_stack;
    info->wide_stack = s->wide_stack;
    info->device_bytes = s->device_bytes;
    for (int k = 0; k < 3; ++k) {
        info->bbox_lo[k] = s->dev.root_lo[k];
        info->bbox_hi[k] = s->dev.root_hi[k];
    }
    return GQ_OK;
}

gq_status gq_scene_ref_array(const gq_scene *s, int32_t which, float *dst, int64_t cap, int64_t *len) {
    if (!s || !len) return fail(GQ_ERR_INVALID, "null argument");
    std::vector<float> v;
    if (which == GQ_ARRAY_WIDE_NODES || which == GQ_ARRAY_SNCH_PAIRS || which == GQ_ARRAY_SIL_RECORDS ||
        which == GQ_ARRAY_WIDE16_BOUNDS) {
        if (s->device >= 0) return fail(GQ_ERR_UNSUPPORTED, "device record dumps are kept for host-only scenes");
        const std::vector<float> &w = which == GQ_ARRAY_WIDE_NODES     ? s->wide_words
                                      : which == GQ_ARRAY_SNCH_PAIRS   ? s->spair_words
                                      : which == GQ_ARRAY_WIDE16_BOUNDS ? s->wide16_words
                                                                       : s->sil_words;
        *len = (int64_t)w.size();
        if (dst && cap > 0) std::memcpy(dst, w.data(), sizeof(float) * (size_t)std::min<int64_t>(cap, *len));
        return GQ_OK;
    }
    const bool snch_needed = which == GQ_ARRAY_SNCH_NODES || which == GQ_ARRAY_SILHOUETTES ||
                             which == GQ_ARRAY_RAW_SILHOUETTES;
    if (snch_needed && !s->has_snch) return fail(GQ_ERR_UNSUPPORTED, "scene was built without the SNCH");
    if (s->gpu_built)
        return fail(GQ_ERR_UNSUPPORTED, "scene was built on the device; the reference arrays describe the host SAH build");
    gq_status tst = ensure_trees(const_cast<gq_scene *>(s));
    if (tst != GQ_OK) return tst;
    if (s->dim == 2) {
        PrimSource<2> src{s->verts.data(), s->nv, s->index.data(), s->np};
        switch (which) {
            case GQ_ARRAY_BVH_NODES: v = ref_node_data<2>(s->t2); break;
            case GQ_ARRAY_PRIMITIVES: v = ref_prim_data<2>(src, s->t2); break;
            case GQ_ARRAY_SNCH_NODES: v = ref_snch_node_data<2>(s->t2, s->s2); break;
            case GQ_ARRAY_SILHOUETTES: v = ref_silhouette_data<2>(s->s2, true); break;
            case GQ_ARRAY_RAW_SILHOUETTES: v = ref_silhouette_data<2>(s->s2, false); break;
            default: return fail(GQ_ERR_INVALID, "unknown array id");
        }
    } else {
        PrimSource<3> src{s->verts.data(), s->nv, s->index.data(), s->np};
        switch (which) {
            case GQ_ARRAY_BVH_NODES: v = ref_node_data<3>(s->t3); break;
            case GQ_ARRAY_PRIMITIVES: v = ref_prim_data<3>(src, s->t3); break;
            case GQ_ARRAY_SNCH_NODES: v = ref_snch_node_data<3>(s->t3, s->s3); break;
            case GQ_ARRAY_SILHOUETTES: v = ref_silhouette_data<3>(s->s3, true); break;
            case GQ_ARRAY_RAW_SILHOUETTES: v = ref_silhouette_data<3>(s->s3, false); break;
            default: return fail(GQ_ERR_INVALID, "unknown array id");
        }
    }
    *len = (int64_t)v.size();
    if (dst && cap > 0) std::memcpy(dst, v.data(), sizeof(float) * (size_t)std::min<int64_t>(cap, *len));
    return GQ_OK;
}

gq_status gq_flat_silhouette_edges(const float *vertices, int64_t nv, const int32_t *faces, int64_t nf, float *dst,
                                   int64_t cap, int64_t *len) {
    if (!vertices || !faces || !len) return fail(GQ_ERR_INVALID, "null argument");
    PrimSource<3> src{vertices, nv, faces, nf};
    std::string bad = validate_source<3>(src);
    if (!bad.empty()) return fail(GQ_ERR_INVALID, bad);
    SnchTree<3> tmp;
    tmp.raw = build_silhouette_edges(src, nullptr);
    std::vector<float> v = ref_silhouette_data<3>(tmp, false);
    *len = (int64_t)v.size();
    if (dst && cap > 0) std::memcpy(dst, v.data(), sizeof(float) * (size_t)std::min<int64_t>(cap, *len));
    return GQ_OK;
}

gq_status gq_flat_silhouette_edges_device(const float *vertices, int64_t nv, const int32_t *faces, int64_t nf,
                                          float *dst, int64_t cap, int64_t *len, int32_t device, void *stream) {
    if (!len || (nf > 0 && (!vertices || !faces))) return fail(GQ_ERR_INVALID, "null argument");
    if (nv < 0 || nf < 0 || nf > (int64_t)(INT32_MAX / 3)) return fail(GQ_ERR_INVALID, "bad vertex or face count");
    DeviceGuard g(device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the device");
    int64_t n_edges = 0;
    int bad = 0;
    const int64_t cap_edges = dst ? cap / 19 : 0;
    cudaError_t e = gqd::gpu_silhouette_edges(vertices, nv, faces, nf, dst, cap_edges, &n_edges, &bad,
                                              (cudaStream_t)stream);
    if (e != cudaSuccess) return fail_cuda(e, "device silhouette edges");
    if (bad) return fail(GQ_ERR_INVALID, "face index out of range");
    *len = n_edges * 19;
    if (dst && cap_edges < n_edges) return fail(GQ_ERR_INVALID, "destination holds fewer floats than *len");
    return GQ_OK;
}

int64_t gq_query_scratch_bytes(int64_t n) {
    if (n <= 0) return 0;
    return (int64_t)(kCounterBytes + align256((size_t)n * 4) + gqd::morton_scratch_bytes(n));
}

int64_t gq_order_scratch_bytes(int64_t n) {
    if (n <= 0) return 0;
    return (int64_t)gqd::morton_scratch_bytes(n);
}

static gq_status order_impl(const gq_scene *s, gq_vecs points, int64_t n, int32_t *order, void *scratch,
                            int64_t scratch_bytes, void *stream, int ray_mode, gq_vecs dirs);

gq_status gq_ray_order(const gq_scene *s, gq_vecs origins, gq_vecs dirs, int64_t n, int32_t mode, int32_t *order,
                       void *scratch, int64_t scratch_bytes, void *stream) {
    if (!s || !order) return fail(GQ_ERR_INVALID, "null scene or order");
    if (mode < 0 || mode > 2) return fail(GQ_ERR_INVALID, "ray order mode must be 0, 1 or 2");
    if (mode > 0 && s->dim != 3) return fail(GQ_ERR_UNSUPPORTED, "direction keys are for 3D scenes");
    if (n > 0 && mode > 0 && !vecs_ok(dirs)) return fail(GQ_ERR_INVALID, "null direction array");
    return order_impl(s, origins, n, order, scratch, scratch_bytes, stream, mode, dirs);
}

gq_status gq_query_order(const gq_scene *s, gq_vecs points, int64_t n, int32_t *order, void *scratch,
                         int64_t scratch_bytes, void *stream) {
    if (!s || !order) return fail(GQ_ERR_INVALID, "null scene or order");
    return order_impl(s, points, n, order, scratch, scratch_bytes, stream, 0, gq_vecs{});
}

static gq_status order_impl(const gq_scene *s, gq_vecs points, int64_t n, int32_t *order, void *scratch,
                            int64_t scratch_bytes, void *stream, int ray_mode, gq_vecs dirs) {
    if (n < 0) return fail(GQ_ERR_INVALID, "negative count");
    if (n == 0) return GQ_OK;
    if (!vecs_ok(points)) return fail(GQ_ERR_INVALID, "null point array");
    if (on_host_only(s)) return fail(GQ_ERR_UNSUPPORTED, "scene was built without a device copy");
    DeviceGuard g(s->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's CUDA device");
    cudaStream_t cs = (cudaStream_t)stream;
    const size_t need = gqd::morton_scratch_bytes(n);
    Scratch scr;
    if (scratch) {
        if ((size_t)scratch_bytes < need) return fail(GQ_ERR_INVALID, "scratch buffer too small");
        scr.p = scratch;
    } else {
        cudaError_t e = cudaMallocAsync(&scr.p, need, cs);
        if (e != cudaSuccess) return fail(GQ_ERR_NOMEM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
        scr.owned = true;
        scr.st = cs;
    }
    cudaError_t e = gqd::morton_order(s->dev, points, n, order, scr.p, need, cs, ray_mode, dirs);
    if (e != cudaSuccess) return fail_cuda(e, "morton_order");
    return GQ_OK;
}

gq_status gq_closest_point(const gq_scene *s, gq_vecs q, int64_t n, const gq_cp_out *out, const gq_query_opts *opts,
                           void *stream) {
    if (!s || !out) return fail(GQ_ERR_INVALID, "null scene or output");
    if (n < 0) return fail(GQ_ERR_INVALID, "negative query count");
    if (n == 0) return GQ_OK;
    if (!vecs_ok(q)) return fail(GQ_ERR_INVALID, "null query array");
    const int v = resolve_variant(s, opts, GQ_KIND_CLOSEST_POINT);
    gq_status st = check_variant(s, v);
    if (st != GQ_OK) return st;
    if (on_host_only(s)) return fail(GQ_ERR_UNSUPPORTED, "scene was built without a device copy");
    DeviceGuard g(s->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's CUDA device");
    cudaStream_t cs = (cudaStream_t)stream;
    Scratch scr;
    const int32_t *perm = nullptr;
    unsigned long long *counter = nullptr;
    if ((st = prepare_order(s, q, n, opts, cs, scr, &perm, &counter)) != GQ_OK) return st;
    cudaError_t e = gqd::launch_cp(s->dev, v, to_tune(s, GQ_KIND_CLOSEST_POINT, v), q, n, perm, *out, counter, cs);
    if (e != cudaSuccess) return fail_cuda(e, "closest_point launch");
    return GQ_OK;
}

int64_t gq_noalloc_max_queries(void) { return gqd::noalloc_max_queries(); }

gq_status gq_closest_point_noalloc(const gq_scene *s, gq_vecs q, int64_t n, const gq_cp_out *out, int32_t variant,
                                   int32_t sort, void *stream) {
    if (!s || !out) return fail(GQ_ERR_INVALID, "null scene or output");
    if (n < 0) return fail(GQ_ERR_INVALID, "negative query count");
    if (n > gqd::noalloc_max_queries())
        return fail(GQ_ERR_INVALID, "gq_closest_point_noalloc takes at most " +
                                        std::to_string(gqd::noalloc_max_queries()) + " queries per call");
    if (n == 0) return GQ_OK;
    if (!vecs_ok(q)) return fail(GQ_ERR_INVALID, "null query array");
    gq_query_opts o{};
    o.variant = variant;
    const int v = resolve_variant(s, &o, GQ_KIND_CLOSEST_POINT);
    gq_status st = check_variant(s, v);
    if (st != GQ_OK) return st;
    if (on_host_only(s)) return fail(GQ_ERR_UNSUPPORTED, "scene was built without a device copy");
    DeviceGuard g(s->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's CUDA device");
    cudaError_t e = gqd::noalloc_closest_point(s->dev, v, to_tune(s, GQ_KIND_CLOSEST_POINT, v), q, n, sort,
                                               *out, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail_cuda(e, "closest_point_noalloc");
    return GQ_OK;
}

gq_status gq_intersect(const gq_scene *s, gq_vecs origin, gq_vecs dir, const float *r_max, int64_t n,
                       const gq_ray_out *out, const gq_query_opts *opts, void *stream) {
    if (!s || !out) return fail(GQ_ERR_INVALID, "null scene or output");
    if (n < 0) return fail(GQ_ERR_INVALID, "negative query count");
    if (n == 0) return GQ_OK;
    if (!vecs_ok(origin) || !vecs_ok(dir)) return fail(GQ_ERR_INVALID, "null ray array");
    const int v = resolve_variant(s, opts, GQ_KIND_INTERSECT);
    gq_status st = check_variant(s, v);
    if (st != GQ_OK) return st;
    if (on_host_only(s)) return fail(GQ_ERR_UNSUPPORTED, "scene was built without a device copy");
    DeviceGuard g(s->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's CUDA device");
    cudaStream_t cs = (cudaStream_t)stream;
    Scratch scr;
    const int32_t *perm = nullptr;
    unsigned long long *counter = nullptr;
    if ((st = prepare_order(s, origin, n, opts, cs, scr, &perm, &counter, &dir)) != GQ_OK) return st;
    cudaError_t e = gqd::launch_ray(s->dev, v, to_tune(s, GQ_KIND_INTERSECT, v), origin, dir, r_max, n, perm,
                                    *out, counter, cs);
    if (e != cudaSuccess) return fail_cuda(e, "intersect launch");
    return GQ_OK;
}

gq_status gq_closest_silhouette(const gq_scene *s, gq_vecs x, const float *r_max, int64_t n, const gq_sil_out *out,
                                const gq_query_opts *opts, void *stream) {
    if (!s || !out) return fail(GQ_ERR_INVALID, "null scene or output");
    if (n < 0) return fail(GQ_ERR_INVALID, "negative query count");
    if (n == 0) return GQ_OK;
    if (!vecs_ok(x)) return fail(GQ_ERR_INVALID, "null query array");
    if (!s->has_snch) return fail(GQ_ERR_UNSUPPORTED, "scene was built without the SNCH");
    if (s->exact_stack > GQ_STACK_EXACT) return fail(GQ_ERR_DEPTH, "tree deeper than gQuery's 64-entry stack");
    if (on_host_only(s)) return fail(GQ_ERR_UNSUPPORTED, "scene was built without a device copy");
    int v = resolve_variant(s, opts, GQ_KIND_SILHOUETTE);
    if ((!opts || opts->variant == GQ_VARIANT_AUTO) && v == GQ_VARIANT_WARP && s->tune[GQ_KIND_SILHOUETTE].packet &&
        n >= kSilCoherentFrom)
        v = GQ_VARIANT_COHERENT;  // many queries: neighbours share their walks
    if (v != GQ_VARIANT_EXACT && v != GQ_VARIANT_COHERENT && v != GQ_VARIANT_WARP)
        return fail(GQ_ERR_UNSUPPORTED, "silhouette queries run the exact, coherent or warp variant");
    DeviceGuard g(s->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's CUDA device");
    cudaStream_t cs = (cudaStream_t)stream;
    Scratch scr;
    const int32_t *perm = nullptr;
    unsigned long long *counter = nullptr;
    gq_status st;
    if ((st = prepare_order(s, x, n, opts, cs, scr, &perm, &counter)) != GQ_OK) return st;
    cudaError_t e = gqd::launch_sil(s->dev, v, to_tune(s, GQ_KIND_SILHOUETTE, v), x, r_max, n, perm, *out, counter,
                                    cs);
    if (e != cudaSuccess) return fail_cuda(e, "closest_silhouette launch");
    return GQ_OK;
}

gq_status gq_closest_point_brute(const gq_scene *s, gq_vecs q, int64_t n, const gq_cp_out *out, void *stream) {
    if (!s || !out) return fail(GQ_ERR_INVALID, "null scene or output");
    if (n < 0) return fail(GQ_ERR_INVALID, "negative query count");
    if (n == 0) return GQ_OK;
    if (!vecs_ok(q)) return fail(GQ_ERR_INVALID, "null query array");
    if (on_host_only(s)) return fail(GQ_ERR_UNSUPPORTED, "scene was built without a device copy");
    DeviceGuard g(s->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's CUDA device");
    cudaError_t e = gqd::launch_cp_brute(s->dev, q, n, *out, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail_cuda(e, "closest_point_brute launch");
    return GQ_OK;
}

gq_status gq_intersect_brute(const gq_scene *s, gq_vecs origin, gq_vecs dir, const float *r_max, int64_t n,
                             const gq_ray_out *out, void *stream) {
    if (!s || !out) return fail(GQ_ERR_INVALID, "null scene or output");
    if (n < 0) return fail(GQ_ERR_INVALID, "negative query count");
    if (n == 0) return GQ_OK;
    if (!vecs_ok(origin) || !vecs_ok(dir)) return fail(GQ_ERR_INVALID, "null ray array");
    if (on_host_only(s)) return fail(GQ_ERR_UNSUPPORTED, "scene was built without a device copy");
    DeviceGuard g(s->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's CUDA device");
    cudaError_t e = gqd::launch_ray_brute(s->dev, origin, dir, r_max, n, *out, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail_cuda(e, "intersect_brute launch");
    return GQ_OK;
}

// Uploads (once) the list closest_silhouette_baseline scans: a Mesh's unique edges in
// first-appearance order (build_flat_silhouette_edges), a Polyline's silhouette
// vertices (Polyline.configure_silhouette).
static gq_status ensure_base_sils(gq_scene *s) {
    std::lock_guard<std::mutex> lk(s->base_mu);
    if (s->n_base_sils >= 0) return GQ_OK;
    try {
        gq_status st = GQ_OK;
        if (s->dim == 2) {
            PrimSource<2> src{s->verts.data(), s->nv, s->index.data(), s->np};
            const std::vector<gqb::SilVertex> raw = gqb::build_polyline_silhouettes(src);
            std::vector<gq_silv_t> rec(raw.size());
            for (size_t k = 0; k < raw.size(); ++k) gqb::device_silhouette(raw[k], rec[k]);
            if (!rec.empty()) st = s->upload(rec, &s->base_sils);
            if (st == GQ_OK) s->n_base_sils = (int64_t)rec.size();
        } else {
            PrimSource<3> src{s->verts.data(), s->nv, s->index.data(), s->np};
            const std::vector<gqb::SilEdge> raw = gqb::build_silhouette_edges(src, nullptr);
            std::vector<gq_sile_t> rec(raw.size());
            for (size_t k = 0; k < raw.size(); ++k) gqb::device_silhouette(raw[k], rec[k]);
            if (!rec.empty()) st = s->upload(rec, &s->base_sils);
            if (st == GQ_OK) s->n_base_sils = (int64_t)rec.size();
        }
        return st;
    } catch (const std::bad_alloc &) {
        return fail(GQ_ERR_NOMEM, "out of host memory building the silhouette list");
    }
}

gq_status gq_closest_silhouette_brute(const gq_scene *s, gq_vecs x, const float *r_max, int64_t n,
                                      const gq_sil_out *out, void *stream) {
    if (!s || !out) return fail(GQ_ERR_INVALID, "null scene or output");
    if (n < 0) return fail(GQ_ERR_INVALID, "negative query count");
    if (n == 0) return GQ_OK;
    if (!vecs_ok(x)) return fail(GQ_ERR_INVALID, "null query array");
    if (on_host_only(s)) return fail(GQ_ERR_UNSUPPORTED, "scene was built without a device copy");
    DeviceGuard g(s->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's device");
    gq_status st = ensure_base_sils(const_cast<gq_scene *>(s));
    if (st != GQ_OK) return st;
    cudaError_t e = gqd::launch_sil_brute(s->dev, s->base_sils, s->n_base_sils, x, r_max, n, *out, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail_cuda(e, "closest_silhouette_brute launch");
    return GQ_OK;
}

// Uploads (once) the SNCH's raw silhouette list (one record per polyline vertex, one per
// unique mesh edge) as float positions for the FP64 silhouette scan: 2D a, b, c, flag
// (1 = both neighbours exist), 3D a, b, c, d, flag (1 = boundary edge, always a
// silhouette; the reference's size_t indices never hold -1, so this stays 0).
static gq_status ensure_f64_sils(gq_scene *s) {
    std::lock_guard<std::mutex> lk(s->base_mu);
    if (s->n_f64_sils >= 0) return GQ_OK;
    gq_status st = ensure_trees(s);
    if (st != GQ_OK) return st;
    try {
        std::vector<float> rec;
        int64_t n = 0;
        if (s->dim == 2) {
            for (const gqb::SilVertex &x : s->s2.raw) {
                const bool ok = ((int64_t)(float)x.idx[0] != -1) && ((int64_t)(float)x.idx[2] != -1);
                const float r[8] = {x.v[0].v[0], x.v[0].v[1], x.v[1].v[0], x.v[1].v[1],
                                    x.v[2].v[0], x.v[2].v[1], ok ? 1.f : 0.f, 0.f};
                rec.insert(rec.end(), r, r + 8);
                ++n;
            }
        } else {
            for (const gqb::SilEdge &x : s->s3.raw) {
                const bool boundary = ((int64_t)(float)x.idx[0] == -1) || ((int64_t)(float)x.idx[3] == -1);
                float r[16] = {};
                const int order[4] = {1, 2, 0, 3};  // a, b, c, d of silhouette_edge.py:75-86
                for (int k = 0; k < 4; ++k)
                    for (int c = 0; c < 3; ++c) r[3 * k + c] = x.v[order[k]].v[c];
                r[12] = boundary ? 1.f : 0.f;
                rec.insert(rec.end(), r, r + 16);
                ++n;
            }
        }
        if (!rec.empty()) st = s->upload(rec, &s->f64_sils);
        if (st == GQ_OK) s->n_f64_sils = n;
        return st;
    } catch (const std::bad_alloc &) {
        return fail(GQ_ERR_NOMEM, "out of host memory building the FP64 silhouette list");
    }
}

gq_status gq_brute_f64(const gq_scene *s, int32_t kind, gq_vecs a, gq_vecs b, int64_t n, double *out_d,
                       int32_t *out_id, void *stream) {
    if (!s || !out_d || !out_id) return fail(GQ_ERR_INVALID, "null argument");
    if (kind == 2) {
        if (n < 0) return fail(GQ_ERR_INVALID, "negative query count");
        if (n == 0) return GQ_OK;
        if (!vecs_ok(a)) return fail(GQ_ERR_INVALID, "null query array");
        if (on_host_only(s)) return fail(GQ_ERR_UNSUPPORTED, "scene was built without a device copy");
        if (!s->has_snch) return fail(GQ_ERR_UNSUPPORTED, "scene was built without the SNCH");
        if (s->gpu_built) return fail(GQ_ERR_UNSUPPORTED, "scene was built on the device: no host silhouette list");
        DeviceGuard g(s->device);
        if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's CUDA device");
        gq_status st = ensure_f64_sils(const_cast<gq_scene *>(s));
        if (st != GQ_OK) return st;
        cudaError_t e = gqd::launch_sil_f64(s->dim, (const float *)s->f64_sils, s->n_f64_sils, a, n, out_d, out_id,
                                            (cudaStream_t)stream);
        if (e != cudaSuccess) return fail_cuda(e, "brute_f64 silhouette launch");
        return GQ_OK;
    }
    if (kind != 0 && kind != 1) return fail(GQ_ERR_INVALID, "kind must be 0, 1 or 2");
    if (n < 0) return fail(GQ_ERR_INVALID, "negative query count");
    if (n == 0) return GQ_OK;
    if (!vecs_ok(a) || (kind == 1 && !vecs_ok(b))) return fail(GQ_ERR_INVALID, "null query array");
    if (on_host_only(s)) return fail(GQ_ERR_UNSUPPORTED, "scene was built without a device copy");
    DeviceGuard g(s->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's CUDA device");
    cudaError_t e = gqd::launch_brute_f64(s->dev, kind, a, b, n, out_d, out_id, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail_cuda(e, "brute_f64 launch");
    return GQ_OK;
}

namespace {

// Saved scene: header, then the input geometry and the six device arrays, raw.
struct SceneFileHeader {
    char magic[8];
    int32_t version, dim;
    int64_t nv, np;
    int32_t max_prims_in_node, has_snch, has_wide, exact_stack, wide_stack, max_depth;
    int64_t n_nodes, n_wide, n_sil;
    int32_t root_ref, wroot_ref, sroot_ref, gpu_built;
    float root_lo[3], root_hi[3], coord_bound, pad2;
    uint64_t image_bytes[6];
};
static_assert(sizeof(SceneFileHeader) == 176, "the scene file header is 176 bytes");
constexpr char kSceneMagic[8] = {'G', 'Q', 'S', 'C', 'E', 'N', 'E', '1'};
// 2: 3D silhouette edges carry the pre-test spans (gq_sile_t.span0 / span1)
// 3: 3D SNCH pairs carry the node bounds of both children (gq_spair3_t.l_b / r_b)
// 5: the node bounds hold the delta and cone forms and the pair record is 160 B
// 6: wide nodes hold run children (small subtrees as one leaf); files of version 5 have
//    none and load unchanged
constexpr int32_t kSceneFileVersion = 6;

struct File {
    FILE *f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

}  // namespace

gq_status gq_scene_save(const gq_scene *s, const char *path) {
    if (!s || !path) return fail(GQ_ERR_INVALID, "null argument");
    if (on_host_only(s)) return fail(GQ_ERR_UNSUPPORTED, "only scenes with a device copy can be saved");
    SceneFileHeader h{};
    std::memcpy(h.magic, kSceneMagic, 8);
    h.version = kSceneFileVersion;
    h.dim = s->dim;
    h.nv = s->nv;
    h.np = s->np;
    h.max_prims_in_node = s->max_prims_in_node;
    h.has_snch = s->has_snch;
    h.has_wide = s->has_wide;
    h.exact_stack = s->exact_stack;
    h.wide_stack = s->wide_stack;
    h.max_depth = s->max_depth;
    h.n_nodes = s->n_nodes;
    h.n_wide = s->n_wide;
    h.n_sil = s->n_sil;
    h.root_ref = s->dev.root_ref;
    h.wroot_ref = s->dev.wroot_ref;
    h.sroot_ref = s->dev.sroot_ref;
    h.gpu_built = s->gpu_built;
    for (int k = 0; k < 3; ++k) h.root_lo[k] = s->dev.root_lo[k], h.root_hi[k] = s->dev.root_hi[k];
    h.coord_bound = s->dev.coord_bound;
    for (int k = 0; k < 6; ++k) h.image_bytes[k] = s->image_bytes[k];
    const void *dev_arrays[6] = {s->dev.pairs, s->dev.prims, s->dev.spheres, s->dev.wnodes, s->dev.spairs,
                                 s->dev.sils};
    File out;
    out.f = std::fopen(path, "wb");
    if (!out.f) return fail(GQ_ERR_INVALID, std::string("cannot open ") + path + " for writing");
    bool ok = std::fwrite(&h, sizeof h, 1, out.f) == 1;
    ok = ok && std::fwrite(s->verts.data(), sizeof(float), s->verts.size(), out.f) == s->verts.size();
    ok = ok && std::fwrite(s->index.data(), sizeof(int32_t), s->index.size(), out.f) == s->index.size();
    DeviceGuard g(s->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's CUDA device");
    std::vector<char> buf;
    for (int k = 0; k < 6 && ok; ++k) {
        if (!h.image_bytes[k]) continue;
        buf.resize(h.image_bytes[k]);
        cudaError_t e = cudaMemcpy(buf.data(), dev_arrays[k], buf.size(), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return fail_cuda(e, "scene save");
        ok = std::fwrite(buf.data(), 1, buf.size(), out.f) == buf.size();
    }
    if (!ok || std::fflush(out.f) != 0) return fail(GQ_ERR_INVALID, std::string("write failed: ") + path);
    return GQ_OK;
}

// Structure of a loaded scene image, checked on the host before anything reaches the
// device: the kernels follow its references without bounds checks.  Returns an empty
// string when the arrays agree with the header and with each other: every interior
// reference names a record of its own array that no other reference and not the root
// names (each node has at most one parent, so no walk meets a node twice and every
// walk ends, whatever the numbering: host trees are in preorder, device-built ones in
// the order of the sorted keys), every leaf starts inside its item array and the
// array's last item ends a leaf (so every leaf scan ends), the roots are valid, and
// the wide nodes' used slots follow the same rules.
static std::string check_image(const SceneFileHeader &h, const std::vector<char> (&a)[6]) {
    const bool d3 = h.dim == 3;
    const size_t s_pair = d3 ? sizeof(gq_pair3_t) : sizeof(gq_pair2_t);
    const size_t s_prim = d3 ? sizeof(gq_tri_t) : sizeof(gq_seg_t);
    const size_t s_wide = d3 ? sizeof(gq_wnode3_t) : sizeof(gq_wnode2_t);
    const size_t s_spair = d3 ? sizeof(gq_spair3_t) : sizeof(gq_spair2_t);
    const size_t s_sil = d3 ? sizeof(gq_sile_t) : sizeof(gq_silv_t);
    auto i32 = [&](int k, size_t byte) {
        int32_t v;
        std::memcpy(&v, a[k].data() + byte, 4);
        return v;
    };
    if (a[0].size() % s_pair || a[1].size() != (size_t)h.np * s_prim || a[3].size() % s_wide ||
        a[4].size() % s_spair || a[5].size() % s_sil)
        return "array sizes do not match the record sizes";
    if (d3 && !a[2].empty() && a[2].size() != (size_t)h.np * sizeof(gq_tsph_t)) return "sphere array size";
    const int64_t n_pair = (int64_t)(a[0].size() / s_pair), n_wide = (int64_t)(a[3].size() / s_wide);
    const int64_t n_spair = (int64_t)(a[4].size() / s_spair), n_sil = (int64_t)(a[5].size() / s_sil);
    if (n_wide != (h.has_wide ? h.n_wide : 0) || n_sil != h.n_sil) return "record counts differ from the header";
    if (h.np < 1) return "no primitives";
    const size_t f_prim = d3 ? offsetof(gq_tri_t, flags) : offsetof(gq_seg_t, flags);
    if (!(i32(1, (size_t)(h.np - 1) * s_prim + f_prim) & (int32_t)GQ_ITEM_LAST)) return "the last primitive ends no leaf";
    if (d3 && !a[2].empty()) {
        float r;
        std::memcpy(&r, a[2].data() + (size_t)(h.np - 1) * sizeof(gq_tsph_t) + offsetof(gq_tsph_t, r), 4);
        if (!std::signbit(r)) return "the last bounding sphere ends no leaf";
    }
    const size_t f_sil = d3 ? offsetof(gq_sile_t, flags) : offsetof(gq_silv_t, flags);
    if (n_sil > 0 && !(i32(5, (size_t)(n_sil - 1) * s_sil + f_sil) & (int32_t)GQ_ITEM_LAST))
        return "the last silhouette ends no leaf";
    // a reference into an array of n records over n_items items; `parents` counts the
    // references each record has had
    auto ref_ok = [](int32_t ref, int64_t n, int64_t n_items, bool empty_ok, std::vector<uint8_t> &parents,
                     bool runs_ok = false) {
        if (ref >= 0) return (int64_t)ref < n && parents[(size_t)ref]++ == 0;
        if (ref == INT32_MIN) return empty_ok;
        if (runs_ok && (ref & 0x40000000) == 0) {  // a run child: 1..GQ_COLLAPSE_MAX items
            const int64_t first = ref & 0xffffff, cnt = (ref >> 24) & 0x3f;
            return cnt >= 1 && cnt <= GQ_COLLAPSE_MAX && first + cnt <= n_items;
        }
        return (int64_t)~ref < n_items;
    };
    std::vector<uint8_t> parents;
    const size_t o_pref = d3 ? offsetof(gq_pair3_t, ref_l) : offsetof(gq_pair2_t, ref_l);
    parents.assign((size_t)n_pair, 0);
    if (!ref_ok(h.root_ref, n_pair, h.np, false, parents)) return "BVH root";
    const size_t o_sub = d3 ? offsetof(gq_pair3_t, sub_l) : offsetof(gq_pair2_t, sub_l);
    for (int64_t i = 0; i < n_pair; ++i)
        for (int c = 0; c < 2; ++c) {
            if (!ref_ok(i32(0, (size_t)i * s_pair + o_pref + 4 * c), n_pair, h.np, false, parents))
                return "a BVH pair references outside its arrays or a node twice";
            // a collapsed subtree's run: 1..GQ_COLLAPSE_MAX items inside the primitives
            const uint32_t sub = (uint32_t)i32(0, (size_t)i * s_pair + o_sub + 4 * c), cnt = sub >> 24;
            if (sub != 0 && (cnt < 1 || cnt > GQ_COLLAPSE_MAX || (int64_t)(sub & 0xffffffu) + cnt > h.np))
                return "a BVH pair's collapsed run lies outside the primitives";
        }
    if (h.has_wide) {
        const size_t o_meta = d3 ? offsetof(gq_wnode3_t, meta) : offsetof(gq_wnode2_t, meta);
        const size_t o_ref = d3 ? offsetof(gq_wnode3_t, ref) : offsetof(gq_wnode2_t, ref);
        parents.assign((size_t)n_wide, 0);
        if (!ref_ok(h.wroot_ref, n_wide, h.np, false, parents, true)) return "wide root";
        for (int64_t i = 0; i < n_wide; ++i) {
            const uint32_t nc = (uint32_t)i32(3, (size_t)i * s_wide + o_meta) >> 24;
            if (nc < 1 || nc > GQ_WIDTH) return "a wide node's child count";
            for (uint32_t k = 0; k < nc; ++k)
                if (!ref_ok(i32(3, (size_t)i * s_wide + o_ref + 4 * k), n_wide, h.np, false, parents, true))
                    return "a wide node references outside its arrays or a node twice";
        }
    }
    if (h.has_snch) {
        const size_t o_sref = d3 ? offsetof(gq_spair3_t, ref_l) : offsetof(gq_spair2_t, ref_l);
        parents.assign((size_t)n_spair, 0);
        if (!ref_ok(h.sroot_ref, n_spair, n_sil, true, parents)) return "SNCH root";
        for (int64_t i = 0; i < n_spair; ++i)
            for (int c = 0; c < 2; ++c)
                if (!ref_ok(i32(4, (size_t)i * s_spair + o_sref + 4 * c), n_spair, n_sil, true, parents))
                    return "an SNCH pair references outside its arrays or a node twice";
    }
    return std::string();
}

gq_status gq_scene_load(const char *path, int32_t device, gq_scene **out) {
    if (!path || !out) return fail(GQ_ERR_INVALID, "null argument");
    *out = nullptr;
    if (device < 0) return fail(GQ_ERR_INVALID, "a loaded scene lives on a device");
    File in;
    in.f = std::fopen(path, "rb");
    if (!in.f) return fail(GQ_ERR_INVALID, std::string("cannot open ") + path);
    SceneFileHeader h{};
    if (std::fread(&h, sizeof h, 1, in.f) != 1 || std::memcmp(h.magic, kSceneMagic, 8) != 0 || (h.version != kSceneFileVersion && h.version != 5) ||
        (h.dim != 2 && h.dim != 3) || h.nv < 0 || h.np < 0)
        return fail(GQ_ERR_INVALID, std::string(path) + " is not a saved scene of this version");
    std::unique_ptr<gq_scene> s(new (std::nothrow) gq_scene());
    if (!s) return fail(GQ_ERR_NOMEM, "out of host memory");
    s->dim = h.dim;
    s->device = device;
    s->nv = h.nv;
    s->np = h.np;
    s->max_prims_in_node = h.max_prims_in_node;
    s->has_snch = h.has_snch != 0;
    s->has_wide = h.has_wide != 0;
    s->exact_stack = h.exact_stack;
    s->wide_stack = h.wide_stack;
    s->max_depth = h.max_depth;
    s->n_nodes = h.n_nodes;
    s->n_wide = h.n_wide;
    s->n_sil = h.n_sil;
    s->dev.n_sils = h.n_sil;
    s->trees_ready = false;
    s->gpu_built = h.gpu_built != 0;
    try {
        s->verts.resize((size_t)(h.nv * h.dim));
        s->index.resize((size_t)(h.np * h.dim));
    } catch (const std::bad_alloc &) {
        return fail(GQ_ERR_NOMEM, "out of host memory");
    }
    bool ok = std::fread(s->verts.data(), sizeof(float), s->verts.size(), in.f) == s->verts.size() &&
              std::fread(s->index.data(), sizeof(int32_t), s->index.size(), in.f) == s->index.size();
    std::vector<char> arrays[6];
    for (int k = 0; k < 6 && ok; ++k) {
        s->image_bytes[k] = (size_t)h.image_bytes[k];
        arrays[k].resize(s->image_bytes[k]);
        ok = std::fread(arrays[k].data(), 1, arrays[k].size(), in.f) == arrays[k].size();
    }
    if (!ok) return fail(GQ_ERR_INVALID, std::string(path) + " is truncated");
    std::string bad = check_image(h, arrays);
    if (bad.empty()) {
        if (h.dim == 3)
            bad = gqb::validate_source<3>(gqb::PrimSource<3>{s->verts.data(), h.nv, s->index.data(), h.np});
        else
            bad = gqb::validate_source<2>(gqb::PrimSource<2>{s->verts.data(), h.nv, s->index.data(), h.np});
    }
    if (!bad.empty()) return fail(GQ_ERR_INVALID, std::string(path) + " is corrupt: " + bad);
    default_tuning(s.get());
    gqd::DevScene &d = s->dev;
    d.dim = h.dim;
    for (int k = 0; k < 3; ++k) d.root_lo[k] = h.root_lo[k], d.root_hi[k] = h.root_hi[k];
    DeviceGuard g(device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's CUDA device");
    const void *ptrs[6] = {};
    gq_status st;
    for (int k = 0; k < 6; ++k)
        if ((st = s->upload(arrays[k], &ptrs[k])) != GQ_OK) return st;
    d.pairs = ptrs[0];
    d.prims = ptrs[1];
    d.spheres = (const gq_tsph_t *)ptrs[2];
    d.wnodes = ptrs[3];
    d.spairs = ptrs[4];
    d.sils = ptrs[5];
    const void *pv = nullptr, *pi = nullptr, *pe = nullptr;
    if ((st = s->upload(s->verts, &pv)) != GQ_OK) return st;
    if ((st = s->upload(s->index, &pi)) != GQ_OK) return st;
    std::vector<int32_t> zero(1, 0);
    if ((st = s->upload(zero, &pe)) != GQ_OK) return st;
    d.verts = (const float *)pv;
    d.index = (const int32_t *)pi;
    d.err = (int32_t *)pe;
    d.n_prims = h.np;
    d.coord_bound = h.coord_bound;
    d.root_ref = h.root_ref;
    d.wroot_ref = h.wroot_ref;
    d.sroot_ref = h.sroot_ref;
    *out = s.release();
    return GQ_OK;
}

gq_status gq_read_probe(const void *buf, int64_t bytes, int32_t reps, uint32_t *sink, void *stream) {
    if (!buf || !sink) return fail(GQ_ERR_INVALID, "null buffer or sink");
    if (bytes <= 0 || bytes % 16 != 0 || ((uintptr_t)buf & 15u) != 0)
        return fail(GQ_ERR_INVALID, "the probe reads a 16-byte aligned buffer of a positive multiple of 16 bytes");
    if (reps < 1) return fail(GQ_ERR_INVALID, "reps must be >= 1");
    cudaError_t e = gqd::launch_read_probe(buf, bytes, reps, sink, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail_cuda(e, "read probe launch");
    return GQ_OK;
}

gq_status gq_scene_set_stack_limit(gq_scene *s, int32_t entries) {
    if (!s) return fail(GQ_ERR_INVALID, "null scene");
    if (entries < 0) return fail(GQ_ERR_INVALID, "stack limit must be >= 0");
    s->dev.stack_cap = entries > 0 ? entries : (1 << 30);
    return GQ_OK;
}

gq_status gq_scene_device_error(const gq_scene *s, void *stream, int32_t *flags) {
    if (!s || !flags) return fail(GQ_ERR_INVALID, "null argument");
    if (on_host_only(s)) return fail(GQ_ERR_UNSUPPORTED, "scene was built without a device copy");
    DeviceGuard g(s->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scene's CUDA device");
    cudaStream_t cs = (cudaStream_t)stream;
    int32_t v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, s->dev.err, sizeof v, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    if (e == cudaSuccess && v != 0) e = cudaMemsetAsync(s->dev.err, 0, sizeof v, cs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    if (e != cudaSuccess) return fail_cuda(e, "device error read");
    *flags = v;
    return GQ_OK;
}


gq_status gq_batch_create(gq_scene *const *scenes, int32_t n_scenes, int64_t max_queries, int32_t flags,
                          gq_batch **out) {
    if (!out) return fail(GQ_ERR_INVALID, "null output");
    *out = nullptr;
    if (!scenes || n_scenes <= 0) return fail(GQ_ERR_INVALID, "a batch needs at least one scene");
    if (max_queries < 0 || max_queries > (int64_t)INT32_MAX) return fail(GQ_ERR_INVALID, "max_queries out of range");
    std::unique_ptr<gq_batch> b(new (std::nothrow) gq_batch());
    if (!b) return fail(GQ_ERR_NOMEM, "host allocation");
    b->flags = flags;
    b->max_queries = max_queries;
    std::vector<gqd::DevScene> views((size_t)n_scenes);
    for (int32_t i = 0; i < n_scenes; ++i) {
        const gq_scene *s = scenes[i];
        if (!s) return fail(GQ_ERR_INVALID, "null scene in batch");
        if (on_host_only(s)) return fail(GQ_ERR_UNSUPPORTED, "scene was built without a device copy");
        if (i == 0) {
            b->dim = s->dim;
            b->device = s->device;
        } else if (s->dim != b->dim || s->device != b->device) {
            return fail(GQ_ERR_INVALID, "batch scenes must share dimension and device");
        }
        views[(size_t)i] = s->dev;
        b->scenes.push_back(scenes[i]);
    }
    DeviceGuard g(b->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cudaSetDevice failed");
    const size_t vb = views.size() * sizeof(gqd::DevScene);
    const size_t sb = gqd::batch_scratch_bytes(max_queries);
    cudaError_t e = cudaMalloc((void **)&b->dev_scenes, vb);
    if (e == cudaSuccess) e = cudaMalloc(&b->scratch, sb);
    if (e == cudaSuccess) e = cudaMalloc((void **)&b->err, 256);
    if (e != cudaSuccess) return fail(GQ_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    b->device_bytes = (int64_t)(vb + sb + 256);
    e = cudaMemcpy(b->dev_scenes, views.data(), vb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(b->err, 0, 256);
    if (e != cudaSuccess) return fail_cuda(e, "batch upload");
    *out = b.release();
    return GQ_OK;
}

gq_status gq_batch_free(gq_batch *b) {
    delete b;
    return GQ_OK;
}

int64_t gq_batch_device_bytes(const gq_batch *b) { return b ? b->device_bytes : 0; }

gq_status gq_batch_run(gq_batch *b, const gq_batch_queries *cp, const gq_cp_out *cp_out, const gq_batch_queries *ray,
                       const gq_ray_out *ray_out, const gq_batch_queries *sil, const gq_sil_out *sil_out,
                       void *stream) {
    if (!b) return fail(GQ_ERR_INVALID, "null batch");
    gqd::BatchKind kinds[3];
    const gq_batch_queries *in[3] = {cp, ray, sil};
    const bool has_out[3] = {cp_out != nullptr, ray_out != nullptr, sil_out != nullptr};
    static const char *names[3] = {"closest-point", "ray", "silhouette"};
    for (int k = 0; k < 3; ++k) {
        if (!in[k] || in[k]->n == 0) continue;
        const gq_batch_queries &q = *in[k];
        if (!has_out[k]) return fail(GQ_ERR_INVALID, std::string("null ") + names[k] + " output");
        if (q.n < 0) return fail(GQ_ERR_INVALID, "negative query count");
        if (q.n > b->max_queries)
            return fail(GQ_ERR_INVALID, std::string(names[k]) + " queries exceed the batch's max_queries (" +
                                            std::to_string(q.n) + " > " + std::to_string(b->max_queries) + ")");
        if (!q.scene || !vecs_ok(q.a) || (k == 1 && !vecs_ok(q.b)))
            return fail(GQ_ERR_INVALID, std::string("null ") + names[k] + " query array");
        kinds[k].a = q.a;
        kinds[k].b = q.b;
        kinds[k].r_max = q.r_max;
        kinds[k].scene = q.scene;
        kinds[k].n = q.n;
    }
    if (kinds[2].n > 0) {
        for (const gq_scene *s : b->scenes)
            if (!s->has_snch) return fail(GQ_ERR_UNSUPPORTED, "silhouette queries need every batch scene built with SNCH");
    }
    DeviceGuard g(b->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the batch's CUDA device");
    const gq_cp_out co = cp_out ? *cp_out : gq_cp_out{};
    const gq_ray_out ro = ray_out ? *ray_out : gq_ray_out{};
    const gq_sil_out so = sil_out ? *sil_out : gq_sil_out{};
    bool all_wide = true;
    for (const gq_scene *s : b->scenes) all_wide &= s->has_wide;
    cudaError_t e = gqd::batch_run(b->dev_scenes, (int)b->scenes.size(), b->dim, kinds, co, ro, so,
                                   (b->flags & GQ_BATCH_RAY_EXACT) || !all_wide ? 0 : 1,
                                   gqd::cp_mode_of(b->flags), gqd::sil_mode_of(b->flags),
                                   1.f, 128, true,
                                   b->scratch, b->max_queries, b->err, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail_cuda(e, "batch launch");
    return GQ_OK;
}

gq_status gq_batch_device_error(gq_batch *b, void *stream, int32_t *flags) {
    if (!b || !flags) return fail(GQ_ERR_INVALID, "null argument");
    DeviceGuard g(b->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the batch's CUDA device");
    cudaStream_t cs = (cudaStream_t)stream;
    int32_t v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, b->err, sizeof v, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    if (e == cudaSuccess && v != 0) e = cudaMemsetAsync(b->err, 0, sizeof v, cs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    if (e != cudaSuccess) return fail_cuda(e, "batch error read");
    int32_t all = v << 8;
    for (const gq_scene *s : b->scenes) {
        int32_t f = 0;
        gq_status st = gq_scene_device_error(s, stream, &f);
        if (st != GQ_OK) return st;
        all |= f;
    }
    *flags = all;
    return GQ_OK;
}

}  // extern "C"
