// ORACLE — test infrastructure only.  Nothing in the product links, imports or calls
// this file.  A C entry layer over gQuery's OWN builder sources (src/shapes/bvh.cpp,
// snch.cpp, silhouette_edge.cpp, compiled unchanged from a reference checkout by
// oracle/Makefile's `ref` target against eigen_subset/Eigen/Dense), so tests can compare
// the reference's node_data() / primitive_data() / silhouette_data() /
// raw_silhouette_data() / build_flat_silhouette_edges() (src/gquery.cpp:181-250) with
// this project's builder.
//
// The reference's recursive build calls ParallelFor above 131,072 primitives
// (bvh.cpp:281-292), which throws unless ParallelInit ran; nothing in the reference
// calls it.  Here ParallelInit(1) runs once before the first build: one thread, the
// two halves in order (left, then right).
#include <core/parallel.h>
#include <shapes/bvh.h>
#include <shapes/silhouette_edge.h>
#include <shapes/snch.h>

#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>

namespace {

std::once_flag g_init;
std::string g_err;

template <int D>
struct Built {
    std::unique_ptr<gquery::BVH<D>> bvh;   // when no SNCH was asked for
    std::unique_ptr<gquery::SNCH<D>> snch;  // holds its own BVH (its base class)
};

struct Handle {
    int dim = 0;
    Built<2> b2;
    Built<3> b3;
};

template <int D>
void inputs(const float *v, int64_t nv, const int32_t *idx, int64_t np, std::vector<::Vector<D>> &V,
            std::vector<::Vectori<D>> &I) {
    V.resize((size_t)nv);
    I.resize((size_t)np);
    for (int64_t i = 0; i < nv; ++i)
        for (int k = 0; k < D; ++k) V[(size_t)i][k] = v[i * D + k];
    for (int64_t i = 0; i < np; ++i)
        for (int k = 0; k < D; ++k) I[(size_t)i][k] = idx[i * D + k];
}

template <int D>
void build(Built<D> &b, const float *v, int64_t nv, const int32_t *idx, int64_t np, int max_prims, int snch) {
    std::vector<::Vector<D>> V;
    std::vector<::Vectori<D>> I;
    inputs<D>(v, nv, idx, np, V, I);
    if (snch)
        b.snch = std::make_unique<gquery::SNCH<D>>(V, I, max_prims);
    else
        b.bvh = std::make_unique<gquery::BVH<D>>(V, I, max_prims);
}

int64_t copy_out(const ::ArrayX &a, float *dst, int64_t cap) {
    if (dst && cap > 0) std::memcpy(dst, a.data(), sizeof(float) * (size_t)std::min<int64_t>(cap, a.size()));
    return a.size();
}

template <int D>
int64_t array_of(const Built<D> &b, int which, float *dst, int64_t cap) {
    const gquery::BVH<D> &bvh = b.snch ? static_cast<const gquery::BVH<D> &>(*b.snch) : *b.bvh;
    switch (which) {
        case 0: return copy_out(bvh.node_data(), dst, cap);
        case 1: return copy_out(bvh.primitive_data(), dst, cap);
        default: break;
    }
    if (!b.snch) return -1;
    switch (which) {
        case 2: return copy_out(b.snch->node_data(), dst, cap);
        case 3: return copy_out(b.snch->silhouette_data(), dst, cap);
        case 4: return copy_out(b.snch->raw_silhouette_data(), dst, cap);
        default: return -1;
    }
}

}  // namespace

extern "C" {

// Builds the reference's BVH<dim> (snch = 0) or SNCH<dim> (snch = 1) over vertices
// v [nv][dim] and primitives idx [np][dim]; NULL on failure (gqref_error()).
void *gqref_build(int dim, const float *v, int64_t nv, const int32_t *idx, int64_t np, int max_prims, int snch) {
    std::call_once(g_init, [] { gquery::ParallelInit(1); });
    try {
        auto h = std::make_unique<Handle>();
        h->dim = dim;
        if (dim == 2)
            build<2>(h->b2, v, nv, idx, np, max_prims, snch);
        else if (dim == 3)
            build<3>(h->b3, v, nv, idx, np, max_prims, snch);
        else
            throw std::invalid_argument("dim must be 2 or 3");
        return h.release();
    } catch (const std::exception &e) {
        g_err = e.what();
        return nullptr;
    }
}

// which: 0 node_data (BVH), 1 primitive_data, 2 node_data (SNCH), 3 silhouette_data,
// 4 raw_silhouette_data.  Copies up to cap floats; returns the full length (-1: not built).
int64_t gqref_array(void *h, int which, float *dst, int64_t cap) {
    const Handle *x = static_cast<const Handle *>(h);
    return x->dim == 2 ? array_of<2>(x->b2, which, dst, cap) : array_of<3>(x->b3, which, dst, cap);
}

void gqref_free(void *h) { delete static_cast<Handle *>(h); }

// build_flat_silhouette_edges (silhouette_edge.cpp:62-71); returns the length.
int64_t gqref_flat_silhouette_edges(const float *v, int64_t nv, const int32_t *idx, int64_t np, float *dst,
                                    int64_t cap) {
    std::vector<::Vector<3>> V;
    std::vector<::Vectori<3>> I;
    inputs<3>(v, nv, idx, np, V, I);
    return copy_out(gquery::build_flat_silhouette_edges(V, I), dst, cap);
}

const char *gqref_error(void) { return g_err.c_str(); }

}  // extern "C"
