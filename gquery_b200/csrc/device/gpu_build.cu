// Binary BVH built on the device (linear BVH): for scenes that must be admitted in
// milliseconds rather than after the host SAH build.  Primitive centroids get 30-bit
// Morton codes over the centroid bounds; (code << 32 | primitive) keys are radix-sorted;
// the hierarchy over the sorted keys follows Karras, "Maximizing parallelism in the
// construction of BVHs, octrees, and k-d trees" (HPG 2012): internal node i covers the
// key range found from the longest common prefixes around i and splits where the
// prefix changes; boxes are formed bottom-up, the second child to arrive at a node
// forming its box.  The result is written straight into the traversal's records: pair
// record i for internal node i (both child boxes and references), one primitive per
// leaf in sorted order with its end-of-leaf flag.  The tree differs from the host SAH
// tree, so queries on it give the reference's answers up to FP32 distance ties.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "gpu_build.cuh"

#include "../sil_filter.h"

namespace gqd {

namespace {

constexpr int kBlock = 256;

inline dim3 grid_of(int64_t n) { return dim3((unsigned)((n + kBlock - 1) / kBlock)); }

__device__ __forceinline__ void atomic_min_f(float *a, float v) {
    if (v >= 0.f)
        atomicMin(reinterpret_cast<int *>(a), __float_as_int(v));
    else
        atomicMax(reinterpret_cast<unsigned *>(a), __float_as_uint(v));
}
__device__ __forceinline__ void atomic_max_f(float *a, float v) {
    if (v >= 0.f)
        atomicMax(reinterpret_cast<int *>(a), __float_as_int(v));
    else
        atomicMin(reinterpret_cast<unsigned *>(a), __float_as_uint(v));
}

template <int D>
__device__ __forceinline__ void prim_box(const float *v, const int32_t *idx, int64_t p, float *lo, float *hi) {
#pragma unroll
    for (int k = 0; k < D; ++k) lo[k] = __int_as_float(0x7f800000), hi[k] = -__int_as_float(0x7f800000);
#pragma unroll
    for (int c = 0; c < D; ++c) {
        const int64_t vi = idx[p * D + c];
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const float x = v[vi * D + k];
            lo[k] = fminf(lo[k], x);
            hi[k] = fmaxf(hi[k], x);
        }
    }
}

// centroid bounds: bounds[0..D) min, bounds[3..3+D) max
template <int D>
__global__ void k_centroid_bounds(const float *v, const int32_t *idx, int64_t n, float *bounds) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    float c[D];
    if (p < n) {
        float lo[D], hi[D];
        prim_box<D>(v, idx, p, lo, hi);
#pragma unroll
        for (int k = 0; k < D; ++k) c[k] = 0.5f * (lo[k] + hi[k]);
    }
#pragma unroll
    for (int k = 0; k < D; ++k) {
        float mn = p < n ? c[k] : __int_as_float(0x7f800000), mx = p < n ? c[k] : -__int_as_float(0x7f800000);
        for (int o = 16; o > 0; o >>= 1) {
            mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
            mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomic_min_f(&bounds[k], mn);
            atomic_max_f(&bounds[3 + k], mx);
        }
    }
}

__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
__device__ __forceinline__ uint32_t spread2(uint32_t v) {
    v &= 0x7fffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

template <int D>
__global__ void k_keys(const float *v, const int32_t *idx, int64_t n, const float *bounds, uint64_t *keys,
                       int32_t *vals) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= n) return;
    float lo[D], hi[D];
    prim_box<D>(v, idx, p, lo, hi);
    uint32_t q[D];
    const float cells = D == 3 ? 1024.f : 32768.f;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const float ext = bounds[3 + k] - bounds[k];
        const float f = ext > 0.f ? (0.5f * (lo[k] + hi[k]) - bounds[k]) * (cells / ext) : 0.f;
        q[k] = (uint32_t)fminf(fmaxf(f, 0.f), cells - 1.f);
    }
    const uint32_t code = D == 3 ? ((spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[D - 1]))
                                 : ((spread2(q[0]) << 1) | spread2(q[D - 1]));
    keys[p] = ((uint64_t)code << 32) | (uint64_t)p;
    vals[p] = (int32_t)p;
}

__device__ __forceinline__ int delta(const uint64_t *k, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    return __clzll(k[i] ^ k[j]);  // keys are unique (primitive index in the low bits)
}

// Karras 2012, internal node i of n - 1; child references: internal >= 0, leaf = ~slot.
__global__ void k_hierarchy(const uint64_t *k, int64_t n, int2 *child, int32_t *parent_int, int32_t *parent_leaf,
                            int2 *range) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (delta(k, n, i, i + 1) - delta(k, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(k, n, i, i - d);
    int64_t lmax = 2;
    while (delta(k, n, i, i + lmax * d) > dmin) lmax *= 2;
    int64_t l = 0;
    for (int64_t t = lmax / 2; t >= 1; t /= 2)
        if (delta(k, n, i, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = delta(k, n, i, j);
    int64_t s = 0, t = l;
    do {
        t = (t + 1) / 2;
        if (delta(k, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int64_t gamma = i + s * d + min(d, 0);
    const int64_t lo = min(i, j), hi = max(i, j);
    const int left = lo == gamma ? ~(int)gamma : (int)gamma;
    const int right = hi == gamma + 1 ? ~(int)(gamma + 1) : (int)(gamma + 1);
    child[i] = make_int2(left, right);
    if (range) range[i] = make_int2((int)lo, (int)hi);  // the leaves below node i
    if (left < 0)
        parent_leaf[~left] = (int32_t)i;
    else
        parent_int[left] = (int32_t)i;
    if (right < 0)
        parent_leaf[~right] = (int32_t)i;
    else
        parent_int[right] = (int32_t)i;
}

template <int D>
struct NodeBox {
    float lo[D], hi[D];
};

// Leaf records in sorted order (one primitive per leaf) and their boxes.
template <int D>
__global__ void k_leaves(const float *v, const int32_t *idx, int64_t n, const int32_t *order, void *prims,
                         NodeBox<D> *leafbox) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int64_t p = order[s];
    NodeBox<D> b;
    prim_box<D>(v, idx, p, b.lo, b.hi);
    leafbox[s] = b;
    if (D == 3) {
        gq_tri_t r{};
        const int64_t a = idx[p * 3], bb = idx[p * 3 + 1], c = idx[p * 3 + 2];
        r.ax = v[a * 3]; r.ay = v[a * 3 + 1]; r.az = v[a * 3 + 2];
        r.bx = v[bb * 3]; r.by = v[bb * 3 + 1]; r.bz = v[bb * 3 + 2];
        r.cx = v[c * 3]; r.cy = v[c * 3 + 1]; r.cz = v[c * 3 + 2];
        r.index = (int32_t)(float)p;  // as the host flattening stores it
        r.flags = GQ_ITEM_LAST;
        static_cast<gq_tri_t *>(prims)[s] = r;
    } else {
        gq_seg_t r{};
        const int64_t a = idx[p * 2], bb = idx[p * 2 + 1];
        r.ax = v[a * 2]; r.ay = v[a * 2 + 1];
        r.bx = v[bb * 2]; r.by = v[bb * 2 + 1];
        r.index = (int32_t)(float)p;
        r.flags = GQ_ITEM_LAST;
        static_cast<gq_seg_t *>(prims)[s] = r;
    }
}

template <int D>
__device__ __forceinline__ NodeBox<D> box_of(int ref, const NodeBox<D> *leafbox, const NodeBox<D> *nodebox) {
    if (ref < 0) return leafbox[~ref];
    NodeBox<D> b;
    const volatile float *q = reinterpret_cast<const volatile float *>(nodebox + ref);
#pragma unroll
    for (int k = 0; k < D; ++k) b.lo[k] = q[k], b.hi[k] = q[D + k];
    return b;
}

// Bottom-up boxes: the second child to reach a node forms its box and its pair record.
template <int D>
__global__ void k_boxes(int64_t n, const int2 *child, const int32_t *parent_int, const int32_t *parent_leaf,
                        const NodeBox<D> *leafbox, NodeBox<D> *nodebox, int32_t *arrivals, void *pairs,
                        int32_t *max_depth) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    // depth of this leaf: internal ancestors up to the root
    int depth = 0;
    for (int32_t q = parent_leaf[s]; q >= 0; q = parent_int[q]) ++depth;
    atomicMax(max_depth, depth);
    int32_t node = parent_leaf[s];
    while (node >= 0) {
        __threadfence();
        if (atomicAdd(&arrivals[node], 1) == 0) return;  // the other child forms this node
        const int2 c = child[node];
        const NodeBox<D> l = box_of<D>(c.x, leafbox, nodebox), r = box_of<D>(c.y, leafbox, nodebox);
        NodeBox<D> u;
#pragma unroll
        for (int k = 0; k < D; ++k) u.lo[k] = fminf(l.lo[k], r.lo[k]), u.hi[k] = fmaxf(l.hi[k], r.hi[k]);
        volatile float *q = reinterpret_cast<volatile float *>(nodebox + node);
#pragma unroll
        for (int k = 0; k < D; ++k) q[k] = u.lo[k], q[D + k] = u.hi[k];
        if (D == 3) {
            gq_pair3_t p{};
            p.l_lox = l.lo[0]; p.l_loy = l.lo[1]; p.l_loz = l.lo[D - 1];
            p.l_hix = l.hi[0]; p.l_hiy = l.hi[1]; p.l_hiz = l.hi[D - 1];
            p.r_lox = r.lo[0]; p.r_loy = r.lo[1]; p.r_loz = r.lo[D - 1];
            p.r_hix = r.hi[0]; p.r_hiy = r.hi[1]; p.r_hiz = r.hi[D - 1];
            p.ref_l = c.x;
            p.ref_r = c.y;
            static_cast<gq_pair3_t *>(pairs)[node] = p;
        } else {
            gq_pair2_t p{};
            p.l_lox = l.lo[0]; p.l_loy = l.lo[D - 1]; p.l_hix = l.hi[0]; p.l_hiy = l.hi[D - 1];
            p.r_lox = r.lo[0]; p.r_loy = r.lo[D - 1]; p.r_hix = r.hi[0]; p.r_hiy = r.hi[D - 1];
            p.ref_l = c.x;
            p.ref_r = c.y;
            static_cast<gq_pair2_t *>(pairs)[node] = p;
        }
        node = parent_int[node];
    }
}

// ---- SNCH on the device-built tree (3D) ----
//
// Leaf s (one triangle, order[s]) lists its three edges as silhouette records 3s..3s+2
// (gq_sile_t, converted from the 19-float records exactly as the host flattening does).
// Each child of each pair gets a normal cone and a node bound over the records of its
// leaves.  The cones are built from the geometry (both face normals of every edge with
// its orientation sign, radius from the box centre to the edge end points), not with
// the reference's midpoint radius, so the walk finds what closest_silhouette_baseline
// finds up to FP32 distance ties; half angle and radius carry a small outward margin.

__device__ gq_sile_t edge_record(const float *s) {
    gq_sile_t r;
    r.ax = s[3]; r.ay = s[4]; r.az = s[5];
    r.bx = s[6]; r.by = s[7]; r.bz = s[8];
    const float cx = s[0], cy = s[1], cz = s[2], dx = s[9], dy = s[10], dz = s[11];
    sil_face_normal(r.bx - r.ax, r.by - r.ay, r.bz - r.az, cx - r.ax, cy - r.ay, cz - r.az, r.n0x, r.n0y, r.n0z);
    sil_face_normal(dx - r.ax, dy - r.ay, dz - r.az, r.bx - r.ax, r.by - r.ay, r.bz - r.az, r.n1x, r.n1y, r.n1z);
    r.prim = (int32_t)s[18];
    const bool boundary = ((int64_t)s[12] == -1) || ((int64_t)s[15] == -1);
    r.flags = boundary ? GQ_ITEM_VALID : 0;
    r.span0 = sil_span(r.n0x, r.n0y, r.n0z, r.ax, r.ay, r.az, r.bx, r.by, r.bz);
    r.span1 = sil_span(r.n1x, r.n1y, r.n1z, r.ax, r.ay, r.az, r.bx, r.by, r.bz);
    if (!boundary && sil_filter_usable(r.n0x, r.n0y, r.n0z, r.n1x, r.n1y, r.n1z, r.span0, r.span1))
        r.flags |= GQ_SIL_FILTER;
    return r;
}

__global__ void k_snch_sils(int64_t n, const int32_t *order, const uint32_t *face_edge, const float *edges19,
                            const float *edge_orient, gq_sile_t *sils, float *rec_orient) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int64_t t = order[s];
    for (int k = 0; k < 3; ++k) {
        const uint32_t e = face_edge[3 * t + k];
        gq_sile_t r = edge_record(edges19 + 19 * (int64_t)e);
        if (k == 2) r.flags |= GQ_ITEM_LAST;
        sils[3 * s + k] = r;
        rec_orient[3 * s + k] = edge_orient[e];
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float up(double x) {
    float f = (float)x;
    return (double)f < x ? nextafterf(f, __builtin_inff()) : f;
}
__device__ __forceinline__ float down(double x) {
    float f = (float)x;
    return (double)f > x ? nextafterf(f, -__builtin_inff()) : f;
}

// One warp per child of a pair (2 (n - 1) warps): cone and node bound over its records.
__global__ void k_snch_pairs(int64_t n, const int2 *child, const int2 *range, const gq_pair3_t *pairs,
                             const gq_sile_t *sils, const float *rec_orient, gq_spair3_t *spairs) {
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= 2 * (n - 1)) return;  // warp-uniform
    const int64_t p = w >> 1;
    const int c = (int)(w & 1);
    const int ref = c ? child[p].y : child[p].x;
    const gq_pair3_t &P = pairs[p];
    const float lo[3] = {c ? P.r_lox : P.l_lox, c ? P.r_loy : P.l_loy, c ? P.r_loz : P.l_loz};
    const float hi[3] = {c ? P.r_hix : P.l_hix, c ? P.r_hiy : P.l_hiy, c ? P.r_hiz : P.l_hiz};
    float ctr[3];
    for (int k = 0; k < 3; ++k) ctr[k] = sil_node_centre(lo[k], hi[k]);
    int64_t b0, b1;
    if (ref < 0) {
        b0 = 3 * (int64_t)~ref;
        b1 = b0 + 3;
    } else {
        const int2 rr = range[ref];
        b0 = 3 * (int64_t)rr.x;
        b1 = 3 * (int64_t)rr.y + 3;
    }
    // pass 1: oriented normal sum, usability
    double m[3] = {0.0, 0.0, 0.0};
    bool bad = false;
    for (int64_t j = b0 + lane; j < b1; j += 32) {
        const gq_sile_t &r = sils[j];
        const double o = rec_orient[j];
        bad |= (r.flags & (GQ_ITEM_VALID | GQ_SIL_FILTER)) != GQ_SIL_FILTER;
        m[0] += o * ((double)r.n0x + (double)r.n1x);
        m[1] += o * ((double)r.n0y + (double)r.n1y);
        m[2] += o * ((double)r.n0z + (double)r.n1z);
    }
    for (int k = 0; k < 3; ++k) m[k] = warp_sum(m[k]);
    bad = __any_sync(0xffffffffu, bad);
    const double ml = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    const bool open = bad || !(ml > 1e-30);
    float A[3] = {0.f, 0.f, 0.f};
    if (!open) {
        // axis: the mean direction, then steps toward the farthest normal (as the host's
        // sil_node_bound, in FP32 here: the axis only has to be good, the spread around it
        // is measured in double below); the axis with the smallest spread wins
        float ax[3] = {(float)(m[0] / ml), (float)(m[1] / ml), (float)(m[2] / ml)};
        double best[3] = {m[0] / ml, m[1] / ml, m[2] / ml};
        float best_c = -2.f;
        const int steps = b1 - b0 <= kSilAxisMaxRecords ? kSilAxisSteps : 0;
        for (int it = 0; it <= steps; ++it) {
            float cmin_it = 2.f, far[3] = {0.f, 0.f, 0.f};
            for (int64_t j = b0 + lane; j < b1; j += 32) {
                const gq_sile_t &r = sils[j];
                const float o = rec_orient[j];
                for (int f = 0; f < 2; ++f) {
                    const float sn[3] = {o * (f ? r.n1x : r.n0x), o * (f ? r.n1y : r.n0y), o * (f ? r.n1z : r.n0z)};
                    const float cs = sn[0] * ax[0] + sn[1] * ax[1] + sn[2] * ax[2];  // stored normals are unit
                    if (cs < cmin_it) {
                        cmin_it = cs;
                        for (int k = 0; k < 3; ++k) far[k] = sn[k];
                    }
                }
            }
            // the warp's farthest normal (lowest lane on a tie), the same on every lane
            int who = lane;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const float oc = __shfl_xor_sync(0xffffffffu, cmin_it, o);
                const int ow = __shfl_xor_sync(0xffffffffu, who, o);
                const float of0 = __shfl_xor_sync(0xffffffffu, far[0], o), of1 = __shfl_xor_sync(0xffffffffu, far[1], o),
                            of2 = __shfl_xor_sync(0xffffffffu, far[2], o);
                if (oc < cmin_it || (oc == cmin_it && ow < who)) {
                    cmin_it = oc;
                    who = ow;
                    far[0] = of0;
                    far[1] = of1;
                    far[2] = of2;
                }
            }
            if (cmin_it > best_c) {
                best_c = cmin_it;
                for (int k = 0; k < 3; ++k) best[k] = ax[k];
            }
            const float w = 1.f / (float)(it + 2);
            float nx[3], nn = 0.f;
            for (int k = 0; k < 3; ++k) {
                nx[k] = ax[k] + w * (far[k] - ax[k]);
                nn += nx[k] * nx[k];
            }
            nn = sqrtf(nn);
            if (!(nn > 1e-6f)) break;
            for (int k = 0; k < 3; ++k) ax[k] = nx[k] / nn;
        }
        for (int k = 0; k < 3; ++k) A[k] = (float)best[k];
    }
    // pass 2: spread of the oriented normals around A, plane offsets, cone, radius
    double dmax = 0.0, mlo = __builtin_inf(), mhi = -__builtin_inf(), cmin = 1.0, cnode = 1.0, rmax = 0.0;
    const double al = sqrt((double)A[0] * A[0] + (double)A[1] * A[1] + (double)A[2] * A[2]);
    for (int64_t j = b0 + lane; j < b1; j += 32) {
        const gq_sile_t &r = sils[j];
        const double o = rec_orient[j];
        const double a[3] = {r.ax, r.ay, r.az}, b[3] = {r.bx, r.by, r.bz};
        double ra = 0.0, rb = 0.0;
        for (int k = 0; k < 3; ++k) {
            ra += (a[k] - ctr[k]) * (a[k] - ctr[k]);
            rb += (b[k] - ctr[k]) * (b[k] - ctr[k]);
        }
        rmax = fmax(rmax, sqrt(fmax(ra, rb)));
        for (int f = 0; f < 2; ++f) {
            const double nn[3] = {o * (f ? r.n1x : r.n0x), o * (f ? r.n1y : r.n0y), o * (f ? r.n1z : r.n0z)};
            double d2 = 0.0, nl = 0.0, ac = 0.0, sp = 0.0, cs = 0.0;
            for (int k = 0; k < 3; ++k) {
                d2 += (nn[k] - A[k]) * (nn[k] - A[k]);
                nl += nn[k] * nn[k];
                ac += nn[k] * (a[k] - ctr[k]);
                sp += nn[k] * (b[k] - a[k]);
                cs += nn[k] * A[k];
            }
            dmax = fmax(dmax, sqrt(d2));
            mlo = fmin(mlo, ac + fmin(0.0, sp));
            mhi = fmax(mhi, ac + fmax(0.0, sp));
            cmin = fmin(cmin, cs);
            if (!open) cnode = fmin(cnode, cs / (sqrt(nl) * al));
        }
    }
    dmax = warp_max(dmax);
    cnode = warp_min(cnode);
    mlo = warp_min(mlo);
    mhi = warp_max(mhi);
    cmin = warp_min(cmin);
    rmax = warp_max(rmax);
    if (lane != 0) return;
    // cone: the largest angle to A (normals are unit up to rounding: clamp), widened
    const double half = open ? 3.14159265358979 : acos(fmax(-1.0, fmin(1.0, cmin))) + 1e-5;
    const float rad = up(rmax * (1.0 + 1e-6) + 1e-30);
    // node bound of sil_filter.h: never skipped when open (delta = +inf, lo = -inf, hi = +inf)
    float nb[kSilNodeBound] = {A[0], A[1], A[2], __builtin_inff(), 1.f, 0.f, -__builtin_inff(), __builtin_inff()};
    if (!open) {
        const double pad = 1e-12 * (fabs(mlo) + fabs(mhi) + 1.0);
        nb[3] = up(dmax * (1.0 + 1e-12));
        sil_cone_of(cnode, nb[4], nb[5]);
        nb[6] = down(mlo - pad);
        nb[7] = up(mhi + pad);
    }
    gq_spair3_t &S = spairs[p];
    const int out_ref = ref < 0 ? ~(3 * ~ref) : ref;  // leaf: its first silhouette record
    if (c == 0) {
        S.l_lox = lo[0]; S.l_loy = lo[1]; S.l_loz = lo[2];
        S.l_hix = hi[0]; S.l_hiy = hi[1]; S.l_hiz = hi[2];
        S.l_ax = A[0]; S.l_ay = A[1]; S.l_az = A[2];
        S.l_half = up(half);
        S.l_rad = rad;
        S.ref_l = out_ref;
        for (int k = 0; k < kSilNodeBound; ++k) S.l_b[k] = nb[k];
    } else {
        S.r_lox = lo[0]; S.r_loy = lo[1]; S.r_loz = lo[2];
        S.r_hix = hi[0]; S.r_hiy = hi[1]; S.r_hiz = hi[2];
        S.r_ax = A[0]; S.r_ay = A[1]; S.r_az = A[2];
        S.r_half = up(half);
        S.r_rad = rad;
        S.ref_r = out_ref;
        for (int k = 0; k < kSilNodeBound; ++k) S.r_b[k] = nb[k];
    }
}

// ---- SNCH on the device-built tree (2D) ----
//
// The raw silhouette of vertex v (snch.cpp:157-184): its own position, the previous
// vertex from the last edge that ends at v and the next vertex from the last edge that
// starts at v (zero where there is none, like the reference's value-initialised
// records).  Leaf s (segment order[s]) lists its two vertices as records 2s, 2s+1.

__global__ void k_sil_roles(const int32_t *idx, int64_t ne, int32_t *prev_e, int32_t *next_e) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= ne) return;
    atomicMax(&next_e[idx[2 * e]], (int32_t)e);
    atomicMax(&prev_e[idx[2 * e + 1]], (int32_t)e);
}

__global__ void k_snch2_sils(int64_t n, const int32_t *order, const float *v, const int32_t *idx,
                             const int32_t *prev_e, const int32_t *next_e, gq_silv_t *sils) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int64_t t = order[s];
    for (int k = 0; k < 2; ++k) {
        const int64_t u = idx[2 * t + k];
        const int32_t pe = prev_e[u], ne = next_e[u];
        gq_silv_t r;
        r.ax = pe >= 0 ? v[2 * (int64_t)idx[2 * (int64_t)pe]] : 0.f;
        r.ay = pe >= 0 ? v[2 * (int64_t)idx[2 * (int64_t)pe] + 1] : 0.f;
        r.bx = v[2 * u];
        r.by = v[2 * u + 1];
        r.cx = ne >= 0 ? v[2 * (int64_t)idx[2 * (int64_t)ne + 1]] : 0.f;
        r.cy = ne >= 0 ? v[2 * (int64_t)idx[2 * (int64_t)ne + 1] + 1] : 0.f;
        r.prim = (int32_t)(float)u;
        // silhouette_vertex.py:48: both neighbour indices != -1, which stored indices always are
        r.flags = GQ_ITEM_VALID | (k == 1 ? GQ_ITEM_LAST : 0);
        sils[2 * s + k] = r;
    }
}

// unit perpendicular of d, (d.y, -d.x) / |d| (NaN for d = 0)
__device__ __forceinline__ void perp_unit(double dx, double dy, double &nx, double &ny) {
    const double l = sqrt(dx * dx + dy * dy);
    nx = dy / l;
    ny = -dx / l;
}

// One warp per child of a pair: the cone of the vertex records below it.  The test of a
// record is sign(n0 . (b - x)) != sign(n1 . (b - x)) with n0, n1 the unit normals of its
// two segments, so a cone holding every n0, n1 and a radius reaching every b is enough.
__global__ void k_snch2_pairs(int64_t n, const int2 *child, const int2 *range, const gq_pair2_t *pairs,
                              const gq_silv_t *sils, gq_spair2_t *spairs) {
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= 2 * (n - 1)) return;  // warp-uniform
    const int64_t p = w >> 1;
    const int c = (int)(w & 1);
    const int ref = c ? child[p].y : child[p].x;
    const gq_pair2_t &P = pairs[p];
    const float lo[2] = {c ? P.r_lox : P.l_lox, c ? P.r_loy : P.l_loy};
    const float hi[2] = {c ? P.r_hix : P.l_hix, c ? P.r_hiy : P.l_hiy};
    const float ctr[2] = {0.5f * (lo[0] + hi[0]), 0.5f * (lo[1] + hi[1])};
    int64_t b0, b1;
    if (ref < 0) {
        b0 = 2 * (int64_t)~ref;
        b1 = b0 + 2;
    } else {
        const int2 rr = range[ref];
        b0 = 2 * (int64_t)rr.x;
        b1 = 2 * (int64_t)rr.y + 2;
    }
    double m[2] = {0.0, 0.0};
    bool bad = false;
    for (int64_t j = b0 + lane; j < b1; j += 32) {
        const gq_silv_t &r = sils[j];
        double n0x, n0y, n1x, n1y;
        perp_unit((double)r.bx - r.ax, (double)r.by - r.ay, n0x, n0y);
        perp_unit((double)r.cx - r.bx, (double)r.cy - r.by, n1x, n1y);
        bad |= !(isfinite(n0x) && isfinite(n0y) && isfinite(n1x) && isfinite(n1y));
        m[0] += n0x + n1x;
        m[1] += n0y + n1y;
    }
    m[0] = warp_sum(m[0]);
    m[1] = warp_sum(m[1]);
    bad = __any_sync(0xffffffffu, bad);
    const double ml = sqrt(m[0] * m[0] + m[1] * m[1]);
    const bool open = bad || !(ml > 1e-30);
    float A[2] = {0.f, 0.f};
    if (!open) A[0] = (float)(m[0] / ml), A[1] = (float)(m[1] / ml);
    double cmin = 1.0, rmax = 0.0;
    for (int64_t j = b0 + lane; j < b1; j += 32) {
        const gq_silv_t &r = sils[j];
        const double dx = (double)r.bx - ctr[0], dy = (double)r.by - ctr[1];
        rmax = fmax(rmax, sqrt(dx * dx + dy * dy));
        if (!open) {
            double n0x, n0y, n1x, n1y;
            perp_unit((double)r.bx - r.ax, (double)r.by - r.ay, n0x, n0y);
            perp_unit((double)r.cx - r.bx, (double)r.cy - r.by, n1x, n1y);
            cmin = fmin(cmin, fmin(n0x * A[0] + n0y * A[1], n1x * A[0] + n1y * A[1]));
        }
    }
    cmin = warp_min(cmin);
    rmax = warp_max(rmax);
    if (lane != 0) return;
    const double half = open ? 3.14159265358979 : acos(fmax(-1.0, fmin(1.0, cmin))) + 1e-5;
    const float rad = up(rmax * (1.0 + 1e-6) + 1e-30);
    gq_spair2_t &S = spairs[p];
    const int out_ref = ref < 0 ? ~(2 * ~ref) : ref;  // leaf: its first silhouette record
    if (c == 0) {
        S.l_lox = lo[0]; S.l_loy = lo[1]; S.l_hix = hi[0]; S.l_hiy = hi[1];
        S.l_ax = A[0]; S.l_ay = A[1]; S.l_half = up(half); S.l_rad = rad;
        S.ref_l = out_ref;
    } else {
        S.r_lox = lo[0]; S.r_loy = lo[1]; S.r_hix = hi[0]; S.r_hiy = hi[1];
        S.r_ax = A[0]; S.r_ay = A[1]; S.r_half = up(half); S.r_rad = rad;
        S.ref_r = out_ref;
        S.pad0 = S.pad1 = 0;
    }
}

template <int D>
cudaError_t build(const float *v, const int32_t *idx, int64_t n, void *pairs, void *prims, GpuBuildResult &res,
                  const GpuSnchBuild *snch, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
    std::vector<void *> tmp;
    auto grab = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (e == cudaSuccess) e = cudaMallocAsync(&p, std::max<size_t>(bytes, 256), st);
        if (e == cudaSuccess) tmp.push_back(p);
        return p;
    };
    float *bounds = (float *)grab(6 * sizeof(float));
    uint64_t *k_in = (uint64_t *)grab((size_t)n * 8), *k_out = (uint64_t *)grab((size_t)n * 8);
    int32_t *v_in = (int32_t *)grab((size_t)n * 4), *order = (int32_t *)grab((size_t)n * 4);
    int2 *child = (int2 *)grab((size_t)n * sizeof(int2));
    int32_t *parent_int = (int32_t *)grab((size_t)n * 4), *parent_leaf = (int32_t *)grab((size_t)n * 4);
    int32_t *arrivals = (int32_t *)grab((size_t)n * 4), *depth = (int32_t *)grab(4);
    NodeBox<D> *leafbox = (NodeBox<D> *)grab((size_t)n * sizeof(NodeBox<D>));
    NodeBox<D> *nodebox = (NodeBox<D> *)grab((size_t)n * sizeof(NodeBox<D>));
    const bool with_snch = snch != nullptr;
    int2 *range = with_snch ? (int2 *)grab((size_t)n * sizeof(int2)) : nullptr;
    float *rec_orient = with_snch && D == 3 ? (float *)grab((size_t)n * 3 * sizeof(float)) : nullptr;
    // 2D: per vertex the last edges ending / starting at it
    int32_t *prev_e = with_snch && D == 2 ? (int32_t *)grab((size_t)snch->n_verts * 4) : nullptr;
    int32_t *next_e = with_snch && D == 2 ? (int32_t *)grab((size_t)snch->n_verts * 4) : nullptr;
    size_t tb = 0;
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(nullptr, tb, k_in, k_out, v_in, order, (int)n, 0, 64, st);
    void *temp = grab(tb);
    if (e == cudaSuccess) {
        const float init[6] = {__builtin_inff(), __builtin_inff(), __builtin_inff(), -__builtin_inff(),
                               -__builtin_inff(), -__builtin_inff()};
        e = cudaMemcpyAsync(bounds, init, sizeof init, cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(parent_int, 0xff, (size_t)n * 4, st);  // root's parent = -1
    if (e == cudaSuccess) e = cudaMemsetAsync(arrivals, 0, (size_t)n * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(depth, 0, 4, st);
    if (e == cudaSuccess) {
        k_centroid_bounds<D><<<grid_of(n), kBlock, 0, st>>>(v, idx, n, bounds);
        k_keys<D><<<grid_of(n), kBlock, 0, st>>>(v, idx, n, bounds, k_in, v_in);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(temp, tb, k_in, k_out, v_in, order, (int)n, 0, 64, st);
    if (e == cudaSuccess) {
        if (n == 1) {
            int32_t minus1 = -1;
            e = cudaMemcpyAsync(parent_leaf, &minus1, 4, cudaMemcpyHostToDevice, st);
        } else {
            k_hierarchy<<<grid_of(n - 1), kBlock, 0, st>>>(k_out, n, child, parent_int, parent_leaf, range);
        }
    }
    if (e == cudaSuccess) {
        k_leaves<D><<<grid_of(n), kBlock, 0, st>>>(v, idx, n, order, prims, leafbox);
        k_boxes<D><<<grid_of(n), kBlock, 0, st>>>(n, child, parent_int, parent_leaf, leafbox, nodebox, arrivals, pairs,
                                                  depth);
        e = cudaGetLastError();
    }
    if (with_snch && e == cudaSuccess) {
        const int64_t threads = 2 * (n - 1) * 32;
        const dim3 pgrid((unsigned)((threads + kBlock - 1) / kBlock));
        if (D == 3) {
            k_snch_sils<<<grid_of(n), kBlock, 0, st>>>(n, order, snch->face_edge, snch->edges19, snch->edge_orient,
                                                       static_cast<gq_sile_t *>(snch->sils), rec_orient);
            if (n > 1)
                k_snch_pairs<<<pgrid, kBlock, 0, st>>>(n, child, range, static_cast<const gq_pair3_t *>(pairs),
                                                       static_cast<const gq_sile_t *>(snch->sils), rec_orient,
                                                       static_cast<gq_spair3_t *>(snch->spairs));
        } else {
            e = cudaMemsetAsync(prev_e, 0xff, (size_t)snch->n_verts * 4, st);
            if (e == cudaSuccess) e = cudaMemsetAsync(next_e, 0xff, (size_t)snch->n_verts * 4, st);
            if (e == cudaSuccess) {
                k_sil_roles<<<grid_of(n), kBlock, 0, st>>>(idx, n, prev_e, next_e);
                k_snch2_sils<<<grid_of(n), kBlock, 0, st>>>(n, order, v, idx, prev_e, next_e,
                                                            static_cast<gq_silv_t *>(snch->sils));
                if (n > 1)
                    k_snch2_pairs<<<pgrid, kBlock, 0, st>>>(n, child, range, static_cast<const gq_pair2_t *>(pairs),
                                                            static_cast<const gq_silv_t *>(snch->sils),
                                                            static_cast<gq_spair2_t *>(snch->spairs));
            }
        }
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    NodeBox<D> root{};
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&root, n == 1 ? (const void *)leafbox : (const void *)nodebox, sizeof root,
                            cudaMemcpyDeviceToHost, st);
    int32_t dmax = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&dmax, depth, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    for (void *p : tmp) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    for (int k = 0; k < 3; ++k) {
        res.root_lo[k] = k < D ? root.lo[k] : 0.f;
        res.root_hi[k] = k < D ? root.hi[k] : 0.f;
    }
    res.root_ref = n == 1 ? ~0 : 0;
    res.max_depth = dmax;
    return cudaSuccess;
}

// ---- silhouette edges on the device (build_flat_silhouette_edges) ----

__global__ void k_check_faces(const int32_t *faces, int64_t nf, int64_t nv, int32_t *bad) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < nf * 3 && (faces[i] < 0 || (int64_t)faces[i] >= nv)) atomicOr(bad, 1);
}

__global__ void k_half_edges(const int32_t *faces, int64_t nh, uint64_t *keys, uint32_t *vals) {
    const int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (h >= nh) return;
    const int64_t f = h / 3, k = h % 3;
    uint64_t i0 = (uint32_t)faces[f * 3 + k], i1 = (uint32_t)faces[f * 3 + (k + 1) % 3];
    if (i0 > i1) {
        const uint64_t t = i0;
        i0 = i1;
        i1 = t;
    }
    keys[h] = (i0 << 32) | i1;
    vals[h] = (uint32_t)h;
}

// head[i] = 1 where a run of equal keys starts
__global__ void k_heads(const uint64_t *keys, int64_t nh, uint32_t *head) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < nh) head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// per run g (its index = inclusive head scan - 1): start position and first half-edge
__global__ void k_runs(const uint32_t *head, const uint32_t *run_of, const uint32_t *vals, int64_t nh,
                       uint32_t *run_start, uint32_t *run_first, uint32_t *run_id) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nh || !head[i]) return;
    const uint32_t g = run_of[i] - 1;
    run_start[g] = (uint32_t)i;
    run_first[g] = vals[i];
    run_id[g] = g;
}

// edge e (runs ordered by first appearance): replays its half-edges in face order with
// the host's last-writer rule and writes the 19 floats of silhouette_data().
__global__ void k_edges(const float *v, const int32_t *faces, const uint64_t *keys, const uint32_t *vals, int64_t nh,
                        const uint32_t *run_start, const uint32_t *run_by_first, int64_t n_edges, float *out,
                        float *orient) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n_edges) return;
    const uint32_t g = run_by_first[e];
    int64_t i = run_start[g];
    const uint64_t key = keys[i];
    float pv[4][3] = {};
    uint64_t idx[4] = {0, 0, 0, 0}, face[2] = {0, 0};
    bool last_swapped = false;
    for (; i < nh && keys[i] == key; ++i) {
        const int64_t h = vals[i], f = h / 3, k = h % 3;
        uint64_t i0 = (uint32_t)faces[f * 3 + k], i1 = (uint32_t)faces[f * 3 + (k + 1) % 3];
        const uint64_t i2 = (uint32_t)faces[f * 3 + (k + 2) % 3];
        const uint64_t o0 = i0, o1 = i1;
        bool swapped = false;
        if (i0 > i1) {
            const uint64_t t = i0;
            i0 = i1;
            i1 = t;
            swapped = true;
        }
        const int slot = swapped ? 3 : 0;
        for (int c = 0; c < 3; ++c) {
            pv[1][c] = v[o0 * 3 + c];
            pv[2][c] = v[o1 * 3 + c];
            pv[slot][c] = v[i2 * 3 + c];
        }
        idx[1] = i0;
        idx[2] = i1;
        idx[slot] = i2;
        face[swapped ? 1 : 0] = (uint64_t)f;
        last_swapped = swapped;
    }
    // the stored end points follow the last writer's winding: its normals point
    // outward on a consistently wound mesh unless its index pair was swapped
    if (orient) orient[e] = last_swapped ? -1.f : 1.f;
    float *r = out + e * 19;
    for (int a = 0; a < 4; ++a)
        for (int c = 0; c < 3; ++c) r[a * 3 + c] = pv[a][c];
    for (int a = 0; a < 4; ++a) r[12 + a] = (float)idx[a];
    r[16] = (float)face[0];
    r[17] = (float)face[1];
    r[18] = (float)(uint64_t)e;
}

// face_edge[h] = edge index of half-edge h: runs are numbered by first appearance
__global__ void k_edge_of_run(const uint32_t *run_by_first, int64_t runs, uint32_t *edge_of_run) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e < runs) edge_of_run[run_by_first[e]] = (uint32_t)e;
}
__global__ void k_face_edge(const uint32_t *vals, const uint32_t *run_of, int64_t nh, const uint32_t *edge_of_run,
                            uint32_t *face_edge) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < nh) face_edge[vals[i]] = edge_of_run[run_of[i] - 1];
}

}  // namespace

cudaError_t gpu_build_bvh(int dim, const float *verts, const int32_t *index, int64_t n_prims, void *pairs,
                          void *prims, GpuBuildResult &res, cudaStream_t st, const GpuSnchBuild *snch) {
    if (n_prims <= 0) return cudaErrorInvalidValue;
    return dim == 3 ? build<3>(verts, index, n_prims, pairs, prims, res, snch, st)
                    : build<2>(verts, index, n_prims, pairs, prims, res, snch, st);
}

cudaError_t gpu_silhouette_edges(const float *verts, int64_t nv, const int32_t *faces, int64_t nf, float *out,
                                 int64_t cap_edges, int64_t *n_edges, int *bad_input, cudaStream_t st,
                                 uint32_t *face_edge, float *orient) {
    *n_edges = 0;
    *bad_input = 0;
    if (nf <= 0) return cudaSuccess;
    const int64_t nh = nf * 3;
    cudaError_t e = cudaSuccess;
    std::vector<void *> tmp;
    auto grab = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (e == cudaSuccess) e = cudaMallocAsync(&p, std::max<size_t>(bytes, 256), st);
        if (e == cudaSuccess) tmp.push_back(p);
        return p;
    };
    auto done = [&](cudaError_t r) {
        for (void *p : tmp) cudaFreeAsync(p, st);
        cudaStreamSynchronize(st);
        return r;
    };
    int32_t *bad = (int32_t *)grab(4);
    if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, 4, st);
    if (e == cudaSuccess) {
        k_check_faces<<<grid_of(nh), kBlock, 0, st>>>(faces, nf, nv, bad);
        e = cudaGetLastError();
    }
    int32_t hbad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return done(e);
    if (hbad) {
        *bad_input = 1;
        return done(cudaSuccess);
    }
    uint64_t *k_in = (uint64_t *)grab((size_t)nh * 8), *k_out = (uint64_t *)grab((size_t)nh * 8);
    uint32_t *v_in = (uint32_t *)grab((size_t)nh * 4), *v_out = (uint32_t *)grab((size_t)nh * 4);
    uint32_t *head = (uint32_t *)grab((size_t)nh * 4), *run_of = (uint32_t *)grab((size_t)nh * 4);
    uint32_t *run_start = (uint32_t *)grab((size_t)nh * 4), *run_first = (uint32_t *)grab((size_t)nh * 4);
    uint32_t *run_id = (uint32_t *)grab((size_t)nh * 4), *first_sorted = (uint32_t *)grab((size_t)nh * 4);
    uint32_t *run_by_first = (uint32_t *)grab((size_t)nh * 4);
    size_t tb_sort = 0, tb_scan = 0, tb_first = 0;
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(nullptr, tb_sort, k_in, k_out, v_in, v_out, (int)nh, 0, 64, st);
    if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(nullptr, tb_scan, head, run_of, (int)nh, st);
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(nullptr, tb_first, run_first, first_sorted, run_id, run_by_first, (int)nh, 0,
                                            32, st);
    void *temp = grab(std::max(tb_sort, std::max(tb_scan, tb_first)));
    if (e == cudaSuccess) {
        k_half_edges<<<grid_of(nh), kBlock, 0, st>>>(faces, nh, k_in, v_in);
        e = cudaGetLastError();
    }
    size_t tb = tb_sort;
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(temp, tb, k_in, k_out, v_in, v_out, (int)nh, 0, 64, st);
    if (e == cudaSuccess) {
        k_heads<<<grid_of(nh), kBlock, 0, st>>>(k_out, nh, head);
        e = cudaGetLastError();
    }
    tb = tb_scan;
    if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(temp, tb, head, run_of, (int)nh, st);
    uint32_t runs = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&runs, run_of + nh - 1, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return done(e);
    *n_edges = runs;
    if (!out || cap_edges < (int64_t)runs) return done(cudaSuccess);  // size query, or too small
    if (e == cudaSuccess) {
        k_runs<<<grid_of(nh), kBlock, 0, st>>>(head, run_of, v_out, nh, run_start, run_first, run_id);
        e = cudaGetLastError();
    }
    tb = tb_first;
    // runs in order of first appearance (first half-edges are distinct)
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(temp, tb, run_first, first_sorted, run_id, run_by_first, (int)runs, 0, 32,
                                            st);
    if (e == cudaSuccess) {
        k_edges<<<grid_of(runs), kBlock, 0, st>>>(verts, faces, k_out, v_out, nh, run_start, run_by_first, runs, out,
                                                  orient);
        e = cudaGetLastError();
    }
    if (face_edge && e == cudaSuccess) {
        uint32_t *edge_of_run = run_start;  // free now: k_edges has read it
        k_edge_of_run<<<grid_of(runs), kBlock, 0, st>>>(run_by_first, runs, edge_of_run);
        k_face_edge<<<grid_of(nh), kBlock, 0, st>>>(v_out, run_of, nh, edge_of_run, face_edge);
        e = cudaGetLastError();
    }
    return done(e);
}

}  // namespace gqd
