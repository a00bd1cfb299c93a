// SNCH closest-silhouette traversal (gQuery's visit order) as a resumable per-lane
// state machine, shared by the single-scene kernels (queries.cu) and the batch kernel
// (batch.cu).  SNCH.closest_silhouette (snch.py:106-164) and
// SNCH3D.closest_silhouette (snch3d.py:143-203).
//
// A step is either one interior node (both children tested against the current
// r_max, snch.py:140-141) or one silhouette of the current leaf, so a lane can stop
// after a budget of steps and resume later: persistent kernels give a finished lane a
// new query while its neighbours are still working.  Order of visits and every
// decision are the reference's; 3D silhouette edges carry their two face normals,
// computed on the host with the same FP32 operations the reference applies per test.
#pragma once

#include "../sil_filter.h"
#include "prim.cuh"
#include "queries.cuh"

namespace gqd {
namespace snch {

template <int D>
struct Lane {
    float x[D];
    float r;        // r_max, shrinks to the best silhouette distance
    float bp[D];    // best silhouette point
    float bd;
    int bid;
    int bj;         // position of the best silhouette in the leaf order (valid when found)
    int j;          // next silhouette of the current leaf, -1 when not in a leaf
    int sp;         // stack top, -1 when empty
    bool found, ovf;
};

using Stack = int2[GQ_STACK_EXACT];

template <int D>
__device__ __forceinline__ void lane_init(const DevScene &s, Lane<D> &L, const float *x, float r_max, int2 *stk) {
#pragma unroll
    for (int k = 0; k < D; ++k) {
        L.x[k] = x[k];
        L.bp[k] = 0.f;
    }
    L.r = r_max;
    L.bd = 0.f;
    L.bid = 0;
    L.j = -1;
    L.sp = -1;
    L.found = false;
    L.ovf = false;
    float dmin_root, dmax_root;
    if (D == 2)
        box_dist2(s.root_lo[0], s.root_lo[1], s.root_hi[0], s.root_hi[1], x[0], x[1], dmin_root, dmax_root);
    else
        box_dist3(s.root_lo[0], s.root_lo[1], s.root_lo[2], s.root_hi[0], s.root_hi[1], s.root_hi[2], x[0], x[1],
                  x[D - 1], dmin_root, dmax_root);
    if (dmin_root <= r_max) {
        L.sp = 0;
        stk[0] = make_int2(s.sroot_ref, fbits(dmin_root));
    }
}

// One silhouette: SilhouetteVertex.closest_silhouette (silhouette_vertex.py:40-53) /
// SilhouetteEdge.closest_silhouette (silhouette_edge.py:50-64), then the acceptance
// test of snch.py:131-134.  Returns whether it was the last of its leaf.
template <int D>
__device__ __forceinline__ bool test_silhouette(const DevScene &s, Lane<D> &L, int j) {
    bool last, ok = false;
    float p[D], d = 0.f;
    int pid;
    const float *x = L.x;
    if (D == 2) {
        const float4 r0 = ldg4(s.sils, 2 * (int64_t)j);
        const float4 r1 = ldg4(s.sils, 2 * (int64_t)j + 1);
        const int flags = fbits(r1.w);
        last = flags & GQ_ITEM_LAST;
        pid = fbits(r1.z);
        p[0] = r0.z;
        p[D - 1] = r0.w;
        // the reference tests d < r_max first; the silhouette test is independent of
        // d, so it goes first here and the square root only follows for silhouettes
        if (flags & GQ_ITEM_VALID) {
            const float c0 = (r0.z - r0.x) * (x[D - 1] - r0.y) - (r0.w - r0.y) * (x[0] - r0.x);
            const float c1 = (r1.x - r0.z) * (x[D - 1] - r0.w) - (r1.y - r0.w) * (x[0] - r0.z);
            ok = c0 * c1 < 0.f;
            if (ok) d = gq_norm2(x[0] - r0.z, x[D - 1] - r0.w);
        }
    } else {
        const float4 r0 = ldg4(s.sils, 4 * (int64_t)j), r1 = ldg4(s.sils, 4 * (int64_t)j + 1);
        const float4 r2 = ldg4(s.sils, 4 * (int64_t)j + 2), r3 = ldg4(s.sils, 4 * (int64_t)j + 3);
        const int flags = fbits(r3.y);
        last = flags & GQ_ITEM_LAST;
        pid = fbits(r3.x);
        // pre-test (sil_filter.h): skips only edges that are certainly no silhouette
        const bool skip = ((flags & (GQ_ITEM_VALID | GQ_SIL_FILTER)) == GQ_SIL_FILTER) &&
                          sil_edge_excluded(r0.x, r0.y, r0.z, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w, r3.z, r3.w, x[0],
                                            x[1], x[D - 1],
                                            sil_margin(fmaxf(fmaxf(fabsf(x[0]), fabsf(x[1])), fabsf(x[D - 1])),
                                                       s.coord_bound));
        if (!skip) {
            float qx, qy, qz;
            d = seg_dist3(x[0], x[1], x[D - 1], r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, qx, qy, qz);
            p[0] = qx;
            p[1] = qy;
            p[D - 1] = qz;
            if (d < L.r) {
                ok = flags & GQ_ITEM_VALID;  // boundary edge: always a silhouette
                if (!ok) {
                    // is_silhouette_edge (silhouette_edge.py:7-12) with the stored face normals
                    const float wx = qx - x[0], wy = qy - x[1], wz = qz - x[D - 1];
                    const float dot0 = gq_dot3(wx, wy, wz, r1.z, r1.w, r2.x);
                    const float dot1 = gq_dot3(wx, wy, wz, r2.y, r2.z, r2.w);
                    ok = dot0 * dot1 < 0.f;
                }
            }
        }
    }
    if (ok && (d < L.r)) {
        L.r = fminf(L.r, d);
        L.found = true;
#pragma unroll
        for (int k = 0; k < D; ++k) L.bp[k] = p[k];
        L.bd = d;
        L.bid = pid;
        L.bj = j;
    }
    return last;
}

constexpr int kSPair3Vec = 10;  // float4s per gq_spair3_t

// One pair record: both children's boxes and normal cones (the reference's), their
// references and, in 3D, their node bounds (sil_filter.h).
template <int D>
struct PairView {
    float lo[2][D], hi[2][D], ax[2][D], half[2], rad[2];
    int refs[2];
    float nb[2][D == 3 ? kSilNodeBound : 1];
};

template <int D>
__device__ __forceinline__ void load_pair(const DevScene &s, int ref, PairView<D> &P) {
    if (D == 2) {
        const float4 a0 = ldg4(s.spairs, 5 * (int64_t)ref), a1 = ldg4(s.spairs, 5 * (int64_t)ref + 1),
                     a2 = ldg4(s.spairs, 5 * (int64_t)ref + 2), a3 = ldg4(s.spairs, 5 * (int64_t)ref + 3);
        const int4 rr = __ldg(reinterpret_cast<const int4 *>(s.spairs) + 5 * (int64_t)ref + 4);
        P.lo[0][0] = a0.x; P.lo[0][D - 1] = a0.y; P.hi[0][0] = a0.z; P.hi[0][D - 1] = a0.w;
        P.ax[0][0] = a1.x; P.ax[0][D - 1] = a1.y; P.half[0] = a1.z; P.rad[0] = a1.w;
        P.lo[1][0] = a2.x; P.lo[1][D - 1] = a2.y; P.hi[1][0] = a2.z; P.hi[1][D - 1] = a2.w;
        P.ax[1][0] = a3.x; P.ax[1][D - 1] = a3.y; P.half[1] = a3.z; P.rad[1] = a3.w;
        P.refs[0] = rr.x;
        P.refs[1] = rr.y;
    } else {
        const int64_t b = kSPair3Vec * (int64_t)ref;
        const float4 f0 = ldg4(s.spairs, b), f1 = ldg4(s.spairs, b + 1), f2 = ldg4(s.spairs, b + 2),
                     f3 = ldg4(s.spairs, b + 3), f4 = ldg4(s.spairs, b + 4), f5 = ldg4(s.spairs, b + 5);
        const float4 f6 = ldg4(s.spairs, b + 6), f7 = ldg4(s.spairs, b + 7), f8 = ldg4(s.spairs, b + 8),
                     f9 = ldg4(s.spairs, b + 9);
        P.lo[0][0] = f0.x; P.lo[0][1] = f0.y; P.lo[0][D - 1] = f0.z;
        P.hi[0][0] = f0.w; P.hi[0][1] = f1.x; P.hi[0][D - 1] = f1.y;
        P.ax[0][0] = f1.z; P.ax[0][1] = f1.w; P.ax[0][D - 1] = f2.x;
        P.half[0] = f2.y; P.rad[0] = f2.z;
        P.lo[1][0] = f2.w; P.lo[1][1] = f3.x; P.lo[1][D - 1] = f3.y;
        P.hi[1][0] = f3.z; P.hi[1][1] = f3.w; P.hi[1][D - 1] = f4.x;
        P.ax[1][0] = f4.y; P.ax[1][1] = f4.z; P.ax[1][D - 1] = f4.w;
        P.half[1] = f5.x; P.rad[1] = f5.y;
        P.refs[0] = fbits(f5.z);
        P.refs[1] = fbits(f5.w);
        float *n0 = P.nb[0], *n1 = P.nb[D == 3 ? 1 : 0];
        if (D == 3) {
            n0[0] = f6.x; n0[1] = f6.y; n0[2] = f6.z; n0[3] = f6.w;
            n0[4] = f7.x; n0[5] = f7.y; n0[6] = f7.z; n0[7] = f7.w;
            n1[0] = f8.x; n1[1] = f8.y; n1[2] = f8.z; n1[3] = f8.w;
            n1[4] = f9.x; n1[5] = f9.y; n1[6] = f9.z; n1[7] = f9.w;
        }
    }
}

// Child c of the pair certainly holds no silhouette for x (3D node bound, sil_filter.h;
// skipping it leaves the reference's answers and the order of its other visits as
// they are).  The delta form first; with CONE the cone form where it does not decide
// (it is never wider, and skips nodes seen head-on with larger normal spreads).
// Always false in 2D.
template <int D, bool CONE = true>
__device__ __forceinline__ bool child_free(const DevScene &s, const PairView<D> &P, int c, const float *x) {
    if (D == 2) return false;
    const float *b = P.nb[D == 3 ? c : 0];
    const float m = sil_node_margin(fmaxf(fmaxf(fabsf(x[0]), fabsf(x[1])), fabsf(x[D - 1])), s.coord_bound);
    const float cx = sil_node_centre(P.lo[c][0], P.hi[c][0]), cy = sil_node_centre(P.lo[c][1], P.hi[c][1]),
                cz = sil_node_centre(P.lo[c][D - 1], P.hi[c][D - 1]);
    if (sil_node_excluded_delta(cx, cy, cz, b, x[0], x[1], x[D - 1], m)) return true;
    return CONE && sil_node_excluded_cone(cx, cy, cz, b, x[0], x[1], x[D - 1], m);
}

// Interior node `ref`: both children against the current r_max, closer pushed last.
template <int D>
__device__ __forceinline__ void visit_interior(const DevScene &s, Lane<D> &L, int2 *stk, int ref) {
    PairView<D> P;
    load_pair<D>(s, ref, P);
    bool hit[2];
    float dm[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        float dmax;
        if (D == 2)
            box_dist2(P.lo[c][0], P.lo[c][D - 1], P.hi[c][0], P.hi[c][D - 1], L.x[0], L.x[D - 1], dm[c], dmax);
        else
            box_dist3(P.lo[c][0], P.lo[c][1], P.lo[c][D - 1], P.hi[c][0], P.hi[c][1], P.hi[c][D - 1], L.x[0],
                      L.x[1], L.x[D - 1], dm[c], dmax);
        hit[c] = dm[c] <= L.r;
        // the node bound first: it rejects most of what the cone test rejects, for less
        // (both must admit a child, so the order changes no decision)
        if (hit[c]) hit[c] = !child_free<D>(s, P, c, L.x);
        if ((P.half[c] >= 0.f) & hit[c])
            hit[c] = cone_overlaps<D>(P.lo[c], P.hi[c], P.ax[c], P.half[c], P.rad[c], L.x, dm[c]);
    }
    if (hit[0] & hit[1]) {
        if (L.sp + 2 >= min(GQ_STACK_EXACT, s.stack_cap)) {
            L.ovf = true;
            L.sp = -1;
            L.j = -1;
            return;
        }
        const bool sw = dm[1] < dm[0];
        stk[++L.sp] = sw ? make_int2(P.refs[0], fbits(dm[0])) : make_int2(P.refs[1], fbits(dm[1]));
        stk[++L.sp] = sw ? make_int2(P.refs[1], fbits(dm[1])) : make_int2(P.refs[0], fbits(dm[0]));
    } else if (hit[0]) {
        stk[++L.sp] = make_int2(P.refs[0], fbits(dm[0]));
    } else if (hit[1]) {
        stk[++L.sp] = make_int2(P.refs[1], fbits(dm[1]));
    }
}

// Up to `budget` steps; true when the query is finished.
template <int D>
__device__ __forceinline__ bool lane_run(const DevScene &s, Lane<D> &L, int2 *stk, int budget) {
    for (int it = 0; it < budget; ++it) {
        if (L.j >= 0) {
            const int j = L.j;
            L.j = test_silhouette<D>(s, L, j) ? -1 : j + 1;
            continue;
        }
        if (L.sp < 0) return true;
        const int2 e = stk[L.sp--];
        if (!(__int_as_float(e.y) <= L.r)) continue;  // pop-time test (snch.py:118)
        if (e.x < 0) {
            if (e.x != INT32_MIN) L.j = ~e.x;  // INT32_MIN: leaf without silhouettes
            continue;
        }
        visit_interior<D>(s, L, stk, e.x);
    }
    return L.j < 0 && L.sp < 0;
}

// The whole query in one call.
template <int D>
__device__ __forceinline__ void closest_silhouette(const DevScene &s, const float *x, float r_max, bool &found,
                                                   float *bp, float &bd, int &bid, bool &ovf) {
    Stack stk;
    Lane<D> L;
    lane_init<D>(s, L, x, r_max, stk);
    while (!lane_run<D>(s, L, stk, 1 << 30)) {
    }
    found = L.found && !L.ovf;
    ovf = L.ovf;
#pragma unroll
    for (int k = 0; k < D; ++k) bp[k] = L.bp[k];
    bd = L.bd;
    bid = L.bid;
}

}  // namespace snch
}  // namespace gqd
