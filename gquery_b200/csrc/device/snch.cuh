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
    }
    return last;
}

// Interior node `ref`: both children against the current r_max, closer pushed last.
template <int D>
__device__ __forceinline__ void visit_interior(const DevScene &s, Lane<D> &L, int2 *stk, int ref) {
    float lo[2][D], hi[2][D], ax[2][D], half[2], rad[2];
    int refs[2];
    if (D == 2) {
        const float4 a0 = ldg4(s.spairs, 5 * (int64_t)ref), a1 = ldg4(s.spairs, 5 * (int64_t)ref + 1),
                     a2 = ldg4(s.spairs, 5 * (int64_t)ref + 2), a3 = ldg4(s.spairs, 5 * (int64_t)ref + 3);
        const int4 rr = __ldg(reinterpret_cast<const int4 *>(s.spairs) + 5 * (int64_t)ref + 4);
        lo[0][0] = a0.x; lo[0][D - 1] = a0.y; hi[0][0] = a0.z; hi[0][D - 1] = a0.w;
        ax[0][0] = a1.x; ax[0][D - 1] = a1.y; half[0] = a1.z; rad[0] = a1.w;
        lo[1][0] = a2.x; lo[1][D - 1] = a2.y; hi[1][0] = a2.z; hi[1][D - 1] = a2.w;
        ax[1][0] = a3.x; ax[1][D - 1] = a3.y; half[1] = a3.z; rad[1] = a3.w;
        refs[0] = rr.x;
        refs[1] = rr.y;
    } else {
        const int64_t b = 6 * (int64_t)ref;
        const float4 f0 = ldg4(s.spairs, b), f1 = ldg4(s.spairs, b + 1), f2 = ldg4(s.spairs, b + 2),
                     f3 = ldg4(s.spairs, b + 3), f4 = ldg4(s.spairs, b + 4), f5 = ldg4(s.spairs, b + 5);
        lo[0][0] = f0.x; lo[0][1] = f0.y; lo[0][D - 1] = f0.z;
        hi[0][0] = f0.w; hi[0][1] = f1.x; hi[0][D - 1] = f1.y;
        ax[0][0] = f1.z; ax[0][1] = f1.w; ax[0][D - 1] = f2.x;
        half[0] = f2.y; rad[0] = f2.z;
        lo[1][0] = f2.w; lo[1][1] = f3.x; lo[1][D - 1] = f3.y;
        hi[1][0] = f3.z; hi[1][1] = f3.w; hi[1][D - 1] = f4.x;
        ax[1][0] = f4.y; ax[1][1] = f4.z; ax[1][D - 1] = f4.w;
        half[1] = f5.x; rad[1] = f5.y;
        refs[0] = fbits(f5.z);
        refs[1] = fbits(f5.w);
    }
    bool hit[2];
    float dm[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        float dmax;
        if (D == 2)
            box_dist2(lo[c][0], lo[c][D - 1], hi[c][0], hi[c][D - 1], L.x[0], L.x[D - 1], dm[c], dmax);
        else
            box_dist3(lo[c][0], lo[c][1], lo[c][D - 1], hi[c][0], hi[c][1], hi[c][D - 1], L.x[0], L.x[1],
                      L.x[D - 1], dm[c], dmax);
        hit[c] = dm[c] <= L.r;
        if ((half[c] >= 0.f) & hit[c]) hit[c] = cone_overlaps<D>(lo[c], hi[c], ax[c], half[c], rad[c], L.x, dm[c]);
    }
    if (hit[0] & hit[1]) {
        if (L.sp + 2 >= GQ_STACK_EXACT) {
            L.ovf = true;
            L.sp = -1;
            L.j = -1;
            return;
        }
        const bool sw = dm[1] < dm[0];
        stk[++L.sp] = sw ? make_int2(refs[0], fbits(dm[0])) : make_int2(refs[1], fbits(dm[1]));
        stk[++L.sp] = sw ? make_int2(refs[1], fbits(dm[1])) : make_int2(refs[0], fbits(dm[0]));
    } else if (hit[0]) {
        stk[++L.sp] = make_int2(refs[0], fbits(dm[0]));
    } else if (hit[1]) {
        stk[++L.sp] = make_int2(refs[1], fbits(dm[1]));
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
