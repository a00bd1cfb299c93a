// SNCH closest-silhouette traversal (gQuery's visit order), shared by the
// single-scene kernel (queries.cu) and the batch kernel (batch.cu).
// SNCH.closest_silhouette (snch.py:106-164) and SNCH3D.closest_silhouette (snch3d.py:143-203).
#pragma once

#include "prim.cuh"
#include "queries.cuh"

namespace gqd {
namespace snch {

// One query: x (D floats), r_max.  On return `found` tells whether a silhouette was
// accepted; bp / bd / bid are its point, distance and id.  `ovf`: stack overflow.
template <int D>
__device__ __forceinline__ void closest_silhouette(const DevScene &s, const float *x, float r_max, bool &found,
                                                   float *bp, float &bd, int &bid, bool &ovf) {
    found = false;
    ovf = false;
    bd = 0.f;
    bid = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) bp[k] = 0.f;
    float dmin_root, dmax_root;
    if (D == 2)
        box_dist2(s.root_lo[0], s.root_lo[1], s.root_hi[0], s.root_hi[1], x[0], x[1], dmin_root, dmax_root);
    else
        box_dist3(s.root_lo[0], s.root_lo[1], s.root_lo[2], s.root_hi[0], s.root_hi[1], s.root_hi[2], x[0], x[1],
                  x[D - 1], dmin_root, dmax_root);
    if (dmin_root <= r_max) {
        int2 stk[GQ_STACK_EXACT];
        int sp = 0;
        stk[0] = make_int2(s.sroot_ref, fbits(dmin_root));
        while (sp >= 0) {
            const int2 e = stk[sp--];
            if (!(__int_as_float(e.y) <= r_max)) continue;
            if (e.x < 0) {
                if (e.x == INT32_MIN) continue;  // leaf without silhouettes
                int j = ~e.x;
                for (;;) {
                    bool last, ok = false;
                    float p[D], d = 0.f;
                    int pid;
                    if (D == 2) {
                        // SilhouetteVertex.closest_silhouette (silhouette_vertex.py:40-53)
                        const float4 r0 = ldg4(s.sils, 2 * (int64_t)j);
                        const float4 r1 = ldg4(s.sils, 2 * (int64_t)j + 1);
                        const int flags = fbits(r1.w);
                        last = flags & GQ_ITEM_LAST;
                        pid = fbits(r1.z);
                        p[0] = r0.z;
                        p[D - 1] = r0.w;
                        d = gq_norm2(x[0] - r0.z, x[D - 1] - r0.w);
                        if ((flags & GQ_ITEM_VALID) && (d < r_max)) {
                            const float c0 = (r0.z - r0.x) * (x[D - 1] - r0.y) - (r0.w - r0.y) * (x[0] - r0.x);
                            const float c1 = (r1.x - r0.z) * (x[D - 1] - r0.w) - (r1.y - r0.w) * (x[0] - r0.z);
                            ok = c0 * c1 < 0.f;
                        }
                    } else {
                        // SilhouetteEdge.closest_silhouette (silhouette_edge.py:50-64)
                        const float4 r0 = ldg4(s.sils, 4 * (int64_t)j), r1 = ldg4(s.sils, 4 * (int64_t)j + 1),
                                     r2 = ldg4(s.sils, 4 * (int64_t)j + 2), r3 = ldg4(s.sils, 4 * (int64_t)j + 3);
                        const int flags = fbits(r3.y);
                        last = flags & GQ_ITEM_LAST;
                        pid = fbits(r3.x);
                        const float ax = r0.x, ay = r0.y, az = r0.z, bx = r0.w, by = r1.x, bz = r1.y;
                        const float cx = r1.z, cy = r1.w, cz = r2.x, dx = r2.y, dy = r2.z, dz = r2.w;
                        float qx, qy, qz;
                        d = seg_dist3(x[0], x[1], x[D - 1], ax, ay, az, bx, by, bz, qx, qy, qz);
                        p[0] = qx;
                        p[1] = qy;
                        p[D - 1] = qz;
                        if (d < r_max) {
                            ok = flags & GQ_ITEM_VALID;
                            if (!ok) {
                                float n0x, n0y, n0z, n1x, n1y, n1z;
                                cross3(bx - ax, by - ay, bz - az, cx - ax, cy - ay, cz - az, n0x, n0y, n0z);
                                const float i0 = gq_rsqrt(gq_dot3(n0x, n0y, n0z, n0x, n0y, n0z));
                                n0x *= i0; n0y *= i0; n0z *= i0;
                                cross3(dx - ax, dy - ay, dz - az, bx - ax, by - ay, bz - az, n1x, n1y, n1z);
                                const float i1 = gq_rsqrt(gq_dot3(n1x, n1y, n1z, n1x, n1y, n1z));
                                n1x *= i1; n1y *= i1; n1z *= i1;
                                const float wx = qx - x[0], wy = qy - x[1], wz = qz - x[D - 1];
                                const float dot0 = gq_dot3(wx, wy, wz, n0x, n0y, n0z);
                                const float dot1 = gq_dot3(wx, wy, wz, n1x, n1y, n1z);
                                ok = dot0 * dot1 < 0.f;
                            }
                        }
                    }
                    if (ok && (d < r_max)) {
                        r_max = fminf(r_max, d);
                        found = true;
#pragma unroll
                        for (int k = 0; k < D; ++k) bp[k] = p[k];
                        bd = d;
                        bid = pid;
                    }
                    if (last) break;
                    ++j;
                }
                continue;
            }
            // interior: both children tested against the same r_max (snch.py:140-141)
            float lo[2][D], hi[2][D], ax[2][D], half[2], rad[2];
            int refs[2];
            if (D == 2) {
                const float4 a0 = ldg4(s.spairs, 5 * (int64_t)e.x), a1 = ldg4(s.spairs, 5 * (int64_t)e.x + 1),
                             a2 = ldg4(s.spairs, 5 * (int64_t)e.x + 2), a3 = ldg4(s.spairs, 5 * (int64_t)e.x + 3);
                const int4 rr = __ldg(reinterpret_cast<const int4 *>(s.spairs) + 5 * (int64_t)e.x + 4);
                lo[0][0] = a0.x; lo[0][D - 1] = a0.y; hi[0][0] = a0.z; hi[0][D - 1] = a0.w;
                ax[0][0] = a1.x; ax[0][D - 1] = a1.y; half[0] = a1.z; rad[0] = a1.w;
                lo[1][0] = a2.x; lo[1][D - 1] = a2.y; hi[1][0] = a2.z; hi[1][D - 1] = a2.w;
                ax[1][0] = a3.x; ax[1][D - 1] = a3.y; half[1] = a3.z; rad[1] = a3.w;
                refs[0] = rr.x;
                refs[1] = rr.y;
            } else {
                const int64_t b = 6 * (int64_t)e.x;
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
                    box_dist2(lo[c][0], lo[c][D - 1], hi[c][0], hi[c][D - 1], x[0], x[D - 1], dm[c], dmax);
                else
                    box_dist3(lo[c][0], lo[c][1], lo[c][D - 1], hi[c][0], hi[c][1], hi[c][D - 1], x[0], x[1],
                              x[D - 1], dm[c], dmax);
                hit[c] = dm[c] <= r_max;
                if ((half[c] >= 0.f) & hit[c]) hit[c] = cone_overlaps<D>(lo[c], hi[c], ax[c], half[c], rad[c], x, dm[c]);
            }
            if (hit[0] & hit[1]) {
                if (sp + 2 >= GQ_STACK_EXACT) {
                    ovf = true;
                    break;
                }
                const bool sw = dm[1] < dm[0];
                stk[++sp] = sw ? make_int2(refs[0], fbits(dm[0])) : make_int2(refs[1], fbits(dm[1]));
                stk[++sp] = sw ? make_int2(refs[1], fbits(dm[1])) : make_int2(refs[0], fbits(dm[0]));
            } else if (hit[0]) {
                stk[++sp] = make_int2(refs[0], fbits(dm[0]));
            } else if (hit[1]) {
                stk[++sp] = make_int2(refs[1], fbits(dm[1]));
            }
        }
    }
}

}  // namespace snch
}  // namespace gqd
