// One closest-point query per warp ("wide frontier") over the binary BVH, for the few
// queries of a sparse set whose traversal is long: the 32 lanes expand up to 32 stack
// entries of the same query per step, so a query that visits 10^4 nodes takes a few
// hundred steps instead of 10^4 dependent node loads.  The batch kernel hands such
// queries over when their per-lane traversal passes a visit budget (batch.cu).
//
// Per step every lane takes one entry from the top of this warp's shared-memory stack
// and applies the reference's tests against its copy of the warp's r_max: the pop-time
// test dist <= r_max (bvh3d.py:121-123), for an interior node the box test and d_max
// shrink of both children (BoundingBox.overlaps, bvh.py:22-31, bvh3d.py:150-160) with
// the nearer child pushed above the farther, for a leaf the primitive distances with
// the acceptance test d < r_max (bvh3d.py:140-148).  The warp then takes the minimum
// r_max over its lanes.  The answer is the smallest accepted distance over the lanes:
// the reference's answer except at FP32 distance ties, which another visit order may
// break differently.  Stack bound as in sil_warp.cuh: 32 entries are taken only while
// a depth-first descent still fits; an overflow is reported, never written.
#pragma once

#include "prim.cuh"
#include "queries.cuh"
#include "sil_warp.cuh"
#include "traverse.cuh"

namespace gqd {
namespace wcp {

constexpr int kWarpStack = wsil::kWarpStack;
constexpr int kReserve = wsil::kReserve;

// All 32 lanes call with the same query point p; stk: this warp's kWarpStack entries of
// shared memory.  r0 / idx0: a pruning radius and the primitive accepted under it (-1
// for none) from an earlier, unfinished traversal of the same query (kInf / -1 for a
// fresh start): r0 is an upper bound of the closest distance (every shrink of r_max is
// an accepted distance or a box's d_max), so the walk may start from it.  Every lane
// returns the answer: idx (-1 when none) and ovf.
template <int D>
__device__ __forceinline__ void closest_point(const DevScene &s, const float *p, float r0, int idx0, int2 *stk,
                                              int &idx, bool &ovf) {
    const unsigned lane = threadIdx.x & 31u;
    float pmax = 0.f;
#pragma unroll
    for (int k = 0; k < D; ++k) pmax = fmaxf(pmax, fabsf(p[k]));
    const float eps = (pmax + s.coord_bound) * 1.9073486e-06f;  // as the per-lane traversal (traverse.cuh)
    float r = kInf;  // this lane's r_max
    float bk = kInf;  // smallest distance this lane accepted
    int bi = -1;
    if (lane == 0 && idx0 >= 0) {  // the carried primitive, its distance recomputed
        if (D == 3) {
            const float4 t0 = ldg4(s.prims, 3 * (int64_t)idx0), t1 = ldg4(s.prims, 3 * (int64_t)idx0 + 1),
                         t2 = ldg4(s.prims, 3 * (int64_t)idx0 + 2);
            bk = tri_closest<false>(p[0], p[1], p[D - 1], t0.x, t0.y, t0.z, t0.w, t1.x, t1.y, t1.z, t1.w, t2.x);
        } else {
            const float4 a = ldg4(s.prims, 2 * (int64_t)idx0);
            bk = seg_dist(p[0], p[D - 1], a.x, a.y, a.z, a.w);
        }
        bi = idx0;
    }
    int sp = 1;
    if (lane == 0) stk[0] = make_int2(s.root_ref, fbits(0.f));
    __syncwarp();
    float R = r0;
    ovf = false;
    while (sp > 0) {
        const int take = (sp + 32 <= kWarpStack - kReserve) ? min(sp, 32) : 1;
        const bool mine = (int)lane < take;
        int2 e = make_int2(0, 0);
        if (mine) e = stk[sp - 1 - (int)lane];
        __syncwarp();
        sp -= take;
        r = R;
        int2 push0 = make_int2(0, 0), push1 = make_int2(0, 0);  // the lane's entries, push1 on top
        int np = 0;
        if (mine && __int_as_float(e.y) <= r) {
            if (e.x < 0) {
                int j = ~e.x;
                if (D == 3) {
                    // bounding-sphere rejection as the per-lane traversal (device-built
                    // scenes have no spheres)
                    const bool sph_ok = s.spheres != nullptr;
                    float rl = r;
                    for (;;) {
                        bool last = false, test = true;
                        if (sph_ok) {
                            const float4 sph = __ldg(reinterpret_cast<const float4 *>(s.spheres) + j);
                            last = signbit(sph.w);
                            const float lim = (rl + fabsf(sph.w) + eps) * trav::kSq20;
                            const float dx = p[0] - sph.x, dy = p[1] - sph.y, dz = p[D - 1] - sph.z;
                            test = !(gq_dot3(dx, dy, dz, dx, dy, dz) > lim * lim * trav::kSq20);
                        }
                        if (test) {
                            const float4 t0 = ldg4(s.prims, 3 * (int64_t)j), t1 = ldg4(s.prims, 3 * (int64_t)j + 1),
                                         t2 = ldg4(s.prims, 3 * (int64_t)j + 2);
                            if (!sph_ok) last = fbits(t2.z) & GQ_ITEM_LAST;
                            const float key = tri_closest<false>(p[0], p[1], p[D - 1], t0.x, t0.y, t0.z, t0.w, t1.x,
                                                                 t1.y, t1.z, t1.w, t2.x);
                            if (key < r) {
                                r = key;
                                rl = key;
                                if (key < bk) {
                                    bk = key;
                                    bi = j;
                                }
                            }
                        }
                        if (last) break;
                        ++j;
                    }
                } else {
                    for (;;) {
                        const float4 a = ldg4(s.prims, 2 * (int64_t)j);
                        const int4 f = __ldg(reinterpret_cast<const int4 *>(s.prims) + 2 * (int64_t)j + 1);
                        const float key = seg_dist(p[0], p[D - 1], a.x, a.y, a.z, a.w);
                        if (key < r) {
                            r = key;
                            if (key < bk) {
                                bk = key;
                                bi = j;
                            }
                        }
                        if (f.y & GQ_ITEM_LAST) break;
                        ++j;
                    }
                }
            } else {
                float lo[2][D], hi[2][D];
                int rl, rr;
                if (D == 3) {
                    const float4 a = ldg4(s.pairs, 4 * (int64_t)e.x), b = ldg4(s.pairs, 4 * (int64_t)e.x + 1),
                                 c = ldg4(s.pairs, 4 * (int64_t)e.x + 2);
                    const int4 rf = __ldg(reinterpret_cast<const int4 *>(s.pairs) + 4 * (int64_t)e.x + 3);
                    lo[0][0] = a.x; lo[0][1] = a.y; lo[0][D - 1] = a.z;
                    hi[0][0] = a.w; hi[0][1] = b.x; hi[0][D - 1] = b.y;
                    lo[1][0] = b.z; lo[1][1] = b.w; lo[1][D - 1] = c.x;
                    hi[1][0] = c.y; hi[1][1] = c.z; hi[1][D - 1] = c.w;
                    rl = rf.x;
                    rr = rf.y;
                } else {
                    const float4 a = ldg4(s.pairs, 3 * (int64_t)e.x), b = ldg4(s.pairs, 3 * (int64_t)e.x + 1);
                    const int4 rf = __ldg(reinterpret_cast<const int4 *>(s.pairs) + 3 * (int64_t)e.x + 2);
                    lo[0][0] = a.x; lo[0][D - 1] = a.y; hi[0][0] = a.z; hi[0][D - 1] = a.w;
                    lo[1][0] = b.x; lo[1][D - 1] = b.y; hi[1][0] = b.z; hi[1][D - 1] = b.w;
                    rl = rf.x;
                    rr = rf.y;
                }
                bool h0, h1;
                float k0, k1;
                trav::child_cp<D, 0>(lo[0], hi[0], p, r, h0, k0);
                trav::child_cp<D, 0>(lo[1], hi[1], p, r, h1, k1);
                h0 = h0 && k0 <= r;
                h1 = h1 && k1 <= r;
                // push the farther first so the nearer is taken first
                const bool sw = k1 < k0;
                const bool hf = sw ? h0 : h1, hn = sw ? h1 : h0;
                const int2 ef = sw ? make_int2(rl, fbits(k0)) : make_int2(rr, fbits(k1));
                const int2 en = sw ? make_int2(rr, fbits(k1)) : make_int2(rl, fbits(k0));
                np = (int)hf + (int)hn;
                push0 = hf ? ef : en;
                push1 = en;
            }
        }
        R = pkt::warp_min(r);
        const unsigned has1 = __ballot_sync(0xffffffffu, np >= 1), has2 = __ballot_sync(0xffffffffu, np >= 2);
        const unsigned above = ~((2u << lane) - 1u);  // lanes with a higher index
        const int before = __popc(has1 & above) + __popc(has2 & above);
        const int total = __popc(has1) + __popc(has2);
        if (sp + total > kWarpStack) {
            ovf = true;
            break;
        }
        if (np >= 1) stk[sp + before] = push0;
        if (np >= 2) stk[sp + before + 1] = push1;
        __syncwarp();
        sp += total;
    }
    float m;
    int who;
    wsil::warp_argmin(bk, m, who);
    idx = __shfl_sync(0xffffffffu, bi, who);
    if (!(m < kInf)) idx = -1;
}

}  // namespace wcp
}  // namespace gqd
