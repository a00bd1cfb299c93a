// One closest-silhouette query per warp ("wide frontier"), for sparse query sets whose
// per-query work is large and uneven: the 32 lanes expand up to 32 stack entries of
// the same query per step, so a query that visits 10^5 nodes takes about 10^5 / 32
// steps instead of 10^5.  Used by the single-scene kernel (queries.cu) and the server's
// silhouette steps (batch.cu).
//
// Per step: the warp takes the top `take` entries of a shared-memory stack (lane l
// gets the l-th from the top), every lane applies the reference's pop-time test
// (snch.py:118) against the warp's current r_max, then either scans its leaf's
// silhouettes with the reference's per-silhouette test and acceptance rule
// (snch.py:131-134), shrinking its own copy of r_max as it goes, or tests both
// children of its interior node with the reference's box and normal-cone tests
// (snch3d.py:55-95, snch.py:60-97).  The warp then takes the minimum r_max over its
// lanes and pushes the admitted children (lane 0's on top, the nearer child above the
// farther).  Answers equal the reference's except at FP32 distance ties, for the
// reasons given in sil_packet.cuh (the cone test does not depend on r_max; its
// trigonometry-free form cone_overlaps_fast admits every node the reference admits).
//
// Stack bound: a step that takes `take` entries pushes at most 2*take, so the warp
// takes 32 entries only while that leaves room for a depth-first descent, and one
// entry otherwise; a depth-first descent adds at most the tree depth (<= 64, checked
// on the host), so a stack of kWarpStack entries never overflows.  An overflow is
// still detected and reported instead of written.
#pragma once

#include "packet.cuh"
#include "prim.cuh"
#include "queries.cuh"
#include "snch.cuh"

namespace gqd {
namespace wsil {

constexpr int kWarpStack = 512;  // entries per warp (4 KB of shared memory)
constexpr int kReserve = 2 * GQ_STACK_EXACT + 2;

// min over the warp of a non-negative float (or +inf) and the lowest lane holding it
__device__ __forceinline__ void warp_argmin(float v, float &m, int &who) {
    m = pkt::warp_min(v);
    const unsigned hit = __ballot_sync(0xffffffffu, v == m);
    who = __ffs(hit) - 1;
}

// All 32 lanes call with the same query (x, r_max); stk: this warp's kWarpStack entries
// of shared memory.  On return every lane holds the answer in L (found, bp, bd, bid, ovf).
template <int D>
__device__ __forceinline__ void closest_silhouette(const DevScene &s, const float *x, float r_max, snch::Lane<D> &L,
                                                   int2 *stk) {
    const unsigned lane = threadIdx.x & 31u;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        L.x[k] = x[k];
        L.bp[k] = 0.f;
    }
    L.r = r_max;
    L.found = false;
    L.ovf = false;
    L.bd = 0.f;
    L.bid = 0;
    float dmin_root, dmax_root;
    if (D == 2)
        box_dist2(s.root_lo[0], s.root_lo[1], s.root_hi[0], s.root_hi[1], x[0], x[1], dmin_root, dmax_root);
    else
        box_dist3(s.root_lo[0], s.root_lo[1], s.root_lo[2], s.root_hi[0], s.root_hi[1], s.root_hi[2], x[0], x[1],
                  x[D - 1], dmin_root, dmax_root);
    int sp = 0;  // entries on the stack (warp-uniform)
    if (dmin_root <= r_max) {
        if (lane == 0) stk[0] = make_int2(s.sroot_ref, fbits(dmin_root));
        sp = 1;
    }
    __syncwarp();
    float R = r_max;  // warp's r_max
    bool ovf = false;
    while (sp > 0) {
        const int take = (sp + 32 <= kWarpStack - kReserve) ? min(sp, 32) : 1;
        const bool mine = (int)lane < take;
        int2 e = make_int2(0, 0);
        if (mine) e = stk[sp - 1 - (int)lane];
        __syncwarp();
        sp -= take;
        L.r = R;
        int2 push0 = make_int2(0, 0), push1 = make_int2(0, 0);  // the lane's entries, push1 on top
        int np = 0;
        if (mine && __int_as_float(e.y) <= R) {
            if (e.x < 0) {
                if (e.x != INT32_MIN)
                    for (int j = ~e.x;; ++j)
                        if (snch::test_silhouette<D>(s, L, j)) break;
            } else {
                // interior node: both children against this lane's r_max, nearer pushed last
                snch::PairView<D> P;
                snch::load_pair<D>(s, e.x, P);
                bool hit[2];
                float dm[2];
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    float dmax;
                    if (D == 2)
                        box_dist2(P.lo[c][0], P.lo[c][D - 1], P.hi[c][0], P.hi[c][D - 1], x[0], x[D - 1], dm[c],
                                  dmax);
                    else
                        box_dist3(P.lo[c][0], P.lo[c][1], P.lo[c][D - 1], P.hi[c][0], P.hi[c][1], P.hi[c][D - 1],
                                  x[0], x[1], x[D - 1], dm[c], dmax);
                    hit[c] = dm[c] <= L.r;
                    // the node bound first: it rejects most of what the cone test rejects, for less
                    // (both must admit a child, so the order changes no decision)
                    if (hit[c]) hit[c] = !snch::child_free<D>(s, P, c, x);
                    if ((P.half[c] >= 0.f) & hit[c])
                        hit[c] = cone_overlaps_fast<D>(P.lo[c], P.hi[c], P.ax[c], P.half[c], P.rad[c], x, dm[c]);
                }
                // push the farther first so the nearer is taken first (selects, not indexed
                // arrays, so that nothing here lives in local memory)
                const bool sw = dm[1] < dm[0];
                const bool hf = sw ? hit[0] : hit[1], hn = sw ? hit[1] : hit[0];
                const int2 ef = sw ? make_int2(P.refs[0], fbits(dm[0])) : make_int2(P.refs[1], fbits(dm[1]));
                const int2 en = sw ? make_int2(P.refs[1], fbits(dm[1])) : make_int2(P.refs[0], fbits(dm[0]));
                np = (int)hf + (int)hn;
                push0 = hf ? ef : en;
                push1 = en;
            }
        }
        // new r_max of the warp
        float m;
        int who;
        warp_argmin(L.r, m, who);
        R = m;
        // push: lane 31's entries at the bottom, lane 0's on top
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
    // answer: the lane with the smallest accepted distance (lowest lane on a tie)
    const float mine_d = L.found ? L.bd : kInf;
    float m;
    int who;
    warp_argmin(mine_d, m, who);
    const bool any = m < kInf;
    L.found = any && !ovf;
    L.ovf = ovf;
#pragma unroll
    for (int k = 0; k < D; ++k) L.bp[k] = __shfl_sync(0xffffffffu, L.bp[k], who);
    L.bd = __shfl_sync(0xffffffffu, L.bd, who);
    L.bid = __shfl_sync(0xffffffffu, L.bid, who);
}

}  // namespace wsil
}  // namespace gqd
