// Warp-coherent ("packet") closest-silhouette traversal of the SNCH, shared by the
// single-scene kernel (queries.cu) and the batch kernel (batch.cu).
//
// The lanes of a warp that hold queries on the same scene walk the tree once: the warp
// pops one entry, every lane whose own stack key passes its own r_max takes part,
// interior nodes are tested per lane with the reference's box test and normal-cone test
// (SNCHNode3D.overlaps, snch3d.py:55-95; snch.py:60-97) against the lane's r_max, and
// a child is entered when at least one lane admits it.  Leaves are scanned by all
// participating lanes together with the reference's per-silhouette test and acceptance
// rule (snch.py:131-134).  Each lane keeps its own r_max and best silhouette.
//
// Answers equal the reference's except at FP32 distance ties: the cone test does not
// depend on r_max, so the silhouettes a lane can reach are the same in any visit
// order, and r_max only prunes boxes that cannot hold a closer silhouette.  The order
// (nearest lane's box first) changes only which of two equally distant silhouettes
// wins.  The cone test is the trigonometry-free restatement cone_overlaps_fast, which
// admits every node the reference's test admits.
#pragma once

#include "packet.cuh"
#include "prim.cuh"
#include "queries.cuh"
#include "snch.cuh"

namespace gqd {
namespace pkt {

constexpr int kSilNone = 0x7fffffff;
// The packet form tests the node bound in its delta form only: its queries are dense
// and rarely see a node head-on, where the cone form would skip more for twice the
// arithmetic.
constexpr bool kPacketCone = false;

// One traversal for the lanes in `mask` (warp-uniform); all 32 lanes must call it.
// L: this lane's query state (x and r set by the caller, as snch::lane_init would);
// on return L.found / bp / bd / bid hold its answer and L.ovf a stack overflow.
template <int D>
__device__ __forceinline__ void closest_silhouette(const DevScene &s, unsigned mask, snch::Lane<D> &L, int2 *stk) {
    const unsigned lane = threadIdx.x & 31u;
    const bool mine = (mask >> lane) & 1u;
    L.found = false;
    L.ovf = false;
    L.bd = 0.f;
    L.bid = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) L.bp[k] = 0.f;
    float dmin_root = kInf, dmax_root;
    if (mine) {
        if (D == 2)
            box_dist2(s.root_lo[0], s.root_lo[1], s.root_hi[0], s.root_hi[1], L.x[0], L.x[1], dmin_root, dmax_root);
        else
            box_dist3(s.root_lo[0], s.root_lo[1], s.root_lo[2], s.root_hi[0], s.root_hi[1], s.root_hi[2], L.x[0],
                      L.x[1], L.x[D - 1], dmin_root, dmax_root);
    }
    unsigned cmask = __ballot_sync(0xffffffffu, mine && dmin_root <= L.r);
    int cur = cmask ? s.sroot_ref : kSilNone;
    int sp = -1;
    bool ovf = false;
    for (;;) {
        if (cur == kSilNone) {
            bool got = false;
            while (sp >= 0) {
                const int2 e = stk[sp--];
                // pop-time test of the reference, per lane (snch.py:118)
                const unsigned m = __ballot_sync(0xffffffffu, mine && __int_as_float(e.y) <= L.r);
                if (m) {
                    cur = e.x;
                    cmask = m;
                    got = true;
                    break;
                }
            }
            if (!got) break;
        }
        const bool act = (cmask >> lane) & 1u;
        if (cur < 0) {
            if (cur != INT32_MIN) {  // INT32_MIN: leaf without silhouettes
                for (int j = ~cur;; ++j) {
                    const int flags = D == 2 ? fbits(ldg4(s.sils, 2 * (int64_t)j + 1).w)
                                             : fbits(ldg4(s.sils, 4 * (int64_t)j + 3).y);
                    if (act) snch::test_silhouette<D>(s, L, j);
                    if (flags & GQ_ITEM_LAST) break;
                }
            }
            cur = kSilNone;
            continue;
        }
        snch::PairView<D> P;
        snch::load_pair<D>(s, cur, P);
        bool hit[2] = {false, false};
        float dm[2] = {kInf, kInf};
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            if (act) {
                float dmax;
                if (D == 2)
                    box_dist2(P.lo[c][0], P.lo[c][D - 1], P.hi[c][0], P.hi[c][D - 1], L.x[0], L.x[D - 1], dm[c],
                              dmax);
                else
                    box_dist3(P.lo[c][0], P.lo[c][1], P.lo[c][D - 1], P.hi[c][0], P.hi[c][1], P.hi[c][D - 1], L.x[0],
                              L.x[1], L.x[D - 1], dm[c], dmax);
                hit[c] = dm[c] <= L.r;
                // the node bound first: it rejects most of what the cone test rejects, for less
                // (both must admit a child, so the order changes no decision)
                if (hit[c]) hit[c] = !snch::child_free<D, kPacketCone>(s, P, c, L.x);
                if ((P.half[c] >= 0.f) & hit[c])
                    hit[c] = cone_overlaps_fast<D>(P.lo[c], P.hi[c], P.ax[c], P.half[c], P.rad[c], L.x, dm[c]);
            }
        }
        const unsigned m0 = __ballot_sync(0xffffffffu, hit[0]), m1 = __ballot_sync(0xffffffffu, hit[1]);
        if (m0 && m1) {
            const float k0 = warp_min(hit[0] ? dm[0] : kInf), k1 = warp_min(hit[1] ? dm[1] : kInf);
            const bool second_first = k1 < k0;  // the nearer child (over the lanes) is entered first
            if (sp + 1 >= min(GQ_STACK_EXACT, s.stack_cap)) {
                ovf = true;
                break;
            }
            stk[++sp] = second_first ? make_int2(P.refs[0], fbits(hit[0] ? dm[0] : kInf))
                                     : make_int2(P.refs[1], fbits(hit[1] ? dm[1] : kInf));
            cur = second_first ? P.refs[1] : P.refs[0];
            cmask = second_first ? m1 : m0;
        } else if (m0) {
            cur = P.refs[0];
            cmask = m0;
        } else if (m1) {
            cur = P.refs[1];
            cmask = m1;
        } else {
            cur = kSilNone;
        }
    }
    L.ovf = ovf;
}

}  // namespace pkt
}  // namespace gqd
