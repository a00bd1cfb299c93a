// Warp-coherent ("packet") closest-point traversal, shared by the single-scene kernel
// (packet.cu) and the multi-scene batch kernel (batch.cu).
//
// The lanes of a warp that hold queries on the same scene walk its tree once: every
// lane tests the same node against its own query, a child is entered when at least one
// lane's search ball reaches it, and each lane keeps its own squared radius, winner and
// per-entry stack keys (a lane skips a popped entry whose key exceeds its radius).
// Morton-adjacent queries share most of the nodes they need, so the warp runs with its
// lanes in step instead of diverging per query.
//
// Answers equal those of the binary reference traversal except at FP32 distance ties:
// box tests are conservative (squared distances, 2^-18 slack, outward-rounded quantised
// boxes), leaf tests use the reference's closest-point formulas, and the caller
// recomputes the winner's record exactly.
#pragma once

#include <cuda_fp16.h>

#include "prim.cuh"
#include "queries.cuh"

namespace gqd {
namespace pkt {

constexpr int kNone = 0x7fffffff;
// Largest sort key of a hit child of a wide node: unused and missed child slots sort as
// +inf, and a hit whose key overflowed to +inf (a query with an infinite or huge
// coordinate) is clamped so that the hits stay ahead of them in the sorted order.
constexpr float kMaxHitKey = 3.40282347e38f;
constexpr float kSlack = 1.0000038f;  // 1 + 2^-18
constexpr int kPStack = 96;

__device__ __forceinline__ float exp_scale(uint32_t meta, int ax) {
    return __int_as_float((int)((meta >> (8 * ax)) & 0xffu) << 23);
}
__device__ __forceinline__ float qf(uint32_t lo4, uint32_t hi4, int k) {
    return __int_as_float((int)__byte_perm((k < 4) ? lo4 : hi4, 0x4B000000u, 0x7540u + (unsigned)(k & 3)));
}
// minimum of a non-negative float (or +inf) over the warp
__device__ __forceinline__ float warp_min(float x) {
    return __uint_as_float(__reduce_min_sync(0xffffffffu, __float_as_uint(x)));
}
__device__ __forceinline__ void pcas(float &ka, int &ra, float &kb, int &rb) {
    const bool sw = kb < ka;
    const float k0 = sw ? kb : ka, k1 = sw ? ka : kb;
    const int r0 = sw ? rb : ra, r1 = sw ? ra : rb;
    ka = k0; kb = k1; ra = r0; rb = r1;
}
__device__ __forceinline__ void psort8(float (&k)[8], int (&r)[8]) {  // Batcher odd-even merge sort
    pcas(k[0], r[0], k[1], r[1]); pcas(k[2], r[2], k[3], r[3]); pcas(k[4], r[4], k[5], r[5]); pcas(k[6], r[6], k[7], r[7]);
    pcas(k[0], r[0], k[2], r[2]); pcas(k[1], r[1], k[3], r[3]); pcas(k[4], r[4], k[6], r[6]); pcas(k[5], r[5], k[7], r[7]);
    pcas(k[1], r[1], k[2], r[2]); pcas(k[5], r[5], k[6], r[6]);
    pcas(k[0], r[0], k[4], r[4]); pcas(k[1], r[1], k[5], r[5]); pcas(k[2], r[2], k[6], r[6]); pcas(k[3], r[3], k[7], r[7]);
    pcas(k[2], r[2], k[4], r[4]); pcas(k[3], r[3], k[5], r[5]);
    pcas(k[1], r[1], k[2], r[2]); pcas(k[3], r[3], k[4], r[4]); pcas(k[5], r[5], k[6], r[6]);
}

// The walk's stack of (node, this lane's key) entries.
// Plain: each lane keeps both words of every entry in its local memory.
// Compact: the node of each entry is kept once per warp in shared memory (every lane
// writes the same word and reads back its own write, so no lane depends on another's
// store), and the lane's key is rounded down to FP16 in its local memory: 10 bytes per
// entry and warp instead of 256.  A key rounded down admits every entry the exact key
// admits, and at worst a few more, which cost a visit and change no answer.
template <bool COMPACT>
struct PStack;
template <>
struct PStack<false> {
    int2 *e;
    __device__ __forceinline__ PStack(int2 *p) : e(p) {}
    __device__ __forceinline__ void put(int i, int ref, float key) { e[i] = make_int2(ref, fbits(key)); }
    __device__ __forceinline__ void get(int i, int &ref, float &key) const {
        const int2 x = e[i];
        ref = x.x;
        key = __int_as_float(x.y);
    }
};
template <>
struct PStack<true> {
    int *refs;     // this warp's row (shared memory)
    __half *keys;  // this lane's keys (local memory)
    __device__ __forceinline__ void put(int i, int ref, float key) {
        refs[i] = ref;
        keys[i] = __float2half_rd(key);
    }
    __device__ __forceinline__ void get(int i, int &ref, float &key) const {
        ref = refs[i];
        key = __half2float(keys[i]);
    }
};

// squared distances from p to the nearest / farthest point of a box
template <int D>
__device__ __forceinline__ void box_sq(const float *lo, const float *hi, const float *p, float &a2, float &b2) {
    a2 = 0.f;
    b2 = 0.f;
#pragma unroll
    for (int c = 0; c < D; ++c) {
        const float u = lo[c] - p[c], v = p[c] - hi[c];
        const float a = fmaxf(fmaxf(u, v), 0.f), b = fminf(u, v);
        a2 = __fmaf_rn(a, a, a2);
        b2 = __fmaf_rn(b, b, b2);
    }
}

// Leaf: every lane that needs it tests the leaf's items against its query.
template <int D>
__device__ __forceinline__ void leaf(const DevScene &s, int ref, bool act, const float *p, float &r, int &idx) {
    // a run of a collapsed subtree (bit 30 clear): first in bits 0-23, count in 24-29;
    // an ordinary leaf ~first (first < 2^30, so bit 30 set) runs to its last item
    const bool run = (ref & 0x40000000) == 0;
    int j = run ? (ref & 0xffffff) : ~ref;
    const int end = run ? j + ((ref >> 24) & 0x3f) : 0;
    if (run && end == j) return;  // an empty run (INT32_MIN, an unused wide slot): nothing to test
    for (;;) {
        bool last;
        if (D == 3) {
            const float4 t0 = ldg4(s.prims, 3 * (int64_t)j), t1 = ldg4(s.prims, 3 * (int64_t)j + 1),
                         t2 = ldg4(s.prims, 3 * (int64_t)j + 2);
            last = run ? j + 1 == end : (fbits(t2.z) & GQ_ITEM_LAST) != 0;
            if (act) {
                float pt[3], u, v;
                tri_closest<true>(p[0], p[1], p[D - 1], t0.x, t0.y, t0.z, t0.w, t1.x, t1.y, t1.z, t1.w, t2.x, pt, &u,
                                  &v);
                const float ex = p[0] - pt[0], ey = p[1] - pt[1], ez = p[D - 1] - pt[2];
                const float key = gq_dot3(ex, ey, ez, ex, ey, ez);
                if (key < r) {
                    r = key;
                    idx = j;
                }
            }
        } else {
            const float4 a = ldg4(s.prims, 2 * (int64_t)j);
            const int4 f = __ldg(reinterpret_cast<const int4 *>(s.prims) + 2 * (int64_t)j + 1);
            last = run ? j + 1 == end : (f.y & GQ_ITEM_LAST) != 0;
            if (act) {
                const float ux = a.z - a.x, uy = a.w - a.y, vx = p[0] - a.x, vy = p[D - 1] - a.y;
                const float t = gq_clamp(gq_div(gq_dot2(vx, vy, ux, uy), gq_dot2(ux, uy, ux, uy)), 0.f, 1.f);
                const float qx = gq_lerp(a.x, a.z, t) - p[0], qy = gq_lerp(a.y, a.w, t) - p[D - 1];
                const float key = gq_dot2(qx, qy, qx, qy);
                if (key < r) {
                    r = key;
                    idx = j;
                }
            }
        }
        if (last) break;
        ++j;
    }
}

// One traversal for the lanes in `mask` (warp-uniform).  All 32 lanes must call it.
// r: this lane's squared search radius (+inf to start; lanes outside `mask` are
// ignored), idx: its best item slot (-1: none).  LAYOUT 0: binary pairs,
// 1: quantised 8-wide nodes (3D only).  STK: entries of the caller's stack `stk`; the
// warp stops with `ovf` set rather than overflow it.
// COMPACT: the stack of PStack<true> (FP16 keys, one node word per warp).
template <int D, int LAYOUT, bool MINFIRST, int STK = kPStack, bool COMPACT = false>
__device__ __forceinline__ void closest_point(const DevScene &s, unsigned mask, const float *p, float &r, int &idx,
                                              bool &ovf, PStack<COMPACT> stk) {
    const unsigned lane = threadIdx.x & 31u;
    const bool mine = (mask >> lane) & 1u;
    if (!mine) r = 0.f;  // never needs a node
    int cur = LAYOUT ? s.wroot_ref : s.root_ref;
    unsigned cmask = mask;
    int sp = -1;
    for (;;) {
        if (cur == kNone) {
            bool found = false;
            while (sp >= 0) {
                int eref;
                float ekey;
                stk.get(sp--, eref, ekey);
                const unsigned m = __ballot_sync(0xffffffffu, ekey <= r * kSlack);
                if (m) {
                    cur = eref;
                    cmask = m;
                    found = true;
                    break;
                }
            }
            if (!found) break;
        }
        const bool act = (cmask >> lane) & 1u;
        if (cur < 0) {
            leaf<D>(s, cur, act, p, r, idx);
            cur = kNone;
            continue;
        }
        if (LAYOUT == 0) {
            float lo[2][D], hi[2][D];
            int rl, rr;
            if (D == 3) {
                const float4 a = ldg4(s.pairs, 4 * (int64_t)cur), b = ldg4(s.pairs, 4 * (int64_t)cur + 1),
                             c = ldg4(s.pairs, 4 * (int64_t)cur + 2);
                const int4 rf = __ldg(reinterpret_cast<const int4 *>(s.pairs) + 4 * (int64_t)cur + 3);
                lo[0][0] = a.x; lo[0][1] = a.y; lo[0][D - 1] = a.z; hi[0][0] = a.w; hi[0][1] = b.x; hi[0][D - 1] = b.y;
                lo[1][0] = b.z; lo[1][1] = b.w; lo[1][D - 1] = c.x; hi[1][0] = c.y; hi[1][1] = c.z; hi[1][D - 1] = c.w;
                // a small subtree is tested as one run (sub_l / sub_r of the pair record)
                rl = rf.z ? (int)(0x80000000u | (unsigned)rf.z) : rf.x;
                rr = rf.w ? (int)(0x80000000u | (unsigned)rf.w) : rf.y;
            } else {
                const float4 a = ldg4(s.pairs, 3 * (int64_t)cur), b = ldg4(s.pairs, 3 * (int64_t)cur + 1);
                const int4 rf = __ldg(reinterpret_cast<const int4 *>(s.pairs) + 3 * (int64_t)cur + 2);
                lo[0][0] = a.x; lo[0][D - 1] = a.y; hi[0][0] = a.z; hi[0][D - 1] = a.w;
                lo[1][0] = b.x; lo[1][D - 1] = b.y; hi[1][0] = b.z; hi[1][D - 1] = b.w;
                rl = rf.z ? (int)(0x80000000u | (unsigned)rf.z) : rf.x;
                rr = rf.w ? (int)(0x80000000u | (unsigned)rf.w) : rf.y;
            }
            float a2l = kInf, b2l = kInf, a2r = kInf, b2r = kInf;
            if (act) {
                box_sq<D>(lo[0], hi[0], p, a2l, b2l);
                box_sq<D>(lo[1], hi[1], p, a2r, b2r);
                r = fminf(r, fminf(b2l, b2r) * kSlack);
            }
            const float lim = r * kSlack;
            const bool hl = act && a2l <= lim, hr = act && a2r <= lim;
            const unsigned ml = __ballot_sync(0xffffffffu, hl), mr = __ballot_sync(0xffffffffu, hr);
            if (ml && mr) {
                const float kl = warp_min(hl ? a2l : kInf), kr = warp_min(hr ? a2r : kInf);
                const bool right_first = kr < kl;
                if (sp + 1 >= min(STK, s.stack_cap)) {
                    ovf = true;
                    break;
                }
                ++sp;
                stk.put(sp, right_first ? rl : rr, right_first ? (hl ? a2l : kInf) : (hr ? a2r : kInf));
                cur = right_first ? rr : rl;
                cmask = right_first ? mr : ml;
            } else if (ml) {
                cur = rl;
                cmask = ml;
            } else if (mr) {
                cur = rr;
                cmask = mr;
            } else {
                cur = kNone;
            }
        } else {
            const int64_t nb = 6 * (int64_t)cur;
            const float4 h = ldg4(s.wnodes, nb);
            const int4 r0 = __ldg(reinterpret_cast<const int4 *>(s.wnodes) + nb + 1);
            const int4 r1 = __ldg(reinterpret_cast<const int4 *>(s.wnodes) + nb + 2);
            const uint4 q0 = __ldg(reinterpret_cast<const uint4 *>(s.wnodes) + nb + 3);
            const uint4 q1 = __ldg(reinterpret_cast<const uint4 *>(s.wnodes) + nb + 4);
            const uint4 q2 = __ldg(reinterpret_cast<const uint4 *>(s.wnodes) + nb + 5);
            const uint32_t meta = (uint32_t)fbits(h.w);
            const int nc = (int)(meta >> 24);
            const float sx = exp_scale(meta, 0), sy = exp_scale(meta, 1), sz = exp_scale(meta, 2);
            float key[8];
            int ref[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
            float shrink = kInf;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                // NaN for inactive lanes and unused slots: it fails every `<= lim`, also while
                // lim is +inf (an unused slot holds no node)
                float a2 = __int_as_float(0x7fc00000), b2 = kInf;
                if (act && k < nc) {
                    const float lo3[3] = {__fmaf_rn(qf(q0.x, q0.y, k), sx, h.x), __fmaf_rn(qf(q0.z, q0.w, k), sy, h.y),
                                          __fmaf_rn(qf(q1.x, q1.y, k), sz, h.z)};
                    const float hi3[3] = {__fmaf_rn(qf(q1.z, q1.w, k), sx, h.x), __fmaf_rn(qf(q2.x, q2.y, k), sy, h.y),
                                          __fmaf_rn(qf(q2.z, q2.w, k), sz, h.z)};
                    box_sq<3>(lo3, hi3, p, a2, b2);
                }
                key[k] = a2;
                shrink = fminf(shrink, b2);
            }
            if (act) r = fminf(r, shrink * kSlack);
            const float lim = r * kSlack;
            float wkey[8];
            unsigned wmask[8];
            int cnt = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const bool hit = key[k] <= lim;
                key[k] = hit ? key[k] : kInf;
                wmask[k] = __ballot_sync(0xffffffffu, hit);
                // hits clamped below the others' +inf: they sort first, and the nearest-first
                // choice is a hit, so that it pushes at most cnt - 1 entries
                wkey[k] = wmask[k] ? fminf(warp_min(key[k]), kMaxHitKey) : kInf;
                cnt += wmask[k] ? 1 : 0;
            }
            if (cnt == 0) {
                cur = kNone;
                continue;
            }
            if (sp + cnt > min(STK, s.stack_cap)) {
                ovf = true;
                break;
            }
            if (MINFIRST) {
                float bk = wkey[0];
                int best = 0;
#pragma unroll
                for (int k = 1; k < 8; ++k) {
                    const bool lt = wkey[k] < bk;
                    bk = lt ? wkey[k] : bk;
                    best = lt ? k : best;
                }
                int c0 = ref[0];
                unsigned m0 = wmask[0];
#pragma unroll
                for (int k = 7; k >= 0; --k) {
                    if (k == best) {
                        c0 = ref[k];
                        m0 = wmask[k];
                    } else if (wmask[k]) {
                        stk.put(++sp, ref[k], key[k]);
                    }
                }
                cur = c0;
                cmask = m0;
                continue;
            }
            // children in the order of the nearest lane's distance; lane keys travel with the refs
            int slot[8] = {0, 1, 2, 3, 4, 5, 6, 7};
            float wk[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) wk[k] = wkey[k];
            psort8(wk, slot);
#pragma unroll
            for (int k = 7; k >= 1; --k) {
                if (k < cnt) {
                    int sref = ref[0];
                    float skey = key[0];
#pragma unroll
                    for (int m = 1; m < 8; ++m) {
                        sref = (slot[k] == m) ? ref[m] : sref;
                        skey = (slot[k] == m) ? key[m] : skey;
                    }
                    stk.put(++sp, sref, skey);
                }
            }
            int c0 = ref[0];
            unsigned m0 = wmask[0];
#pragma unroll
            for (int m = 1; m < 8; ++m) {
                c0 = (slot[0] == m) ? ref[m] : c0;
                m0 = (slot[0] == m) ? wmask[m] : m0;
            }
            cur = c0;
            cmask = m0;
        }
    }
}

}  // namespace pkt
}  // namespace gqd
