// Per-lane traversal state machine shared by the single-scene kernels (traverse.cu)
// and the multi-scene batch kernel (batch.cu).  See traverse.cu for the design notes.
#pragma once

#include "prim.cuh"
#include "queries.cuh"
#include "records.cuh"

namespace gqd {
namespace trav {

constexpr int kNone = 0x7fffffff;
constexpr float kSlack = 1.0000038f;  // 1 + 2^-18 (wide, squared space)
constexpr float kSq20 = 1.00000095f;  // 1 + 2^-20
constexpr float kSq21 = 1.00000048f;  // 1 + 2^-21
constexpr float kFar = 1.000000477f;  // slab widening of the wide ray test
// Largest key a hit child of a wide node carries.  Unused child slots (and missed
// children) sort as +inf; a hit whose key is +inf too (a query with an infinite or
// overflowing coordinate) is clamped here, so the sorted hits always come first and an
// unused slot, whose reference names no node, is never pushed.
constexpr float kMaxHitKey = 3.40282347e38f;

// CFG bits
constexpr int CFG_SPHERE = 1;     // triangle bounding-sphere rejection (closest point, 3D)
constexpr int CFG_SQRTSKIP = 2;   // exact: skip square roots decided by squared distances
constexpr int CFG_WW = 4;         // while-while scheduling
constexpr int CFG_MINFIRST = 8;   // wide: nearest child first, other hits unsorted
constexpr int CFG_Q16 = 16;       // wide: child bounds from the 16-bit records (s.wq16)

__device__ __forceinline__ float qget(const gq_vecs &v, int64_t i, int k) {
    return v.ptr[(int64_t)k * v.comp_stride + i * v.elem_stride];
}
__device__ __forceinline__ float exp_scale(uint32_t meta, int ax) {
    return __int_as_float((int)((meta >> (8 * ax)) & 0xffu) << 23);
}
// 2^23 + byte k of the 8-byte row (lo4, hi4), built with one byte permute.
__device__ __forceinline__ float qf(uint32_t lo4, uint32_t hi4, int k) {
    return __int_as_float((int)__byte_perm((k < 4) ? lo4 : hi4, 0x4B000000u, 0x7540u + (unsigned)(k & 3)));
}
// 2^23 + the 16-bit step k of a 16-byte row of eight steps, built with one byte permute
// (bytes 2(k&1), 2(k&1)+1 of word k/2 below the exponent byte 0x4B).
__device__ __forceinline__ float qf16(const uint4 &row, int k) {
    const uint32_t w = (k >> 1) == 0 ? row.x : (k >> 1) == 1 ? row.y : (k >> 1) == 2 ? row.z : row.w;
    return __int_as_float((int)__byte_perm(w, 0x4B000000u, (k & 1) ? 0x7432u : 0x7410u));
}
__device__ __forceinline__ void cas(float &ka, int &ra, float &kb, int &rb) {
    const bool sw = kb < ka;
    const float k0 = sw ? kb : ka, k1 = sw ? ka : kb;
    const int r0 = sw ? rb : ra, r1 = sw ? ra : rb;
    ka = k0; kb = k1; ra = r0; rb = r1;
}
__device__ __forceinline__ void sort8(float (&k)[8], int (&r)[8]) {  // Batcher odd-even merge sort
    cas(k[0], r[0], k[1], r[1]); cas(k[2], r[2], k[3], r[3]); cas(k[4], r[4], k[5], r[5]); cas(k[6], r[6], k[7], r[7]);
    cas(k[0], r[0], k[2], r[2]); cas(k[1], r[1], k[3], r[3]); cas(k[4], r[4], k[6], r[6]); cas(k[5], r[5], k[7], r[7]);
    cas(k[1], r[1], k[2], r[2]); cas(k[5], r[5], k[6], r[6]);
    cas(k[0], r[0], k[4], r[4]); cas(k[1], r[1], k[5], r[5]); cas(k[2], r[2], k[6], r[6]); cas(k[3], r[3], k[7], r[7]);
    cas(k[2], r[2], k[4], r[4]); cas(k[3], r[3], k[5], r[5]);
    cas(k[1], r[1], k[2], r[2]); cas(k[3], r[3], k[4], r[4]); cas(k[5], r[5], k[6], r[6]);
}

// ---------------------------------------------------------------------------
// Lane state
// ---------------------------------------------------------------------------

template <int D, bool RAY, bool WIDE>
struct Lane {
    float p[D], v[D], iv[D];
    float r;      // pruning radius: cp exact r_max; cp wide r_max^2; rays r_max (2D wide: best hit)
    float best;   // 2D exact rays only: best hit d_min (r_max stays fixed there)
    float eps;    // absolute rounding margin of the triangle distance (cp 3D)
    int idx;
    int cur;
    int sp;
    bool ovf;
};

template <int D, bool RAY, bool WIDE>
__device__ __forceinline__ float best_key(const Lane<D, RAY, WIDE> &L) {
    return (RAY && D == 2 && !WIDE) ? L.best : L.r;
}

// ---------------------------------------------------------------------------
// Leaves
// ---------------------------------------------------------------------------

template <int D, bool RAY, bool WIDE, int CFG>
__device__ __forceinline__ void visit_leaf(const DevScene &s, Lane<D, RAY, WIDE> &L, int ref) {
    // wide nodes: a run child (bit 30 clear, layout.h) ends after its count, an ordinary
    // leaf ~first (bit 30 set) at its last item
    const bool run = WIDE && (ref & 0x40000000) == 0;
    int j = run ? (ref & 0xffffff) : ~ref;
    const int end = run ? j + ((ref >> 24) & 0x3f) : 0;
    if (run && end == j) return;
    if constexpr (D == 3 && !RAY) {
        float rl = WIDE ? gq_sqrt(L.r) : L.r;
        for (;;) {
            bool last, test = true;
            if (CFG & CFG_SPHERE) {
                const float4 sp = __ldg(reinterpret_cast<const float4 *>(s.spheres) + j);
                last = run ? j + 1 == end : signbit(sp.w);
                const float lim = (rl + fabsf(sp.w) + L.eps) * kSq20;
                const float dx = L.p[0] - sp.x, dy = L.p[1] - sp.y, dz = L.p[D - 1] - sp.z;
                test = !(gq_dot3(dx, dy, dz, dx, dy, dz) > lim * lim * kSq20);
            }
            if (test) {
                const float4 t0 = ldg4(s.prims, 3 * (int64_t)j), t1 = ldg4(s.prims, 3 * (int64_t)j + 1),
                             t2 = ldg4(s.prims, 3 * (int64_t)j + 2);
                if (!(CFG & CFG_SPHERE)) last = run ? j + 1 == end : (fbits(t2.z) & GQ_ITEM_LAST) != 0;
                float key;
                if (WIDE) {
                    float pt[3], u, v;
                    tri_closest<true>(L.p[0], L.p[1], L.p[D - 1], t0.x, t0.y, t0.z, t0.w, t1.x, t1.y, t1.z, t1.w,
                                      t2.x, pt, &u, &v);
                    const float ex = L.p[0] - pt[0], ey = L.p[1] - pt[1], ez = L.p[D - 1] - pt[2];
                    key = gq_dot3(ex, ey, ez, ex, ey, ez);
                } else {
                    key = tri_closest<false>(L.p[0], L.p[1], L.p[D - 1], t0.x, t0.y, t0.z, t0.w, t1.x, t1.y, t1.z,
                                             t1.w, t2.x);
                }
                if (key < L.r) {
                    L.r = key;
                    L.idx = j;
                    rl = WIDE ? gq_sqrt(L.r) : L.r;
                }
            }
            if (last) break;
            ++j;
        }
        return;
    }
    for (;;) {
        bool last;
        float key;
        if (D == 3) {
            const float4 t0 = ldg4(s.prims, 3 * (int64_t)j), t1 = ldg4(s.prims, 3 * (int64_t)j + 1),
                         t2 = ldg4(s.prims, 3 * (int64_t)j + 2);
            last = run ? j + 1 == end : (fbits(t2.z) & GQ_ITEM_LAST) != 0;
            key = tri_ray(L.p[0], L.p[1], L.p[D - 1], L.v[0], L.v[1], L.v[D - 1], t0.x, t0.y, t0.z, t0.w, t1.x, t1.y,
                          t1.z, t1.w, t2.x, kInf);
        } else {
            const float4 a = ldg4(s.prims, 2 * (int64_t)j);
            const int4 f = __ldg(reinterpret_cast<const int4 *>(s.prims) + 2 * (int64_t)j + 1);
            last = run ? j + 1 == end : (f.y & GQ_ITEM_LAST) != 0;
            if (RAY) {
                key = seg_ray(L.p[0], L.p[D - 1], L.v[0], L.v[D - 1], a.x, a.y, a.z, a.w);
            } else if (WIDE) {
                const float ux = a.z - a.x, uy = a.w - a.y, vx = L.p[0] - a.x, vy = L.p[D - 1] - a.y;
                const float t = gq_clamp(gq_div(gq_dot2(vx, vy, ux, uy), gq_dot2(ux, uy, ux, uy)), 0.f, 1.f);
                const float qx = gq_lerp(a.x, a.z, t) - L.p[0], qy = gq_lerp(a.y, a.w, t) - L.p[D - 1];
                key = gq_dot2(qx, qy, qx, qy);
            } else {
                key = seg_dist(L.p[0], L.p[D - 1], a.x, a.y, a.z, a.w);
            }
        }
        if (RAY && D == 2 && !WIDE) {
            if (key < L.best) {
                L.best = key;
                L.idx = j;
            }
        } else if (key < L.r) {
            L.r = key;
            L.idx = j;
        }
        if (last) break;
        ++j;
    }
}

// ---------------------------------------------------------------------------
// Binary pair records (exact)
// ---------------------------------------------------------------------------

// BoundingBox.overlaps + the d_max shrink of one child (bvh.py:22-31, 162-167).
template <int D, int CFG>
__device__ __forceinline__ void child_cp(const float *lo, const float *hi, const float *p, float &r, bool &hit,
                                         float &dmin) {
    float ua[D], ub[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const float u = lo[k] - p[k], v = p[k] - hi[k];
        ua[k] = fmaxf(fmaxf(u, v), 0.f);
        ub[k] = fminf(u, v);
    }
    float a2, b2;
    if (D == 3) {
        a2 = gq_dot3(ua[0], ua[1], ua[D - 1], ua[0], ua[1], ua[D - 1]);
        b2 = gq_dot3(ub[0], ub[1], ub[D - 1], ub[0], ub[1], ub[D - 1]);
    } else {
        a2 = gq_dot2(ua[0], ua[D - 1], ua[0], ua[D - 1]);
        b2 = gq_dot2(ub[0], ub[D - 1], ub[0], ub[D - 1]);
    }
    if (CFG & CFG_SQRTSKIP) {
        const float rr = r * r;
        hit = false;
        dmin = kInf;
        if (a2 <= rr * kSq20) {  // otherwise sqrt(a2) rounds above r: a miss
            dmin = gq_sqrt(a2);
            hit = dmin <= r;
        }
        // otherwise sqrt(b2) >= r and r is unchanged (rr must be normal for the bound)
        if (!(rr >= 1.17549435e-38f && b2 >= rr * kSq21)) r = fminf(r, gq_sqrt(b2));
    } else {
        dmin = gq_sqrt(a2);
        hit = dmin <= r;
        r = fminf(r, gq_sqrt(b2));
    }
}

template <int D, bool RAY, int CFG>
__device__ __forceinline__ void visit_pair(const DevScene &s, Lane<D, RAY, false> &L, int2 *stk, int node) {
    float lo[2][D], hi[2][D];
    int rl, rr;
    if (D == 3) {
        const float4 a = ldg4(s.pairs, 4 * (int64_t)node), b = ldg4(s.pairs, 4 * (int64_t)node + 1),
                     c = ldg4(s.pairs, 4 * (int64_t)node + 2);
        const int4 r = __ldg(reinterpret_cast<const int4 *>(s.pairs) + 4 * (int64_t)node + 3);
        lo[0][0] = a.x; lo[0][1] = a.y; lo[0][D - 1] = a.z; hi[0][0] = a.w; hi[0][1] = b.x; hi[0][D - 1] = b.y;
        lo[1][0] = b.z; lo[1][1] = b.w; lo[1][D - 1] = c.x; hi[1][0] = c.y; hi[1][1] = c.z; hi[1][D - 1] = c.w;
        rl = r.x;
        rr = r.y;
    } else {
        const float4 a = ldg4(s.pairs, 3 * (int64_t)node), b = ldg4(s.pairs, 3 * (int64_t)node + 1);
        const int4 r = __ldg(reinterpret_cast<const int4 *>(s.pairs) + 3 * (int64_t)node + 2);
        lo[0][0] = a.x; lo[0][D - 1] = a.y; hi[0][0] = a.z; hi[0][D - 1] = a.w;
        lo[1][0] = b.x; lo[1][D - 1] = b.y; hi[1][0] = b.z; hi[1][D - 1] = b.w;
        rl = r.x;
        rr = r.y;
    }
    bool h0, h1;
    float k0, k1;
    if (!RAY) {  // left test, shrink by left d_max, right test, shrink
        child_cp<D, CFG>(lo[0], hi[0], L.p, L.r, h0, k0);
        child_cp<D, CFG>(lo[1], hi[1], L.p, L.r, h1, k1);
    } else {  // both slab tests against the same r_max (bvh.py:239-240)
        if (D == 3) {
            h0 = box_ray3(lo[0][0], lo[0][1], lo[0][D - 1], hi[0][0], hi[0][1], hi[0][D - 1], L.p[0], L.p[1],
                          L.p[D - 1], L.v[0], L.v[1], L.v[D - 1], L.r, k0);
            h1 = box_ray3(lo[1][0], lo[1][1], lo[1][D - 1], hi[1][0], hi[1][1], hi[1][D - 1], L.p[0], L.p[1],
                          L.p[D - 1], L.v[0], L.v[1], L.v[D - 1], L.r, k1);
        } else {
            h0 = box_ray2(lo[0][0], lo[0][D - 1], hi[0][0], hi[0][D - 1], L.p[0], L.p[D - 1], L.v[0], L.v[D - 1], L.r,
                          k0);
            h1 = box_ray2(lo[1][0], lo[1][D - 1], hi[1][0], hi[1][D - 1], L.p[0], L.p[D - 1], L.v[0], L.v[D - 1], L.r,
                          k1);
        }
    }
    // The reference pushes (other, closer) and pops `closer` at once under
    // dist <= r_max; here `closer` continues directly under the same test.
    if (h0 & h1) {
        if (L.sp + 1 >= min(GQ_STACK_EXACT, s.stack_cap)) {
            L.ovf = true;
            L.cur = kNone;
            L.sp = -1;
            return;
        }
        const bool sw = k1 < k0;
        stk[++L.sp] = sw ? make_int2(rl, fbits(k0)) : make_int2(rr, fbits(k1));
        const float kc = sw ? k1 : k0;
        L.cur = (kc <= L.r) ? (sw ? rr : rl) : kNone;
    } else if (h0) {
        L.cur = (k0 <= L.r) ? rl : kNone;
    } else if (h1) {
        L.cur = (k1 <= L.r) ? rr : kNone;
    } else {
        L.cur = kNone;
    }
}

// ---------------------------------------------------------------------------
// Quantised wide nodes
// ---------------------------------------------------------------------------

template <int D, bool RAY, int CFG>
__device__ __forceinline__ void visit_wide(const DevScene &s, Lane<D, RAY, true> &L, int2 *stk, int node) {
    constexpr bool Q16 = (CFG & CFG_Q16) != 0;
    constexpr int F4 = (D == 3) ? 6 : 5;           // 16-byte words per 8-bit node
    constexpr int G4 = (D == 3) ? 7 : 5;           // 16-byte words per 16-bit bounds record
    const int64_t base = F4 * (int64_t)node;
    const int64_t base16 = G4 * (int64_t)node;
    // the children's references are in the 8-bit node; the header (origin, exponents,
    // child count) and the bounds come from the 16-bit record when Q16
    const float4 h = Q16 ? ldg4(s.wq16, base16) : ldg4(s.wnodes, base);
    const int4 r0 = __ldg(reinterpret_cast<const int4 *>(s.wnodes) + base + 1);
    const int4 r1 = __ldg(reinterpret_cast<const int4 *>(s.wnodes) + base + 2);
    uint4 q0 = make_uint4(0, 0, 0, 0), q1 = q0, q2 = q0;
    uint4 w16[2 * D];  // Q16: one row of eight 16-bit steps per bound (lo_x.., hi_x..)
    if (Q16) {
#pragma unroll
        for (int rr = 0; rr < 2 * D; ++rr) w16[rr] = __ldg(reinterpret_cast<const uint4 *>(s.wq16) + base16 + 1 + rr);
    } else {
        q0 = __ldg(reinterpret_cast<const uint4 *>(s.wnodes) + base + 3);
        q1 = __ldg(reinterpret_cast<const uint4 *>(s.wnodes) + base + 4);
        if (D == 3) q2 = __ldg(reinterpret_cast<const uint4 *>(s.wnodes) + base + 5);
    }
    const uint32_t meta = (uint32_t)fbits(D == 3 ? h.w : h.z);
    const int nc = (int)(meta >> 24);
    const float sx = exp_scale(meta, 0), sy = exp_scale(meta, 1), sz = exp_scale(meta, 2);
    float key[8];
    int ref[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
    int cnt = 0;
    float shrink = kInf;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float lo[D], hi[D];
        if (Q16) {
            const float sc[3] = {sx, sy, sz}, org[3] = {h.x, h.y, D == 3 ? h.z : 0.f};
#pragma unroll
            for (int c = 0; c < D; ++c) {
                lo[c] = __fmaf_rn(qf16(w16[c], k), sc[c], org[c]);
                hi[c] = __fmaf_rn(qf16(w16[D + c], k), sc[c], org[c]);
            }
        } else if (D == 3) {
            lo[0] = __fmaf_rn(qf(q0.x, q0.y, k), sx, h.x);
            lo[1] = __fmaf_rn(qf(q0.z, q0.w, k), sy, h.y);
            lo[D - 1] = __fmaf_rn(qf(q1.x, q1.y, k), sz, h.z);
            hi[0] = __fmaf_rn(qf(q1.z, q1.w, k), sx, h.x);
            hi[1] = __fmaf_rn(qf(q2.x, q2.y, k), sy, h.y);
            hi[D - 1] = __fmaf_rn(qf(q2.z, q2.w, k), sz, h.z);
        } else {
            lo[0] = __fmaf_rn(qf(q0.x, q0.y, k), sx, h.x);
            lo[D - 1] = __fmaf_rn(qf(q0.z, q0.w, k), sy, h.y);
            hi[0] = __fmaf_rn(qf(q1.x, q1.y, k), sx, h.x);
            hi[D - 1] = __fmaf_rn(qf(q1.z, q1.w, k), sy, h.y);
        }
        if (!RAY) {
            float a2 = 0.f, b2 = 0.f;
#pragma unroll
            for (int c = 0; c < D; ++c) {
                const float u = lo[c] - L.p[c], w = L.p[c] - hi[c];
                const float ua = fmaxf(fmaxf(u, w), 0.f), ub = fminf(u, w);
                a2 = __fmaf_rn(ua, ua, a2);
                b2 = __fmaf_rn(ub, ub, b2);
            }
            key[k] = a2;
            if (k < nc) shrink = fminf(shrink, b2);
        } else {
            float tn = 0.f, tf = kInf;
#pragma unroll
            for (int c = 0; c < D; ++c) {
                const float t0 = (lo[c] - L.p[c]) * L.iv[c], t1 = (hi[c] - L.p[c]) * L.iv[c];
                tn = fmaxf(tn, fminf(t0, t1));
                tf = fminf(tf, fmaxf(t0, t1));
            }
            const bool hit = (k < nc) && (tn <= fminf(tf * kFar, L.r * kFar));
            key[k] = hit ? fminf(tn, kMaxHitKey) : kInf;
            cnt += hit ? 1 : 0;
        }
    }
    if (!RAY) {
        L.r = fminf(L.r, shrink * kSlack);
        const float lim = L.r * kSlack;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const bool hit = (k < nc) && (key[k] <= lim);
            key[k] = hit ? fminf(key[k], kMaxHitKey) : kInf;
            cnt += hit ? 1 : 0;
        }
    }
    if (cnt == 0) {
        L.cur = kNone;
        return;
    }
    if (L.sp + cnt > min(GQ_STACK_WIDE, s.stack_cap)) {
        L.ovf = true;
        L.cur = kNone;
        L.sp = -1;
        return;
    }
    if (CFG & CFG_MINFIRST) {
        // nearest hit continues; the others go on the stack in child order
        float kb = key[0];
        int best = 0;
#pragma unroll
        for (int k = 1; k < 8; ++k) {
            const bool lt = key[k] < kb;
            kb = lt ? key[k] : kb;
            best = lt ? k : best;
        }
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (k != best && key[k] < kInf) stk[++L.sp] = make_int2(ref[k], fbits(key[k]));
        int c = ref[0];
#pragma unroll
        for (int k = 1; k < 8; ++k) c = (k == best) ? ref[k] : c;
        L.cur = c;
    } else {
        sort8(key, ref);
#pragma unroll
        for (int k = 7; k >= 1; --k)
            if (k < cnt) stk[++L.sp] = make_int2(ref[k], fbits(key[k]));
        L.cur = ref[0];
    }
}

template <int D, bool RAY, bool WIDE>
__device__ __forceinline__ bool pop(Lane<D, RAY, WIDE> &L, const int2 *stk) {
    const float lim = (WIDE && !RAY) ? L.r * kSlack : L.r;
    while (L.sp >= 0) {
        const int2 e = stk[L.sp--];
        if (__int_as_float(e.y) <= lim) {
            L.cur = e.x;
            return true;
        }
    }
    return false;
}

template <int D, bool RAY, bool WIDE>
__device__ __forceinline__ void lane_init(const DevScene &s, Lane<D, RAY, WIDE> &L, const gq_vecs &a,
                                          const gq_vecs &b, const float *rmax_in, int64_t qi) {
    float pmax = 0.f;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        L.p[k] = qget(a, qi, k);
        pmax = fmaxf(pmax, fabsf(L.p[k]));
    }
    L.eps = (pmax + s.coord_bound) * 1.9073486e-06f;  // 2^-19 of the coordinate scale
    L.idx = -1;
    L.sp = -1;
    L.ovf = false;
    const int root = WIDE ? s.wroot_ref : s.root_ref;
    if (RAY) {
#pragma unroll
        for (int k = 0; k < D; ++k) {
            L.v[k] = qget(b, qi, k);
            L.iv[k] = gq_div(1.f, L.v[k]);
        }
        L.r = rmax_in ? rmax_in[qi] : kInf;
        L.best = L.r;
        float t_root;
        bool hit;
        if (D == 3)
            hit = box_ray3(s.root_lo[0], s.root_lo[1], s.root_lo[2], s.root_hi[0], s.root_hi[1], s.root_hi[2],
                           L.p[0], L.p[1], L.p[D - 1], L.v[0], L.v[1], L.v[D - 1], L.r, t_root);
        else
            hit = box_ray2(s.root_lo[0], s.root_lo[1], s.root_hi[0], s.root_hi[1], L.p[0], L.p[D - 1], L.v[0],
                           L.v[D - 1], L.r, t_root);
        // the root is pushed with t_min and popped under `t_min <= r_max`
        L.cur = (hit && t_root <= L.r) ? root : kNone;
    } else {
        L.r = kInf;
        L.best = kInf;
        L.cur = root;
    }
}

template <int D, bool RAY, bool WIDE, int CFG>
__device__ __forceinline__ void visit_inner(const DevScene &s, Lane<D, RAY, WIDE> &L, int2 *stk, int c) {
    if constexpr (WIDE)
        visit_wide<D, RAY, CFG>(s, L, stk, c);
    else
        visit_pair<D, RAY, CFG>(s, L, stk, c);
}

// Up to `budget` rounds; true when the query is finished.
template <int D, bool RAY, bool WIDE, int CFG>
__device__ __forceinline__ bool lane_run(const DevScene &s, Lane<D, RAY, WIDE> &L, int2 *stk, int budget) {
    for (int it = 0; it < budget; ++it) {
        if (L.cur == kNone && !pop(L, stk)) return true;
        if (CFG & CFG_WW) {
            // descend interior nodes until a leaf turns up (or the stack runs dry)
            while (L.cur >= 0) {
                if (L.cur == kNone) {
                    if (!pop(L, stk)) return true;
                    continue;
                }
                visit_inner<D, RAY, WIDE, CFG>(s, L, stk, L.cur);
            }
            visit_leaf<D, RAY, WIDE, CFG>(s, L, L.cur);
            L.cur = kNone;
        } else {
            const int c = L.cur;
            if (c < 0) {
                visit_leaf<D, RAY, WIDE, CFG>(s, L, c);
                L.cur = kNone;
            } else {
                visit_inner<D, RAY, WIDE, CFG>(s, L, stk, c);
            }
        }
    }
    return L.cur == kNone && L.sp < 0;
}

template <int D, bool RAY, bool WIDE>
__device__ __forceinline__ void lane_write(const DevScene &s, const Lane<D, RAY, WIDE> &L, int64_t qi, int64_t n,
                                           const gq_cp_out &oc, const gq_ray_out &orr) {
    const bool found = (L.idx >= 0) && !L.ovf;
    if (L.ovf && s.err) atomicOr(s.err, GQ_DEVERR_STACK);
    if (!RAY) {
        if (D == 3)
            cp3_record(s.prims, L.idx, found, L.p[0], L.p[1], L.p[D - 1], oc, n, qi);
        else
            cp2_record(s.prims, L.idx, found, L.p[0], L.p[D - 1], oc, n, qi);
    } else {
        const float bk = best_key(L);
        if (D == 3)
            ray3_record(s.prims, L.idx, found, L.p[0], L.p[1], L.p[D - 1], L.v[0], L.v[1], L.v[D - 1], bk, orr, n,
                        qi);
        else
            ray2_record(s.prims, L.idx, found, L.p[0], L.p[D - 1], L.v[0], L.v[D - 1], bk, orr, n, qi);
    }
}


template <bool WIDE>
using Stack = int2[WIDE ? GQ_STACK_WIDE : GQ_STACK_EXACT];

}  // namespace trav
}  // namespace gqd
