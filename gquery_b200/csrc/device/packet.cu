// Warp-coherent ("packet") closest-point traversal, 3D.
//
// A warp takes 32 consecutive queries of the Morton order and walks the tree once
// for all of them: every lane tests the same node against its own query, a child is
// entered when at least one lane's search ball reaches it, and each lane keeps its
// own squared radius, winner and per-entry stack keys (a lane skips a popped entry
// whose key exceeds its radius).  Nearby queries share most of the nodes they need,
// so the warp runs with all lanes in step instead of diverging per query.
//
// The answers equal those of the binary reference traversal except at FP32 distance
// ties: box tests are conservative (squared distances, 2^-18 slack, outward-rounded
// quantised boxes), leaf tests use the reference's closest-point formula, and the
// winner's record is recomputed exactly.
//
// Layouts: binary pair records (fp32 child boxes) or quantised 8-wide nodes.
#include <algorithm>
#include <cstdlib>

#include "prim.cuh"
#include "queries.cuh"
#include "records.cuh"

namespace gqd {

namespace {

constexpr int kBlock = 128;
constexpr int kNone = 0x7fffffff;
constexpr float kSlack = 1.0000038f;  // 1 + 2^-18
constexpr int kPStack = 96;

__device__ __forceinline__ float qget(const gq_vecs &v, int64_t i, int k) {
    return v.ptr[(int64_t)k * v.comp_stride + i * v.elem_stride];
}
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
__device__ __forceinline__ void cas(float &ka, int &ra, float &kb, int &rb) {
    const bool sw = kb < ka;
    const float k0 = sw ? kb : ka, k1 = sw ? ka : kb;
    const int r0 = sw ? rb : ra, r1 = sw ? ra : rb;
    ka = k0; kb = k1; ra = r0; rb = r1;
}
__device__ __forceinline__ void sort8(float (&k)[8], int (&r)[8]) {
    cas(k[0], r[0], k[1], r[1]); cas(k[2], r[2], k[3], r[3]); cas(k[4], r[4], k[5], r[5]); cas(k[6], r[6], k[7], r[7]);
    cas(k[0], r[0], k[2], r[2]); cas(k[1], r[1], k[3], r[3]); cas(k[4], r[4], k[6], r[6]); cas(k[5], r[5], k[7], r[7]);
    cas(k[1], r[1], k[2], r[2]); cas(k[5], r[5], k[6], r[6]);
    cas(k[0], r[0], k[4], r[4]); cas(k[1], r[1], k[5], r[5]); cas(k[2], r[2], k[6], r[6]); cas(k[3], r[3], k[7], r[7]);
    cas(k[2], r[2], k[4], r[4]); cas(k[3], r[3], k[5], r[5]);
    cas(k[1], r[1], k[2], r[2]); cas(k[3], r[3], k[4], r[4]); cas(k[5], r[5], k[6], r[6]);
}

__device__ __forceinline__ void box_sq(float lox, float loy, float loz, float hix, float hiy, float hiz,
                                       const float *p, float &a2, float &b2) {
    const float ux = lox - p[0], uy = loy - p[1], uz = loz - p[2];
    const float vx = p[0] - hix, vy = p[1] - hiy, vz = p[2] - hiz;
    const float ax = fmaxf(fmaxf(ux, vx), 0.f), ay = fmaxf(fmaxf(uy, vy), 0.f), az = fmaxf(fmaxf(uz, vz), 0.f);
    const float bx = fminf(ux, vx), by = fminf(uy, vy), bz = fminf(uz, vz);
    a2 = __fmaf_rn(az, az, __fmaf_rn(ay, ay, ax * ax));
    b2 = __fmaf_rn(bz, bz, __fmaf_rn(by, by, bx * bx));
}

// Leaf: every lane that needs it tests the leaf's triangles against its query.
__device__ __forceinline__ void packet_leaf(const DevScene &s, int ref, bool act, const float *p, float &r,
                                            int &idx) {
    int j = ~ref;
    for (;;) {
        const float4 t0 = ldg4(s.prims, 3 * (int64_t)j), t1 = ldg4(s.prims, 3 * (int64_t)j + 1),
                     t2 = ldg4(s.prims, 3 * (int64_t)j + 2);
        if (act) {
            float pt[3], u, v;
            tri_closest<true>(p[0], p[1], p[2], t0.x, t0.y, t0.z, t0.w, t1.x, t1.y, t1.z, t1.w, t2.x, pt, &u, &v);
            const float ex = p[0] - pt[0], ey = p[1] - pt[1], ez = p[2] - pt[2];
            const float key = gq_dot3(ex, ey, ez, ex, ey, ez);
            if (key < r) {
                r = key;
                idx = j;
            }
        }
        if (fbits(t2.z) & GQ_ITEM_LAST) break;
        ++j;
    }
}

template <int LAYOUT, bool MINFIRST>  // LAYOUT 0: binary pairs, 1: quantised 8-wide
__global__ void __launch_bounds__(kBlock) k_cp3_packet(DevScene s, gq_vecs q, int64_t n, const int32_t *perm,
                                                       gq_cp_out o, unsigned long long *counter) {
    const unsigned lane = threadIdx.x & 31u;
    int2 stk[kPStack];  // (ref, this lane's key); refs are the same in every lane
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(counter, 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= (unsigned long long)n) break;
        const int64_t i = (int64_t)base + lane;
        const bool alive = i < n;
        const int64_t qi = alive ? (perm ? (int64_t)__ldg(perm + i) : i) : 0;
        float p[3] = {0.f, 0.f, 0.f};
        if (alive)
            for (int k = 0; k < 3; ++k) p[k] = qget(q, qi, k);
        float r = alive ? kInf : 0.f;  // squared search radius
        int idx = -1;
        int cur = LAYOUT ? s.wroot_ref : s.root_ref;
        unsigned cmask = __ballot_sync(0xffffffffu, alive);
        int sp = -1;
        bool ovf = false;
        for (;;) {
            if (cur == kNone) {
                bool found = false;
                while (sp >= 0) {
                    const int2 e = stk[sp--];
                    const unsigned m = __ballot_sync(0xffffffffu, __int_as_float(e.y) <= r * kSlack);
                    if (m) {
                        cur = e.x;
                        cmask = m;
                        found = true;
                        break;
                    }
                }
                if (!found) break;
            }
            const bool act = (cmask >> lane) & 1u;
            if (cur < 0) {
                packet_leaf(s, cur, act, p, r, idx);
                cur = kNone;
                continue;
            }
            if (LAYOUT == 0) {
                const float4 a = ldg4(s.pairs, 4 * (int64_t)cur), b = ldg4(s.pairs, 4 * (int64_t)cur + 1),
                             c = ldg4(s.pairs, 4 * (int64_t)cur + 2);
                const int4 rr = __ldg(reinterpret_cast<const int4 *>(s.pairs) + 4 * (int64_t)cur + 3);
                float a2l = kInf, b2l = kInf, a2r = kInf, b2r = kInf;
                if (act) {
                    box_sq(a.x, a.y, a.z, a.w, b.x, b.y, p, a2l, b2l);
                    box_sq(b.z, b.w, c.x, c.y, c.z, c.w, p, a2r, b2r);
                    r = fminf(r, fminf(b2l, b2r) * kSlack);
                }
                const float lim = r * kSlack;
                const bool hl = act && a2l <= lim, hr = act && a2r <= lim;
                const unsigned ml = __ballot_sync(0xffffffffu, hl), mr = __ballot_sync(0xffffffffu, hr);
                if (ml && mr) {
                    const float kl = warp_min(hl ? a2l : kInf), kr = warp_min(hr ? a2r : kInf);
                    const bool right_first = kr < kl;
                    if (sp + 1 >= kPStack) {
                        ovf = true;
                        break;
                    }
                    stk[++sp] = right_first ? make_int2(rr.x, fbits(hl ? a2l : kInf))
                                            : make_int2(rr.y, fbits(hr ? a2r : kInf));
                    cur = right_first ? rr.y : rr.x;
                    cmask = right_first ? mr : ml;
                } else if (ml) {
                    cur = rr.x;
                    cmask = ml;
                } else if (mr) {
                    cur = rr.y;
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
                    float a2 = kInf, b2 = kInf;
                    if (act && k < nc)
                        box_sq(__fmaf_rn(qf(q0.x, q0.y, k), sx, h.x), __fmaf_rn(qf(q0.z, q0.w, k), sy, h.y),
                               __fmaf_rn(qf(q1.x, q1.y, k), sz, h.z), __fmaf_rn(qf(q1.z, q1.w, k), sx, h.x),
                               __fmaf_rn(qf(q2.x, q2.y, k), sy, h.y), __fmaf_rn(qf(q2.z, q2.w, k), sz, h.z), p, a2,
                               b2);
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
                    const bool hit = act && key[k] <= lim;
                    key[k] = hit ? key[k] : kInf;
                    wmask[k] = __ballot_sync(0xffffffffu, hit);
                    wkey[k] = wmask[k] ? warp_min(key[k]) : kInf;
                    cnt += wmask[k] ? 1 : 0;
                }
                if (cnt == 0) {
                    cur = kNone;
                    continue;
                }
                if (sp + cnt > kPStack) {
                    ovf = true;
                    break;
                }
                if (MINFIRST) {
                    // the child nearest to any lane continues; the other hits are pushed
                    // in descending child order (static indices, no data movement)
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
                            stk[++sp] = make_int2(ref[k], fbits(key[k]));
                        }
                    }
                    cur = c0;
                    cmask = m0;
                    continue;
                }
                // warp order by the nearest lane's distance; lane keys travel with the refs
                int slot[8] = {0, 1, 2, 3, 4, 5, 6, 7};
                float wk[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) wk[k] = wkey[k];
                sort8(wk, slot);
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
                        stk[++sp] = make_int2(sref, fbits(skey));
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
        if (ovf && lane == 0 && s.err) atomicOr(s.err, GQ_DEVERR_STACK);
        if (alive) cp3_record(s.prims, idx, (idx >= 0) && !ovf, p[0], p[1], p[2], o, n, qi);
    }
}

}  // namespace

cudaError_t launch_cp3_packet(const DevScene &s, int layout, gq_vecs q, int64_t n, const int32_t *perm,
                              const gq_cp_out &o, unsigned long long *counter, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    // layout: 0 binary pairs, 1 quantised 8-wide (sorted children), 2 quantised 8-wide (nearest first)
    static int bps[3] = {0, 0, 0}, n_sm = 0;
    if (!bps[layout]) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        if (layout == 2)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps[2], k_cp3_packet<1, true>, kBlock, 0);
        else if (layout == 1)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps[1], k_cp3_packet<1, false>, kBlock, 0);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps[0], k_cp3_packet<0, false>, kBlock, 0);
        if (bps[layout] < 1) bps[layout] = 1;
    }
    const int64_t warps = (n + 31) / 32;
    const int64_t want = std::min<int64_t>((int64_t)bps[layout] * n_sm, (warps * 32 + kBlock - 1) / kBlock);
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    const dim3 g((unsigned)want);
    if (layout == 2)
        k_cp3_packet<1, true><<<g, kBlock, 0, st>>>(s, q, n, perm, o, counter);
    else if (layout == 1)
        k_cp3_packet<1, false><<<g, kBlock, 0, st>>>(s, q, n, perm, o, counter);
    else
        k_cp3_packet<0, false><<<g, kBlock, 0, st>>>(s, q, n, perm, o, counter);
    return cudaGetLastError();
}

}  // namespace gqd
