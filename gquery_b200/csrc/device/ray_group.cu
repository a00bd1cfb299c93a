// Ray traversal over the quantised 8-wide BVH with one ray per group of 8 lanes.
//
// The per-lane wide traversal (traverse.cuh) gives each lane a ray of its own: a lane
// decodes and slab-tests all eight children of every node it visits, and lanes of one
// warp are soon at different nodes, at leaves or refilling, so few lanes do work in
// any one instruction.  Here the eight lanes of a group carry the same ray: at a node
// lane j decodes child j alone and tests it; the group then continues into its nearest
// hit child and pushes the others (in child order) on a stack it keeps in shared
// memory; at a leaf the lanes test up to eight of its items at once and keep the
// nearest (the first in leaf order among equal distances, like the per-lane loop).
// A warp holds four rays; a group that finishes takes the next ray of the permutation
// (one atomic per warp for all groups that need one).
//
// Decisions follow the per-lane wide traversal: the same decoded child boxes, the same
// widened slab test against the current best hit, the same pop test, the same leaf
// tests (tri_ray / seg_ray) and record writers, so the answers equal it, and the exact
// traversal, except at FP32 distance ties (a different visit order can meet the other
// of two equally distant hits first).
#include <algorithm>

#include "prim.cuh"
#include "queries.cuh"
#include "records.cuh"
#include "traverse.cuh"

namespace gqd {

namespace {

constexpr int kG = 8;              // lanes per ray
constexpr int kBlockG = 128;       // threads per block
constexpr int kGroups = kBlockG / kG;

template <int D>
__global__ void __launch_bounds__(kBlockG) k_ray_g8(DevScene s, gq_vecs a, gq_vecs b, const float *rmax_in, int64_t n,
                                                 const int32_t *perm, gq_ray_out o, unsigned long long *counter) {
    __shared__ int2 gstk[kGroups][GQ_STACK_WIDE];
    const unsigned lane = threadIdx.x & 31u;
    const int j = (int)(lane & 7u);        // the child / item slot of this lane
    const unsigned g0 = lane & ~7u;        // first lane of the group
    const unsigned gmask = 0xffu << g0;
    int2 *stk = gstk[threadIdx.x >> 3];
    const int cap = min(GQ_STACK_WIDE, s.stack_cap);
    constexpr int F4 = (D == 3) ? 6 : 5;   // 16-byte words per wide node

    float p[D], v[D], iv[D], r = 0.f;
    int cur = trav::kNone, sp = -1, idx = -1;
    bool live = false, drained = false, ovf = false;
    int64_t qi = 0;
    for (;;) {
        if (!drained) {
            const unsigned need = __ballot_sync(0xffffffffu, !live && j == 0);
            if (need) {
                const int leader = __ffs(need) - 1;
                unsigned long long base = 0;
                if ((int)lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(need));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (base + __popc(need) >= (unsigned long long)n) drained = true;
                if (!live) {
                    const unsigned long long mine = base + __popc(need & ((1u << g0) - 1u));
                    if (mine < (unsigned long long)n) {
                        qi = perm ? (int64_t)__ldg(perm + mine) : (int64_t)mine;
#pragma unroll
                        for (int k = 0; k < D; ++k) {
                            p[k] = trav::qget(a, qi, k);
                            v[k] = trav::qget(b, qi, k);
                            iv[k] = gq_div(1.f, v[k]);
                        }
                        r = rmax_in ? rmax_in[qi] : kInf;
                        float t_root;
                        bool hit;
                        if (D == 3)
                            hit = box_ray3(s.root_lo[0], s.root_lo[1], s.root_lo[2], s.root_hi[0], s.root_hi[1],
                                           s.root_hi[2], p[0], p[1], p[D - 1], v[0], v[1], v[D - 1], r, t_root);
                        else
                            hit = box_ray2(s.root_lo[0], s.root_lo[1], s.root_hi[0], s.root_hi[1], p[0], p[D - 1],
                                           v[0], v[D - 1], r, t_root);
                        cur = (hit && t_root <= r) ? s.wroot_ref : trav::kNone;
                        sp = -1;
                        idx = -1;
                        ovf = false;
                        live = true;
                    }
                }
            }
        }
        if (!__any_sync(0xffffffffu, live)) break;
        if (!live) continue;
        // everything below is uniform within the group and synchronises the group only
        if (cur == trav::kNone) {
            while (sp >= 0) {
                const int2 e = stk[sp--];
                if (__int_as_float(e.y) <= r) {
                    cur = e.x;
                    break;
                }
            }
        }
        if (cur == trav::kNone) {  // finished
            if (j == 0) {
                if (ovf && s.err) atomicOr(s.err, GQ_DEVERR_STACK);
                const bool found = idx >= 0 && !ovf;
                if (D == 3)
                    ray3_record(s.prims, idx, found, p[0], p[1], p[D - 1], v[0], v[1], v[D - 1], r, o, n, qi);
                else
                    ray2_record(s.prims, idx, found, p[0], p[D - 1], v[0], v[D - 1], r, o, n, qi);
            }
            live = false;
            continue;
        }
        if (cur >= 0) {
            // node: lane j decodes and tests child j (traverse.cuh visit_wide, one child per lane)
            const int64_t base = F4 * (int64_t)cur;
            const float4 h = ldg4(s.wnodes, base);
            const int myref = __ldg(reinterpret_cast<const int *>(s.wnodes) + 4 * (base + 1) + j);
            const uint4 q0 = __ldg(reinterpret_cast<const uint4 *>(s.wnodes) + base + 3);
            const uint4 q1 = __ldg(reinterpret_cast<const uint4 *>(s.wnodes) + base + 4);
            uint4 q2 = make_uint4(0, 0, 0, 0);
            if (D == 3) q2 = __ldg(reinterpret_cast<const uint4 *>(s.wnodes) + base + 5);
            const uint32_t meta = (uint32_t)fbits(D == 3 ? h.w : h.z);
            const int nc = (int)(meta >> 24);
            bool hit = false;
            float key = kInf;
            if (j < nc) {
                const float sx = trav::exp_scale(meta, 0), sy = trav::exp_scale(meta, 1);
                float lo[D], hi[D];
                if (D == 3) {
                    const float sz = trav::exp_scale(meta, 2);
                    lo[0] = __fmaf_rn(trav::qf(q0.x, q0.y, j), sx, h.x);
                    lo[1] = __fmaf_rn(trav::qf(q0.z, q0.w, j), sy, h.y);
                    lo[D - 1] = __fmaf_rn(trav::qf(q1.x, q1.y, j), sz, h.z);
                    hi[0] = __fmaf_rn(trav::qf(q1.z, q1.w, j), sx, h.x);
                    hi[1] = __fmaf_rn(trav::qf(q2.x, q2.y, j), sy, h.y);
                    hi[D - 1] = __fmaf_rn(trav::qf(q2.z, q2.w, j), sz, h.z);
                } else {
                    lo[0] = __fmaf_rn(trav::qf(q0.x, q0.y, j), sx, h.x);
                    lo[D - 1] = __fmaf_rn(trav::qf(q0.z, q0.w, j), sy, h.y);
                    hi[0] = __fmaf_rn(trav::qf(q1.x, q1.y, j), sx, h.x);
                    hi[D - 1] = __fmaf_rn(trav::qf(q1.z, q1.w, j), sy, h.y);
                }
                float tn = 0.f, tf = kInf;
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    const float t0 = (lo[c] - p[c]) * iv[c], t1 = (hi[c] - p[c]) * iv[c];
                    tn = fmaxf(tn, fminf(t0, t1));
                    tf = fminf(tf, fmaxf(t0, t1));
                }
                hit = tn <= fminf(tf * trav::kFar, r * trav::kFar);
                key = hit ? fminf(tn, trav::kMaxHitKey) : kInf;  // hits stay below the others' +inf
            }
            const unsigned hm = (__ballot_sync(gmask, hit) >> g0) & 0xffu;
            if (hm == 0) {
                cur = trav::kNone;
                continue;
            }
            // the nearest hit child (lowest slot among equal entry distances) continues
            float bk = key;
            int bj = j;
#pragma unroll
            for (int off = 1; off < kG; off <<= 1) {
                const float ok = __shfl_xor_sync(gmask, bk, off);
                const int oj = __shfl_xor_sync(gmask, bj, off);
                const bool take = (ok < bk) || (ok == bk && oj < bj);
                bk = take ? ok : bk;
                bj = take ? oj : bj;
            }
            const unsigned others = hm & ~(1u << bj);
            const int cnt = __popc(others);
            if (sp + cnt >= cap) {
                ovf = true;
                cur = trav::kNone;
                sp = -1;
                continue;
            }
            if ((others >> j) & 1u) stk[sp + 1 + __popc(others & ((1u << j) - 1u))] = make_int2(myref, fbits(key));
            sp += cnt;
            cur = __shfl_sync(gmask, myref, (int)g0 + bj);
            __syncwarp(gmask);  // the group's pushes are visible to its later pops
        } else {
            // leaf: up to eight items at once, the first nearest in leaf order kept; a run
            // child (bit 30 clear) ends after its count, an ordinary leaf at its last item
            const bool run = (cur & 0x40000000) == 0;
            int64_t j0 = run ? (int64_t)(cur & 0xffffff) : ~(int64_t)cur;
            const int64_t end = run ? j0 + ((cur >> 24) & 0x3f) : s.n_prims;
            for (;;) {
                const int64_t it = j0 + j;
                const bool in = it < end;
                bool last = !in;
                float key = kInf;
                if (in) {
                    if (D == 3) {
                        const float4 t0 = ldg4(s.prims, 3 * it), t1 = ldg4(s.prims, 3 * it + 1),
                                     t2 = ldg4(s.prims, 3 * it + 2);
                        last = run ? it + 1 == end : (fbits(t2.z) & GQ_ITEM_LAST) != 0;
                        key = tri_ray(p[0], p[1], p[D - 1], v[0], v[1], v[D - 1], t0.x, t0.y, t0.z, t0.w, t1.x, t1.y,
                                      t1.z, t1.w, t2.x, kInf);
                    } else {
                        const float4 e = ldg4(s.prims, 2 * it);
                        const int4 f = __ldg(reinterpret_cast<const int4 *>(s.prims) + 2 * it + 1);
                        last = run ? it + 1 == end : (f.y & GQ_ITEM_LAST) != 0;
                        key = seg_ray(p[0], p[D - 1], v[0], v[D - 1], e.x, e.y, e.z, e.w);
                    }
                }
                const unsigned lm = (__ballot_sync(gmask, last) >> g0) & 0xffu;
                const int upto = lm ? __ffs(lm) - 1 : kG - 1;  // lanes past the leaf's last item drop out
                if (j > upto) key = kInf;
                float bk = key;
                int bj = j;
#pragma unroll
                for (int off = 1; off < kG; off <<= 1) {
                    const float ok = __shfl_xor_sync(gmask, bk, off);
                    const int oj = __shfl_xor_sync(gmask, bj, off);
                    const bool take = (ok < bk) || (ok == bk && oj < bj);
                    bk = take ? ok : bk;
                    bj = take ? oj : bj;
                }
                if (bk < r) {
                    r = bk;
                    idx = (int)(j0 + bj);
                }
                if (lm) break;
                j0 += kG;
            }
            cur = trav::kNone;
        }
    }
}

template <int D>
cudaError_t launch(const DevScene &s, gq_vecs x, gq_vecs v, const float *r_max, int64_t n, const int32_t *perm,
                   const gq_ray_out &o, unsigned long long *counter, cudaStream_t st) {
    static int bps = 0, n_sm = 0;
    if (!bps) {
        int dev = 0, b = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_ray_g8<D>, kBlockG, 0);
        bps = b < 1 ? 1 : b;
    }
    const int64_t want = std::min<int64_t>((int64_t)bps * n_sm, (n * kG + kBlockG - 1) / kBlockG);
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    k_ray_g8<D><<<dim3((unsigned)want), kBlockG, 0, st>>>(s, x, v, r_max, n, perm, o, counter);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_ray_group(const DevScene &s, gq_vecs x, gq_vecs v, const float *r_max, int64_t n,
                             const int32_t *perm, const gq_ray_out &o, unsigned long long *counter, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (!s.wnodes || !counter) return cudaErrorInvalidValue;
    return s.dim == 3 ? launch<3>(s, x, v, r_max, n, perm, o, counter, st)
                      : launch<2>(s, x, v, r_max, n, perm, o, counter, st);
}

}  // namespace gqd
