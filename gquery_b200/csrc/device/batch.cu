// Many scenes, three query kinds, one persistent launch.
//
// Queries of each kind are sorted by (scene, Hilbert index inside the scene's box).
// Persistent warps work through the kinds in the order closest point, rays,
// silhouettes (a warp-uniform phase).  Closest points run as tiles of 32 sorted
// queries with the warp-coherent traversal once per distinct scene in the tile
// (tiles straddle at most a scene boundary or two); rays and silhouettes run one
// traversal per lane on the lane's own scene, and a lane whose query is done takes
// the next one.  Every launch input lives in caller- or batch-owned device memory,
// so a step can be captured in a CUDA graph.
#include <cub/cub.cuh>

#include "batch.cuh"
#include "cp_warp.cuh"
#include "curves.cuh"
#include "packet.cuh"
#include "records.cuh"
#include "sil_packet.cuh"
#include "sil_warp.cuh"
#include "snch.cuh"
#include "traverse.cuh"

namespace gqd {

namespace {

constexpr int kBlock = 128;

__device__ __forceinline__ float qget(const gq_vecs &v, int64_t i, int k) {
    return v.ptr[(int64_t)k * v.comp_stride + i * v.elem_stride];
}

// Identity order for the three kinds (steps answered without sorting) and the phases'
// claim counters zeroed, in one launch.
__global__ void k_batch_ident(int32_t *perm0, int64_t n0, int32_t *perm1, int64_t n1, int32_t *perm2, int64_t n2,
                              unsigned long long *counter, int n_counters) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n0) perm0[i] = (int32_t)i;
    if (i < n1) perm1[i] = (int32_t)i;
    if (i < n2) perm2[i] = (int32_t)i;
    if (i < n_counters) counter[i] = 0ull;
}

// key = scene << 32 | Hilbert index of the query's cell on a grid over twice the scene's box
__global__ void k_batch_keys(const DevScene *scenes, int n_scenes, BatchKind k, int64_t n, uint64_t *keys,
                             int32_t *vals, int32_t *bad) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int sid = __ldg(k.scene + i);
    if (sid == GQ_BATCH_SKIP) {  // padding slot: sorted last, skipped by the traversal
        keys[i] = ~0ull;
        vals[i] = (int32_t)i;
        return;
    }
    if (sid < 0 || sid >= n_scenes) {
        atomicOr(bad, GQ_BATCH_ERR_SCENE);
        sid = 0;
    }
    const DevScene &s = scenes[sid];
    const int dim = s.dim;
    uint32_t code = 0;
    if (dim == 3) {
        uint32_t c[3];
        for (int a = 0; a < 3; ++a) {
            const float mid = 0.5f * (s.root_lo[a] + s.root_hi[a]);
            float ext = s.root_hi[a] - s.root_lo[a];
            if (!(ext > 0.f)) ext = 1.f;
            float f = (qget(k.a, i, a) - (mid - ext)) * (1024.f / (2.f * ext));
            c[a] = (uint32_t)fminf(fmaxf(f, 0.f), 1023.f);
        }
        code = hilbert3(c[0], c[1], c[2]);
    } else {
        uint32_t c[2];
        for (int a = 0; a < 2; ++a) {
            const float mid = 0.5f * (s.root_lo[a] + s.root_hi[a]);
            float ext = s.root_hi[a] - s.root_lo[a];
            if (!(ext > 0.f)) ext = 1.f;
            float f = (qget(k.a, i, a) - (mid - ext)) * (32768.f / (2.f * ext));
            c[a] = (uint32_t)fminf(fmaxf(f, 0.f), 32767.f);
        }
        code = hilbert2(c[0], c[1]);
    }
    keys[i] = ((uint64_t)(uint32_t)sid << 32) | code;
    vals[i] = (int32_t)i;
}

template <int D>
__device__ __forceinline__ void put_sil(const gq_sil_out &o, int64_t n, int64_t qi, bool found, const float *bp,
                                        float bd, int bid) {
    if (o.valid) o.valid[qi] = found ? 1 : 0;
    if (o.p)
#pragma unroll
        for (int k = 0; k < D; ++k) o.p[k * n + qi] = found ? bp[k] : 0.f;
    if (o.d) o.d[qi] = found ? bd : 0.f;
    if (o.prim_id) o.prim_id[qi] = found ? bid : 0;
}

// Lane-refill loop over the n sorted queries of one kind (persistent warps): a lane
// without a query claims the next one through a warp-aggregated atomic on `counter`;
// `start(i)` sets it up and says whether it needs a traversal (padding slots and bad
// scene indices do not), `step(budget)` runs up to `budget` steps and says whether
// the query is done, `finish()` writes its record.
template <class Start, class Step, class Finish>
__device__ __forceinline__ void refill(int64_t n, unsigned long long *counter, int budget, Start start, Step step,
                                       Finish finish) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    bool live = false, drained = false;
    for (;;) {
        if (!drained) {
            const unsigned need = __ballot_sync(0xffffffffu, !live);
            if (need) {
                const int leader = __ffs(need) - 1;
                unsigned long long base = 0;
                if ((int)lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(need));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (base + __popc(need) >= (unsigned long long)n) drained = true;
                if (!live) {
                    const unsigned long long mine = base + __popc(need & below);
                    if (mine < (unsigned long long)n) live = start((int64_t)mine);
                }
            }
        }
        if (!__any_sync(0xffffffffu, live)) {
            if (drained) break;
            continue;
        }
        if (live && step(budget)) {
            finish();
            live = false;
        }
    }
}

// One silhouette query (sorted position t) on one warp (sil_warp.cuh), the warp's stack
// at wst.
template <int D>
__device__ __forceinline__ void sil_warp_query(const DevScene *scenes, int n_scenes, const BatchKind &sil,
                                               const gq_sil_out &sil_out, int32_t *err, int64_t t, int2 *wst) {
    const unsigned lane = threadIdx.x & 31u;
    const int64_t qi = (int64_t)__ldg(sil.perm + t);
    const int sid = __ldg(sil.scene + qi);
    if (sid == GQ_BATCH_SKIP) return;
    float x[D];
#pragma unroll
    for (int k = 0; k < D; ++k) x[k] = qget(sil.a, qi, k);
    const bool known = (unsigned)sid < (unsigned)n_scenes;
    if (!known || !scenes[sid].spairs) {
        if (lane == 0) {
            atomicOr(err, known ? GQ_BATCH_ERR_NO_SNCH : GQ_BATCH_ERR_SCENE);
            put_sil<D>(sil_out, sil.n, qi, false, x, 0.f, 0);
        }
        return;
    }
    snch::Lane<D> L;
    wsil::closest_silhouette<D>(scenes[sid], x, sil.r_max ? sil.r_max[qi] : kInf, L, wst);
    if (lane == 0) {
        if (L.ovf && scenes[sid].err) atomicOr(scenes[sid].err, GQ_DEVERR_STACK);
        put_sil<D>(sil_out, sil.n, qi, L.found && !L.ovf, L.bp, L.bd, L.bid);
    }
}

// Phase 3, sil_mode 2: one silhouette query per warp, persistent warps claiming the
// next one (counter[2]); the warp's stack in dynamic shared memory.
template <int D>
__device__ __forceinline__ void sil_warp_phase(const DevScene *scenes, int n_scenes, const BatchKind &sil,
                                               const gq_sil_out &sil_out, unsigned long long *counter,
                                               int32_t *err) {
    const unsigned lane = threadIdx.x & 31u;
    extern __shared__ int2 wstk[];
    int2 *wst = wstk + (threadIdx.x >> 5) * wsil::kWarpStack;
    for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(&counter[2], 1ull);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= (unsigned long long)sil.n) break;
        sil_warp_query<D>(scenes, n_scenes, sil, sil_out, err, (int64_t)t, wst);
    }
}

// Closest-point queries whose per-lane traversal passes this many node visits are
// handed to k_cp_heavy (cp_mode 2).
constexpr int kHeavyVisits = 1024;
// Node visits (closest points, rays) or steps (silhouettes) between refills in k_batch.
constexpr int kBudget = 32;

// Hand-over lists of the split modes (in the kinds' sort scratch): query index, and
// (best primitive or silhouette, r_max bits) the lane had reached.
struct Handover {
    int32_t *cp_q = nullptr;
    int2 *cp_r = nullptr;
    int32_t *sil_q = nullptr;
    int2 *sil_r = nullptr;
};
// Silhouette queries whose per-lane traversal passes this many steps (node visits and
// silhouette tests) are handed to k_sil_heavy (sil_mode 3).
constexpr int kHeavySilSteps = 2048;

// One persistent launch per step.  Phase 1: closest points, as warp tiles of 32
// sorted queries (warp-coherent traversal once per distinct scene in the tile) or
// one lane per query (cp_mode 0; in cp_mode 2 a query past kHeavyVisits node visits
// is appended to the hand-over list and left to k_cp_heavy).  Phase 2: rays, one lane
// per query.  Phase 3: silhouettes (sil_mode): 1 warp-coherent tiles like the closest points, 2
// one query per warp (sil_warp.cuh), 0 one lane per query in the reference order, 3
// the same with queries past kHeavySilSteps handed to k_sil_heavy.  Every warp moves
// to the next phase when the current one has no unclaimed work, so the phases' tails
// overlap.  counter[0..2]: claims per phase, counter[3] / [5]: closest points /
// silhouettes handed over.
// SPLIT: compiled with the hand-over of cp_mode 2 / sil_mode 3 (its state costs
// registers that the other modes need not carry); SIL: compiled with the silhouette
// phase (steps without silhouettes, such as the server's general ones, leave it out).
template <int D, bool RAYW, bool SPLIT, bool SIL>
__global__ void __launch_bounds__(kBlock) k_batch(const DevScene *scenes, int n_scenes, BatchKind cp, gq_cp_out cp_out,
                                                  BatchKind ray, gq_ray_out ray_out, BatchKind sil,
                                                  gq_sil_out sil_out, int cp_mode, int sil_mode,
                                                  int budget, unsigned long long *counter, Handover ho,
                                                  int32_t *err) {
    const unsigned lane = threadIdx.x & 31u;
    // ---------------- phase 1: closest points ----------------
    if (cp_mode == 1) {
        const int64_t t_cp = (cp.n + 31) / 32;
        int2 stk[pkt::kPStack];
        for (;;) {
            unsigned long long t = 0;
            if (lane == 0) t = atomicAdd(&counter[0], 1ull);
            t = __shfl_sync(0xffffffffu, t, 0);
            if (t >= (unsigned long long)t_cp) break;
            const int64_t i = (int64_t)t * 32 + lane;
            const bool in = i < cp.n;
            const int64_t qi = in ? (int64_t)__ldg(cp.perm + i) : 0;
            const int sid = in ? __ldg(cp.scene + qi) : GQ_BATCH_SKIP;
            const bool alive = in && (unsigned)sid < (unsigned)n_scenes;
            const bool skip = !in || sid == GQ_BATCH_SKIP;
            if (!skip && !alive) atomicOr(err, GQ_BATCH_ERR_SCENE);
            float p[D];
#pragma unroll
            for (int k = 0; k < D; ++k) p[k] = alive ? qget(cp.a, qi, k) : 0.f;
            int best_idx = -1;
            bool ovf = false;
            unsigned todo = __ballot_sync(0xffffffffu, alive);
            while (todo) {
                const int s0 = __shfl_sync(0xffffffffu, sid, __ffs(todo) - 1);
                const unsigned m = __ballot_sync(0xffffffffu, alive && sid == s0);
                float r = kInf;
                int idx = -1;
                bool o = false;
                pkt::closest_point<D, 0, false>(scenes[s0], m, p, r, idx, o, pkt::PStack<false>(stk));
                if ((m >> lane) & 1u) {
                    best_idx = idx;
                    ovf = o;
                }
                todo &= ~m;
            }
            if (!skip) {
                const DevScene &s = scenes[alive ? sid : 0];
                if (ovf && s.err) atomicOr(s.err, GQ_DEVERR_STACK);
                const bool found = alive && best_idx >= 0 && !ovf;
                if (D == 3)
                    cp3_record(s.prims, best_idx, found, p[0], p[1], p[D - 1], cp_out, cp.n, qi);
                else
                    cp2_record(s.prims, best_idx, found, p[0], p[D - 1], cp_out, cp.n, qi);
            }
        }
    } else if (cp.n > 0) {
        trav::Stack<false> stk;
        trav::Lane<D, false, false> L;
        const DevScene *sc = scenes;
        int64_t qi = 0;
        int visits = 0;
        bool handed = false;
        const bool split = SPLIT && cp_mode == 2;
        const gq_vecs none{};
        refill(
            cp.n, &counter[0], budget,
            [&](int64_t i) {
                visits = 0;
                handed = false;
                qi = (int64_t)__ldg(cp.perm + i);
                const int sid = __ldg(cp.scene + qi);
                if (sid == GQ_BATCH_SKIP) return false;
                if ((unsigned)sid >= (unsigned)n_scenes) {
                    atomicOr(err, GQ_BATCH_ERR_SCENE);
                    if (D == 3)
                        cp3_record(nullptr, -1, false, 0.f, 0.f, 0.f, cp_out, cp.n, qi);
                    else
                        cp2_record(nullptr, -1, false, 0.f, 0.f, cp_out, cp.n, qi);
                    return false;
                }
                sc = scenes + sid;
                trav::lane_init(*sc, L, cp.a, none, nullptr, qi);
                return true;
            },
            [&](int b) {
                if (trav::lane_run<D, false, false, 0>(*sc, L, stk, b)) return true;
                visits += b;
                if (split && visits >= kHeavyVisits) {  // long traversal: one warp takes it over
                    const unsigned long long h = atomicAdd(&counter[3], 1ull);
                    ho.cp_q[h] = (int32_t)qi;
                    ho.cp_r[h] = make_int2(L.idx, fbits(L.r));
                    handed = true;
                    return true;
                }
                return false;
            },
            [&]() {
                if (!handed) trav::lane_write(*sc, L, qi, cp.n, cp_out, gq_ray_out{});
            });
    }
    // ---------------- phase 2: rays ----------------
    if (ray.n > 0) {
        trav::Stack<RAYW> stk;
        trav::Lane<D, true, RAYW> L;
        const DevScene *sc = scenes;
        int64_t qi = 0;
        refill(
            ray.n, &counter[1], budget,
            [&](int64_t i) {
                qi = (int64_t)__ldg(ray.perm + i);
                const int sid = __ldg(ray.scene + qi);
                if (sid == GQ_BATCH_SKIP) return false;
                if ((unsigned)sid >= (unsigned)n_scenes) {
                    atomicOr(err, GQ_BATCH_ERR_SCENE);
                    if (D == 3)
                        ray3_record(nullptr, -1, false, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, ray_out, ray.n, qi);
                    else
                        ray2_record(nullptr, -1, false, 0.f, 0.f, 0.f, 0.f, 0.f, ray_out, ray.n, qi);
                    return false;
                }
                sc = scenes + sid;
                trav::lane_init(*sc, L, ray.a, ray.b, ray.r_max, qi);
                return true;
            },
            [&](int b) { return trav::lane_run<D, true, RAYW, 0>(*sc, L, stk, b); },
            [&]() { trav::lane_write(*sc, L, qi, ray.n, gq_cp_out{}, ray_out); });
    }
    // ---------------- phase 3: silhouettes ----------------
    if (!SIL) return;
    if (sil.n > 0 && sil_mode == 2) {
        sil_warp_phase<D>(scenes, n_scenes, sil, sil_out, counter, err);
    } else if (sil.n > 0 && sil_mode == 1) {
        const int64_t t_sil = (sil.n + 31) / 32;
        snch::Stack stk;
        for (;;) {
            unsigned long long t = 0;
            if (lane == 0) t = atomicAdd(&counter[2], 1ull);
            t = __shfl_sync(0xffffffffu, t, 0);
            if (t >= (unsigned long long)t_sil) break;
            const int64_t i = (int64_t)t * 32 + lane;
            const bool in = i < sil.n;
            const int64_t qi = in ? (int64_t)__ldg(sil.perm + i) : 0;
            const int sid = in ? __ldg(sil.scene + qi) : GQ_BATCH_SKIP;
            const bool known = in && (unsigned)sid < (unsigned)n_scenes;
            const bool alive = known && scenes[sid].spairs != nullptr;
            const bool skip = !in || sid == GQ_BATCH_SKIP;
            if (!skip && !alive) atomicOr(err, known ? GQ_BATCH_ERR_NO_SNCH : GQ_BATCH_ERR_SCENE);
            snch::Lane<D> L;
#pragma unroll
            for (int k = 0; k < D; ++k) L.x[k] = alive ? qget(sil.a, qi, k) : 0.f;
            L.r = alive ? (sil.r_max ? sil.r_max[qi] : kInf) : -1.f;
            L.found = false;
            L.ovf = false;
            unsigned todo = __ballot_sync(0xffffffffu, alive);
            while (todo) {
                const int s0 = __shfl_sync(0xffffffffu, sid, __ffs(todo) - 1);
                const unsigned m = __ballot_sync(0xffffffffu, alive && sid == s0);
                snch::Lane<D> M = L;
                if (!((m >> lane) & 1u)) M.r = -1.f;
                pkt::closest_silhouette<D>(scenes[s0], m, M, stk);
                if ((m >> lane) & 1u) L = M;
                todo &= ~m;
            }
            if (!skip) {
                if (alive && L.ovf && scenes[sid].err) atomicOr(scenes[sid].err, GQ_DEVERR_STACK);
                put_sil<D>(sil_out, sil.n, qi, alive && L.found && !L.ovf, L.bp, L.bd, L.bid);
            }
        }
    } else if (sil.n > 0) {
        snch::Stack stk;
        snch::Lane<D> L;
        const DevScene *sc = scenes;
        int64_t qi = 0;
        int steps = 0;
        bool handed = false;
        const bool split = SPLIT && sil_mode == 3;
        refill(
            sil.n, &counter[2], budget,
            [&](int64_t i) {
                steps = 0;
                handed = false;
                qi = (int64_t)__ldg(sil.perm + i);
                const int sid = __ldg(sil.scene + qi);
                if (sid == GQ_BATCH_SKIP) return false;
                float x[D];
#pragma unroll
                for (int k = 0; k < D; ++k) x[k] = qget(sil.a, qi, k);
                if ((unsigned)sid >= (unsigned)n_scenes || !scenes[sid].spairs) {
                    atomicOr(err, (unsigned)sid >= (unsigned)n_scenes ? GQ_BATCH_ERR_SCENE : GQ_BATCH_ERR_NO_SNCH);
                    put_sil<D>(sil_out, sil.n, qi, false, x, 0.f, 0);
                    return false;
                }
                sc = scenes + sid;
                snch::lane_init<D>(*sc, L, x, sil.r_max ? sil.r_max[qi] : kInf, stk);
                return true;
            },
            [&](int b) {
                if (snch::lane_run<D>(*sc, L, stk, b)) return true;
                steps += b;
                if (split && steps >= kHeavySilSteps) {  // long traversal: one warp takes it over
                    const unsigned long long h = atomicAdd(&counter[5], 1ull);
                    ho.sil_q[h] = (int32_t)qi;
                    // the silhouette accepted so far (its position in the leaf order) and r_max
                    ho.sil_r[h] = make_int2(L.found ? L.bj : -1, fbits(L.r));
                    handed = true;
                    return true;
                }
                return false;
            },
            [&]() {
                if (handed) return;
                if (L.ovf && sc->err) atomicOr(sc->err, GQ_DEVERR_STACK);
                put_sil<D>(sil_out, sil.n, qi, L.found && !L.ovf, L.bp, L.bd, L.bid);
            });
    }
}

// Closest points handed over by k_batch (cp_mode 2): one query per warp (cp_warp.cuh),
// `heavy[0 .. counter[3])` their query indices, heavy_r the (best primitive, r_max) each
// lane had reached, counter[4] the claims.  Runs after k_batch on the same stream, so
// the list is complete.
template <int D>
__global__ void __launch_bounds__(kBlock) k_cp_heavy(const DevScene *scenes, BatchKind cp, gq_cp_out cp_out,
                                                     const int32_t *heavy, const int2 *heavy_r,
                                                     unsigned long long *counter) {
    extern __shared__ int2 hstk[];
    int2 *wst = hstk + (threadIdx.x >> 5) * wcp::kWarpStack;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned long long n_heavy = counter[3];
    for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(&counter[4], 1ull);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= n_heavy) break;
        const int64_t qi = __ldg(heavy + t);
        const DevScene &s = scenes[__ldg(cp.scene + qi)];  // checked by k_batch before the hand-over
        float p[D];
#pragma unroll
        for (int k = 0; k < D; ++k) p[k] = qget(cp.a, qi, k);
        const int2 carried = __ldg(heavy_r + t);
        int idx;
        bool ovf;
        wcp::closest_point<D>(s, p, __int_as_float(carried.y), carried.x, wst, idx, ovf);
        if (lane == 0) {
            if (ovf && s.err) atomicOr(s.err, GQ_DEVERR_STACK);
            const bool found = idx >= 0 && !ovf;
            if (D == 3)
                cp3_record(s.prims, idx, found, p[0], p[1], p[D - 1], cp_out, cp.n, qi);
            else
                cp2_record(s.prims, idx, found, p[0], p[D - 1], cp_out, cp.n, qi);
        }
    }
}

// Silhouettes handed over by k_batch (sil_mode 3): one query per warp (sil_warp.cuh)
// from the lane's r_max; the silhouette the lane had accepted, if any, stands unless a
// nearer one turns up.  sheavy[0 .. counter[5]) the query indices, sheavy_r the
// (accepted silhouette, r_max) pairs, counter[6] the claims.
template <int D>
__global__ void __launch_bounds__(kBlock) k_sil_heavy(const DevScene *scenes, BatchKind sil, gq_sil_out sil_out,
                                                      const int32_t *sheavy, const int2 *sheavy_r,
                                                      unsigned long long *counter) {
    extern __shared__ int2 hstk[];
    int2 *wst = hstk + (threadIdx.x >> 5) * wsil::kWarpStack;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned long long n_heavy = counter[5];
    for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(&counter[6], 1ull);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= n_heavy) break;
        const int64_t qi = __ldg(sheavy + t);
        const DevScene &s = scenes[__ldg(sil.scene + qi)];  // checked by k_batch before the hand-over
        const int2 carried = __ldg(sheavy_r + t);
        float x[D];
#pragma unroll
        for (int k = 0; k < D; ++k) x[k] = qget(sil.a, qi, k);
        snch::Lane<D> L;
        wsil::closest_silhouette<D>(s, x, __int_as_float(carried.y), L, wst);
        if (lane == 0) {
            if (L.ovf && s.err) atomicOr(s.err, GQ_DEVERR_STACK);
            if (!L.found && !L.ovf && carried.x >= 0) {
                // nothing nearer: the carried silhouette, its record recomputed by the same test
                snch::Lane<D> C;
#pragma unroll
                for (int k = 0; k < D; ++k) C.x[k] = x[k];
                C.r = kInf;
                C.found = false;
                snch::test_silhouette<D>(s, C, carried.x);
                put_sil<D>(sil_out, sil.n, qi, C.found, C.bp, C.bd, C.bid);
            } else {
                put_sil<D>(sil_out, sil.n, qi, L.found && !L.ovf, L.bp, L.bd, L.bid);
            }
        }
    }
}

// A step with silhouettes only on the whole GPU: the phase alone, so that its register
// count, not k_batch's, sets the residency; persistent warps.
template <int D>
__global__ void __launch_bounds__(kBlock, 8) k_batch_silw(const DevScene *scenes, int n_scenes, BatchKind sil,
                                                          gq_sil_out sil_out, unsigned long long *counter,
                                                          int32_t *err) {
    sil_warp_phase<D>(scenes, n_scenes, sil, sil_out, counter, err);
}

// A step with silhouettes only beside other work (the server's silhouette slots, which
// pass a share of the GPU): one block of one warp per query, which answers it and exits.
// Blocks end all the time, so the block scheduler places the pending blocks of
// higher-priority streams (the server's closest points and rays) first and fills the
// rest of the GPU with silhouettes: no share has to be set aside, and a large step uses
// all of the GPU when nothing else waits.  One warp per block, so a heavy query holds no
// idle warps; 32 blocks of 64 registers a thread fill the register file as the
// persistent form does.
template <int D>
__global__ void __launch_bounds__(32, 32) k_batch_silw1(const DevScene *scenes, int n_scenes, BatchKind sil,
                                                        gq_sil_out sil_out, int32_t *err) {
    __shared__ int2 wst[wsil::kWarpStack];
    sil_warp_query<D>(scenes, n_scenes, sil, sil_out, err, (int64_t)blockIdx.x, wst);
}

template <int D, bool RAYW>
cudaError_t launch_batch(const DevScene *scenes_dev, int n_scenes, BatchKind kinds[3], const gq_cp_out &cp_out,
                         const gq_ray_out &ray_out, const gq_sil_out &sil_out, int cp_mode, int sil_mode,
                         float grid_share, int block, unsigned long long *counter, Handover ho, int32_t *err,
                         cudaStream_t st) {
    const int bi = block == 32 ? 1 : 0;  // k_batch and the hand-over kernels: blocks of kBlock or 32 threads
    // the one-query-per-warp silhouette phase keeps its stacks in dynamic shared memory
    const size_t smem = (sil_mode == 2 && kinds[2].n > 0) ? (size_t)(block / 32) * wsil::kWarpStack * sizeof(int2) : 0;
    if (smem && kinds[0].n <= 0 && kinds[1].n <= 0) {  // silhouettes only: the phase's own kernel
        if (grid_share > 0.f && grid_share < 1.f) {      // beside other work: one block per query
            if (kinds[2].n > 0x7fffffff) return cudaErrorInvalidValue;
            k_batch_silw1<D><<<dim3((unsigned)kinds[2].n), 32, 0, st>>>(scenes_dev, n_scenes, kinds[2], sil_out,
                                                                        err);
            return cudaGetLastError();
        }
        // persistent warps in blocks of kBlock threads, whatever `block` is
        const size_t wsmem = (size_t)(kBlock / 32) * wsil::kWarpStack * sizeof(int2);
        static int wbps = 0, w_sm = 0;
        if (!wbps) {
            int dev = 0, b = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&w_sm, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch_silw<D>, kBlock, wsmem);
            wbps = b < 1 ? 1 : b;
        }
        const int64_t want = std::min<int64_t>((int64_t)wbps * w_sm, (kinds[2].n * 32 + kBlock - 1) / kBlock);
        k_batch_silw<D><<<dim3((unsigned)want), kBlock, wsmem, st>>>(scenes_dev, n_scenes, kinds[2], sil_out, counter,
                                                                     err);
        return cudaGetLastError();
    }
    const int mi = smem ? 1 : 0;
    const bool split = cp_mode == 2 || sil_mode == 3, sil = kinds[2].n > 0;
    const int si = (split ? 1 : 0) + (sil ? 2 : 0);
    const void *kern = split ? (sil ? (const void *)k_batch<D, RAYW, true, true>
                                    : (const void *)k_batch<D, RAYW, true, false>)
                             : (sil ? (const void *)k_batch<D, RAYW, false, true>
                                    : (const void *)k_batch<D, RAYW, false, false>);
    static int bps_m[2][2][4] = {}, n_sm = 0;
    if (!bps_m[bi][mi][si]) {
        int dev = 0, b = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, block, smem);
        bps_m[bi][mi][si] = b < 1 ? 1 : b;
    }
    const int bps = bps_m[bi][mi][si];
    const int64_t most = std::max(kinds[0].n, std::max(kinds[1].n, kinds[2].n));
    if (most <= 0) return cudaSuccess;
    int64_t want = std::min<int64_t>((int64_t)bps * n_sm,
                                     std::max<int64_t>((most + block - 1) / block, smem ? (kinds[2].n * 32 + block - 1) / block : 0));
    if (grid_share > 0.f && grid_share < 1.f)
        want = std::min<int64_t>(want, std::max<int64_t>(1, (int64_t)(grid_share * (float)(bps * n_sm))));
    void *args[] = {(void *)&scenes_dev, (void *)&n_scenes, (void *)&kinds[0], (void *)&cp_out,
                    (void *)&kinds[1],   (void *)&ray_out,  (void *)&kinds[2], (void *)&sil_out,
                    (void *)&cp_mode,    (void *)&sil_mode, (void *)&kBudget,  (void *)&counter,
                    (void *)&ho,         (void *)&err};
    cudaLaunchKernel(kern, dim3((unsigned)want), dim3((unsigned)block), args, smem, st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // the handed-over queries: persistent grids of one query per warp
    const size_t hsmem = (size_t)(block / 32) * wcp::kWarpStack * sizeof(int2);
    static int hbps[2][2] = {};
    if (!hbps[bi][0]) {
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_cp_heavy<D>, block, hsmem);
        hbps[bi][0] = b < 1 ? 1 : b;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_sil_heavy<D>, block, hsmem);
        hbps[bi][1] = b < 1 ? 1 : b;
    }
    auto hgrid = [&](int which, int64_t n) {
        const int hb = hbps[bi][which];
        int64_t g = std::min<int64_t>((int64_t)hb * n_sm, (n * 32 + block - 1) / block);
        if (grid_share > 0.f && grid_share < 1.f)
            g = std::min<int64_t>(g, std::max<int64_t>(1, (int64_t)(grid_share * (float)(hb * n_sm))));
        return dim3((unsigned)g);
    };
    if (cp_mode == 2 && kinds[0].n > 0) {
        k_cp_heavy<D><<<hgrid(0, kinds[0].n), block, hsmem, st>>>(scenes_dev, kinds[0], cp_out, ho.cp_q, ho.cp_r,
                                                                  counter);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (sil_mode == 3 && kinds[2].n > 0) {
        k_sil_heavy<D><<<hgrid(1, kinds[2].n), block, hsmem, st>>>(scenes_dev, kinds[2], sil_out, ho.sil_q,
                                                                   ho.sil_r, counter);
        e = cudaGetLastError();
    }
    return e;
}

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

size_t sort_temp_bytes(int64_t n) {
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, (const uint64_t *)nullptr, (uint64_t *)nullptr,
                                    (const int32_t *)nullptr, (int32_t *)nullptr, (int)std::max<int64_t>(n, 1), 0,
                                    64);
    return tb;
}

}  // namespace

size_t batch_scratch_bytes(int64_t max_n) {
    // per kind: keys in/out (8 B), values in (4 B), permutation (4 B), sort temp; plus counter
    const size_t per = 2 * align256((size_t)max_n * 8) + 2 * align256((size_t)max_n * 4) + align256(sort_temp_bytes(max_n));
    return 3 * per + 256;
}

cudaError_t batch_run(const DevScene *scenes_dev, int n_scenes, int dim, BatchKind kinds[3], const gq_cp_out &cp_out,
                      const gq_ray_out &ray_out, const gq_sil_out &sil_out, int ray_wide, int cp_mode,
                      int sil_mode, float grid_share, int block, bool sort, void *scratch, int64_t max_n,
                      int32_t *err, cudaStream_t st) {
    block = block == 32 ? 32 : kBlock;
    constexpr int kCounters = 7;  // claims per phase; closest points handed over, their claims; silhouettes the same
    char *p = static_cast<char *>(scratch);
    unsigned long long *counter = reinterpret_cast<unsigned long long *>(p);
    p += 256;
    int end_bit = 32;
    while ((1ll << (end_bit - 32)) < (long long)n_scenes + 1) ++end_bit;  // padding keys sort last
    const size_t tb = sort_temp_bytes(max_n);
    // closest points handed to k_cp_heavy: the cp kind's sort inputs, free after the sort
    Handover ho;
    for (int k = 0; k < 3; ++k) {
        BatchKind &q = kinds[k];
        uint64_t *k_in = reinterpret_cast<uint64_t *>(p);
        p += align256((size_t)max_n * 8);
        uint64_t *k_out = reinterpret_cast<uint64_t *>(p);
        p += align256((size_t)max_n * 8);
        int32_t *v_in = reinterpret_cast<int32_t *>(p);
        p += align256((size_t)max_n * 4);
        int32_t *perm = reinterpret_cast<int32_t *>(p);
        p += align256((size_t)max_n * 4);
        void *temp = p;
        p += align256(tb);
        q.perm = perm;
        if (k == 0) {
            ho.cp_q = v_in;
            ho.cp_r = reinterpret_cast<int2 *>(k_in);
        } else if (k == 2) {
            ho.sil_q = v_in;
            ho.sil_r = reinterpret_cast<int2 *>(k_in);
        }
        if (q.n <= 0 || !sort) continue;
        k_batch_keys<<<dim3((unsigned)((q.n + kBlock - 1) / kBlock)), kBlock, 0, st>>>(scenes_dev, n_scenes, q, q.n,
                                                                                        k_in, v_in, err);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        size_t tbk = tb;
        e = cub::DeviceRadixSort::SortPairs(temp, tbk, k_in, k_out, v_in, perm, (int)q.n, 0, end_bit, st);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = cudaSuccess;
    if (sort) {
        e = cudaMemsetAsync(counter, 0, kCounters * sizeof(unsigned long long), st);
    } else {
        // the identity order where the sort would have put its output (the hand-over
        // lists of the split modes live in the sort's inputs, not here)
        const int64_t most = std::max<int64_t>(kCounters, std::max(kinds[0].n, std::max(kinds[1].n, kinds[2].n)));
        k_batch_ident<<<dim3((unsigned)((most + block - 1) / block)), block, 0, st>>>(
            const_cast<int32_t *>(kinds[0].perm), std::max<int64_t>(kinds[0].n, 0), const_cast<int32_t *>(kinds[1].perm),
            std::max<int64_t>(kinds[1].n, 0), const_cast<int32_t *>(kinds[2].perm), std::max<int64_t>(kinds[2].n, 0),
            counter, kCounters);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return e;
    if (dim == 3)
        return ray_wide ? launch_batch<3, true>(scenes_dev, n_scenes, kinds, cp_out, ray_out, sil_out, cp_mode,
                                                sil_mode, grid_share, block, counter, ho, err, st)
                        : launch_batch<3, false>(scenes_dev, n_scenes, kinds, cp_out, ray_out, sil_out, cp_mode,
                                                 sil_mode, grid_share, block, counter, ho, err, st);
    return ray_wide ? launch_batch<2, true>(scenes_dev, n_scenes, kinds, cp_out, ray_out, sil_out, cp_mode,
                                            sil_mode, grid_share, block, counter, ho, err, st)
                    : launch_batch<2, false>(scenes_dev, n_scenes, kinds, cp_out, ray_out, sil_out, cp_mode,
                                             sil_mode, grid_share, block, counter, ho, err, st);
}

}  // namespace gqd
