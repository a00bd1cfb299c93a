// Many scenes, three query kinds, one persistent launch.
//
// Queries of each kind are sorted by (scene, Morton code inside the scene's box), then
// cut into tiles of 32.  Persistent warps take tiles from one counter in the order
// closest point, rays, silhouettes, so a warp always runs one query kind (a
// warp-uniform branch).  Closest-point tiles run the warp-coherent traversal once per
// distinct scene in the tile (tiles straddle at most a scene boundary or two); ray and
// silhouette tiles run one traversal per lane on the lane's own scene.  Every launch
// input lives in caller- or batch-owned device memory, so a step can be captured in a
// CUDA graph.
#include <cub/cub.cuh>

#include "batch.cuh"
#include "packet.cuh"
#include "records.cuh"
#include "snch.cuh"
#include "traverse.cuh"

namespace gqd {

namespace {

constexpr int kBlock = 128;

__device__ __forceinline__ float qget(const gq_vecs &v, int64_t i, int k) {
    return v.ptr[(int64_t)k * v.comp_stride + i * v.elem_stride];
}

__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
__device__ __forceinline__ uint32_t spread2(uint32_t v) {
    v &= 0x7fffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

// key = scene << 32 | Morton code over twice the scene's box
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
        code = (spread3(c[0]) << 2) | (spread3(c[1]) << 1) | spread3(c[2]);
    } else {
        uint32_t c[2];
        for (int a = 0; a < 2; ++a) {
            const float mid = 0.5f * (s.root_lo[a] + s.root_hi[a]);
            float ext = s.root_hi[a] - s.root_lo[a];
            if (!(ext > 0.f)) ext = 1.f;
            float f = (qget(k.a, i, a) - (mid - ext)) * (32768.f / (2.f * ext));
            c[a] = (uint32_t)fminf(fmaxf(f, 0.f), 32767.f);
        }
        code = (spread2(c[0]) << 1) | spread2(c[1]);
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

// Warp tiles of 32 sorted queries: closest-point tiles first, then rays, then silhouettes.
template <int D>
__global__ void __launch_bounds__(kBlock) k_batch(const DevScene *scenes, int n_scenes, BatchKind cp, gq_cp_out cp_out,
                                                  BatchKind ray, gq_ray_out ray_out, BatchKind sil,
                                                  gq_sil_out sil_out, int ray_wide, int cp_coherent,
                                                  unsigned long long *counter, int32_t *err) {
    const unsigned lane = threadIdx.x & 31u;
    const int64_t t_cp = (cp.n + 31) / 32, t_ray = (ray.n + 31) / 32, t_sil = (sil.n + 31) / 32;
    const int64_t tiles = t_cp + t_ray + t_sil;
    for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(counter, 1ull);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= (unsigned long long)tiles) break;
        int64_t tt = (int64_t)t;
        if (tt < t_cp) {
            // ---- closest point ----
            const int64_t i = tt * 32 + lane;
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
            if (cp_coherent) {
                int2 stk[pkt::kPStack];
                unsigned todo = __ballot_sync(0xffffffffu, alive);
                while (todo) {
                    const int s0 = __shfl_sync(0xffffffffu, sid, __ffs(todo) - 1);
                    const unsigned m = __ballot_sync(0xffffffffu, alive && sid == s0);
                    float r = kInf;
                    int idx = -1;
                    bool o = false;
                    pkt::closest_point<D, 0, false>(scenes[s0], m, p, r, idx, o, stk);
                    if ((m >> lane) & 1u) {
                        best_idx = idx;
                        ovf = o;
                    }
                    todo &= ~m;
                }
            } else if (alive) {
                trav::Stack<false> stk;
                trav::Lane<D, false, false> L;
                const gq_vecs none{};
                trav::lane_init(scenes[sid], L, cp.a, none, nullptr, qi);
                while (!trav::lane_run<D, false, false, 0>(scenes[sid], L, stk, 1 << 30)) {
                }
                best_idx = L.idx;
                ovf = L.ovf;
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
            continue;
        }
        tt -= t_cp;
        if (tt < t_ray) {
            // ---- rays: one traversal per lane ----
            const int64_t i = tt * 32 + lane;
            if (i < ray.n) {
                const int64_t qi = (int64_t)__ldg(ray.perm + i);
                const int sid = __ldg(ray.scene + qi);
                if (sid == GQ_BATCH_SKIP) {
                } else if ((unsigned)sid >= (unsigned)n_scenes) {
                    atomicOr(err, GQ_BATCH_ERR_SCENE);
                    if (D == 3)
                        ray3_record(nullptr, -1, false, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, ray_out, ray.n, qi);
                    else
                        ray2_record(nullptr, -1, false, 0.f, 0.f, 0.f, 0.f, 0.f, ray_out, ray.n, qi);
                } else {
                    const DevScene &s = scenes[sid];
                    if (ray_wide && s.wnodes) {
                        trav::Stack<true> stk;
                        trav::Lane<D, true, true> L;
                        trav::lane_init(s, L, ray.a, ray.b, ray.r_max, qi);
                        while (!trav::lane_run<D, true, true, 0>(s, L, stk, 1 << 30)) {
                        }
                        trav::lane_write(s, L, qi, ray.n, gq_cp_out{}, ray_out);
                    } else {
                        trav::Stack<false> stk;
                        trav::Lane<D, true, false> L;
                        trav::lane_init(s, L, ray.a, ray.b, ray.r_max, qi);
                        while (!trav::lane_run<D, true, false, 0>(s, L, stk, 1 << 30)) {
                        }
                        trav::lane_write(s, L, qi, ray.n, gq_cp_out{}, ray_out);
                    }
                }
            }
            continue;
        }
        tt -= t_ray;
        {
            // ---- silhouettes: one traversal per lane ----
            const int64_t i = tt * 32 + lane;
            if (i < sil.n) {
                const int64_t qi = (int64_t)__ldg(sil.perm + i);
                const int sid = __ldg(sil.scene + qi);
                if (sid == GQ_BATCH_SKIP) continue;
                float bp[D], bd = 0.f;
                int bid = 0;
                bool found = false, ovf = false;
                if ((unsigned)sid >= (unsigned)n_scenes) {
                    atomicOr(err, GQ_BATCH_ERR_SCENE);
                } else {
                    const DevScene &s = scenes[sid];
                    float x[D];
#pragma unroll
                    for (int k = 0; k < D; ++k) x[k] = qget(sil.a, qi, k);
                    const float r_max = sil.r_max ? sil.r_max[qi] : kInf;
                    if (s.spairs) {
                        snch::closest_silhouette<D>(s, x, r_max, found, bp, bd, bid, ovf);
                    } else {
                        atomicOr(err, GQ_BATCH_ERR_NO_SNCH);
                    }
                    if (ovf) {
                        if (s.err) atomicOr(s.err, GQ_DEVERR_STACK);
                        found = false;
                    }
                }
                put_sil<D>(sil_out, sil.n, qi, found, bp, bd, bid);
            }
        }
    }
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
                      const gq_ray_out &ray_out, const gq_sil_out &sil_out, int ray_wide, int cp_coherent,
                      void *scratch, int64_t max_n, int32_t *err, cudaStream_t st) {
    char *p = static_cast<char *>(scratch);
    unsigned long long *counter = reinterpret_cast<unsigned long long *>(p);
    p += 256;
    int end_bit = 32;
    while ((1ll << (end_bit - 32)) < (long long)n_scenes + 1) ++end_bit;  // padding keys sort last
    const size_t tb = sort_temp_bytes(max_n);
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
        if (q.n <= 0) continue;
        k_batch_keys<<<dim3((unsigned)((q.n + kBlock - 1) / kBlock)), kBlock, 0, st>>>(scenes_dev, n_scenes, q, q.n,
                                                                                        k_in, v_in, err);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        size_t tbk = tb;
        e = cub::DeviceRadixSort::SortPairs(temp, tbk, k_in, k_out, v_in, perm, (int)q.n, 0, end_bit, st);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    static int bps[2] = {0, 0}, n_sm = 0;
    const int di = dim == 3 ? 1 : 0;
    if (!bps[di]) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        if (dim == 3)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps[1], k_batch<3>, kBlock, 0);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps[0], k_batch<2>, kBlock, 0);
        if (bps[di] < 1) bps[di] = 1;
    }
    const int64_t tiles = (kinds[0].n + 31) / 32 + (kinds[1].n + 31) / 32 + (kinds[2].n + 31) / 32;
    if (tiles == 0) return cudaSuccess;
    const int64_t want = std::min<int64_t>((int64_t)bps[di] * n_sm, (tiles * 32 + kBlock - 1) / kBlock);
    if (dim == 3)
        k_batch<3><<<dim3((unsigned)want), kBlock, 0, st>>>(scenes_dev, n_scenes, kinds[0], cp_out, kinds[1], ray_out, kinds[2],
                                                            sil_out, ray_wide, cp_coherent, counter, err);
    else
        k_batch<2><<<dim3((unsigned)want), kBlock, 0, st>>>(scenes_dev, n_scenes, kinds[0], cp_out, kinds[1], ray_out, kinds[2],
                                                            sil_out, ray_wide, cp_coherent, counter, err);
    return cudaGetLastError();
}

}  // namespace gqd
