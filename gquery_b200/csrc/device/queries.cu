// Query kernels for sm_100a: the binary SNCH traversal (gQuery's visit order),
// brute-force scans and the reordering of queries along space-filling curves.  Closest-point and ray
// traversals live in traverse.cu.  Compiled with --fmad=false (see gq_fmath.h).
#include <cub/cub.cuh>

#include <algorithm>

#include "curves.cuh"
#include "prim.cuh"
#include "queries.cuh"
#include "records.cuh"
#include "sil_packet.cuh"
#include "sil_warp.cuh"
#include "snch.cuh"

namespace gqd {

namespace {

constexpr int kBlock = 128;
constexpr int kMaxBlock = 256;

__device__ __forceinline__ float qget(const gq_vecs &v, int64_t i, int k) {
    return v.ptr[(int64_t)k * v.comp_stride + i * v.elem_stride];
}

__device__ __forceinline__ void flag_error(int32_t *err, int bits) {
    if (err) atomicOr(err, bits);
}

__device__ __forceinline__ int64_t query_index(const int32_t *perm, int64_t i) {
    return perm ? (int64_t)__ldg(perm + i) : i;
}

// ===========================================================================
// Closest silhouette (SNCH), binary exact
// ===========================================================================

template <int D>
__device__ __forceinline__ void sil_write(const DevScene &s, const snch::Lane<D> &L, int64_t qi, int64_t n,
                                          const gq_sil_out &o) {
    const bool found = L.found && !L.ovf;
    if (L.ovf) flag_error(s.err, GQ_DEVERR_STACK);
    if (o.valid) o.valid[qi] = found ? 1 : 0;
    if (o.p) {
#pragma unroll
        for (int k = 0; k < D; ++k) o.p[k * n + qi] = found ? L.bp[k] : 0.f;
    }
    put1(o.d, qi, found ? L.bd : 0.f);
    if (o.prim_id) o.prim_id[qi] = found ? L.bid : 0;
}

// Warp-coherent closest silhouette (sil_packet.cuh): persistent warps take 32
// consecutive queries of the sorted order at a time.
template <int D>
__global__ void __launch_bounds__(kMaxBlock, 4) k_sil_packet(DevScene s, gq_vecs xq, const float *rmax_in, int64_t n,
                                                       const int32_t *perm, gq_sil_out o, unsigned long long *counter) {
    const unsigned lane = threadIdx.x & 31u;
    snch::Stack stk;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(counter, 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= (unsigned long long)n) break;
        const int64_t i = (int64_t)base + lane;
        const bool alive = i < n;
        const int64_t qi = alive ? query_index(perm, i) : 0;
        snch::Lane<D> L;
#pragma unroll
        for (int k = 0; k < D; ++k) L.x[k] = alive ? qget(xq, qi, k) : 0.f;
        L.r = alive ? (rmax_in ? rmax_in[qi] : kInf) : -1.f;
        pkt::closest_silhouette<D>(s, __ballot_sync(0xffffffffu, alive), L, stk);
        if (alive) sil_write<D>(s, L, qi, n, o);
    }
}

// One query per warp (sil_warp.cuh): persistent warps take the next query of the
// sorted order; the stack lives in dynamic shared memory (kWarpStack entries per warp).
template <int D>
__global__ void __launch_bounds__(kMaxBlock, 4) k_sil_warp(DevScene s, gq_vecs xq, const float *rmax_in, int64_t n,
                                                     const int32_t *perm, gq_sil_out o, unsigned long long *counter) {
    extern __shared__ int2 wstk[];
    const unsigned lane = threadIdx.x & 31u;
    int2 *stk = wstk + (threadIdx.x >> 5) * wsil::kWarpStack;
    for (;;) {
        unsigned long long i = 0;
        if (lane == 0) i = atomicAdd(counter, 1ull);
        i = __shfl_sync(0xffffffffu, i, 0);
        if (i >= (unsigned long long)n) break;
        const int64_t qi = query_index(perm, (int64_t)i);
        float x[D];
#pragma unroll
        for (int k = 0; k < D; ++k) x[k] = qget(xq, qi, k);
        snch::Lane<D> L;
        wsil::closest_silhouette<D>(s, x, rmax_in ? rmax_in[qi] : kInf, L, stk);
        if (lane == 0) sil_write<D>(s, L, qi, n, o);
    }
}

template <int D>
__device__ __forceinline__ void sil_start(const DevScene &s, snch::Lane<D> &L, int2 *stk, gq_vecs xq,
                                          const float *rmax_in, int64_t qi) {
    float x[D];
#pragma unroll
    for (int k = 0; k < D; ++k) x[k] = qget(xq, qi, k);
    snch::lane_init<D>(s, L, x, rmax_in ? rmax_in[qi] : kInf, stk);
}

// One query per thread: SNCH.closest_silhouette (snch.py:106-164) and
// SNCH3D.closest_silhouette (snch3d.py:143-203).
template <int D>
__global__ void __launch_bounds__(kBlock) k_sil_exact(DevScene s, gq_vecs xq, const float *rmax_in, int64_t n,
                                                      const int32_t *perm, gq_sil_out o) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t qi = query_index(perm, i);
    snch::Stack stk;
    snch::Lane<D> L;
    sil_start<D>(s, L, stk, xq, rmax_in, qi);
    while (!snch::lane_run<D>(s, L, stk, 1 << 30)) {
    }
    sil_write<D>(s, L, qi, n, o);
}

// Persistent warps with lane refill: a lane whose query is done takes the next one
// (warp-aggregated atomic on a per-call counter), so a warp never waits for its
// slowest query.  Same visit order and answers as k_sil_exact.
template <int D>
__global__ void __launch_bounds__(kMaxBlock) k_sil_persist(DevScene s, gq_vecs xq, const float *rmax_in, int64_t n,
                                                        const int32_t *perm, gq_sil_out o,
                                                        unsigned long long *counter, int budget) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    snch::Stack stk;
    snch::Lane<D> L;
    int64_t qi = -1;
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
                    if (mine < (unsigned long long)n) {
                        qi = query_index(perm, (int64_t)mine);
                        sil_start<D>(s, L, stk, xq, rmax_in, qi);
                        live = true;
                    }
                }
            }
        }
        if (!__any_sync(0xffffffffu, live)) break;
        if (live && snch::lane_run<D>(s, L, stk, budget)) {
            sil_write<D>(s, L, qi, n, o);
            live = false;
        }
    }
}

// ===========================================================================
// Brute force (closest_point_baseline / intersect_baseline), FP32
// ===========================================================================

template <int D>
__device__ __forceinline__ void vtx(const DevScene &s, int64_t prim, int k, float *out) {
    const int64_t vi = __ldg(s.index + prim * D + k);
#pragma unroll
    for (int c = 0; c < D; ++c) out[c] = __ldg(s.verts + vi * D + c);
}

// polyline.py:176-209 and mesh.py closest_point_baseline
template <int D>
__global__ void __launch_bounds__(kBlock) k_cp_brute(DevScene s, gq_vecs q, int64_t n, gq_cp_out o) {
    const int64_t qi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (qi >= n) return;
    float p[D];
#pragma unroll
    for (int k = 0; k < D; ++k) p[k] = qget(q, qi, k);
    float d_min = kInf;
    int64_t idx = -1;
    for (int64_t f = 0; f < s.n_prims; ++f) {
        float a[D], b[D];
        vtx<D>(s, f, 0, a);
        vtx<D>(s, f, 1, b);
        float d;
        if (D == 2) {
            const float pax = p[0] - a[0], pay = p[D - 1] - a[D - 1];
            const float bax = b[0] - a[0], bay = b[D - 1] - a[D - 1];
            const float h = gq_clamp(gq_div(gq_dot2(pax, pay, bax, bay), gq_dot2(bax, bay, bax, bay)), 0.f, 1.f);
            d = gq_norm2(pax - bax * h, pay - bay * h);
        } else {
            float c[D];
            vtx<D>(s, f, D - 1, c);
            d = tri_closest<false>(p[0], p[1], p[D - 1], a[0], a[1], a[D - 1], b[0], b[1], b[D - 1], c[0], c[1],
                                   c[D - 1]);
        }
        if (d < d_min) {
            d_min = d;
            idx = f;
        }
    }
    const bool ok = idx != -1;
    float rp[3] = {0.f, 0.f, 0.f}, rn[3] = {0.f, 0.f, 0.f}, t0 = 0.f, t1 = 0.f;
    if (ok) {
        float a[D], b[D];
        vtx<D>(s, idx, 0, a);
        vtx<D>(s, idx, 1, b);
        if (D == 2) {
            const float pax = p[0] - a[0], pay = p[D - 1] - a[D - 1];
            const float bax = b[0] - a[0], bay = b[D - 1] - a[D - 1];
            const float h = gq_clamp(gq_div(gq_dot2(pax, pay, bax, bay), gq_dot2(bax, bay, bax, bay)), 0.f, 1.f);
            const float inv = gq_rsqrt(gq_dot2(bay, -bax, bay, -bax));
            rn[0] = bay * inv;
            rn[1] = -bax * inv;
            rp[0] = gq_lerp(a[0], b[0], h);
            rp[1] = gq_lerp(a[D - 1], b[D - 1], h);
            t0 = h;
        } else {
            float c[D];
            vtx<D>(s, idx, D - 1, c);
            tri_closest<true>(p[0], p[1], p[D - 1], a[0], a[1], a[D - 1], b[0], b[1], b[D - 1], c[0], c[1], c[D - 1],
                              rp, &t0, &t1);
            float cx, cy, cz;
            cross3(b[0] - a[0], b[1] - a[1], b[D - 1] - a[D - 1], c[0] - a[0], c[1] - a[1], c[D - 1] - a[D - 1], cx,
                   cy, cz);
            const float inv = gq_rsqrt(gq_dot3(cx, cy, cz, cx, cy, cz));
            rn[0] = cx * inv;
            rn[1] = cy * inv;
            rn[2] = cz * inv;
        }
    }
    if (o.valid) o.valid[qi] = ok ? 1 : 0;
    if (o.p)
        for (int k = 0; k < D; ++k) o.p[k * n + qi] = rp[k];
    if (o.n)
        for (int k = 0; k < D; ++k) o.n[k * n + qi] = rn[k];
    if (D == 2)
        put1(o.t, qi, t0);
    else
        put2(o.t, n, qi, t0, t1);
    put1(o.d, qi, ok ? d_min : 0.f);
    if (o.prim_id) o.prim_id[qi] = ok ? (int)idx : 0;
}

// polyline.py:138-169 and mesh.py intersect_baseline
template <int D>
__global__ void __launch_bounds__(kBlock) k_ray_brute(DevScene s, gq_vecs x, gq_vecs v, const float *rmax_in,
                                                       int64_t n, gq_ray_out o) {
    const int64_t qi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (qi >= n) return;
    float xo[D], vd[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        xo[k] = qget(x, qi, k);
        vd[k] = qget(v, qi, k);
    }
    const float r_max = rmax_in ? rmax_in[qi] : kInf;
    float d_min = r_max;
    int64_t idx = -1;
    for (int64_t f = 0; f < s.n_prims; ++f) {
        float a[D], b[D];
        vtx<D>(s, f, 0, a);
        vtx<D>(s, f, 1, b);
        if (D == 2) {
            const float d = seg_ray(xo[0], xo[D - 1], vd[0], vd[D - 1], a[0], a[D - 1], b[0], b[D - 1]);
            if (d < d_min) {
                d_min = d;
                idx = f;
            }
        } else {
            float c[D];
            vtx<D>(s, f, D - 1, c);
            float vv = __builtin_nanf(""), ww;
            const float t = tri_ray(xo[0], xo[1], xo[D - 1], vd[0], vd[1], vd[D - 1], a[0], a[1], a[D - 1], b[0],
                                    b[1], b[D - 1], c[0], c[1], c[D - 1], r_max, &vv, &ww);
            if ((vv == vv) && (t < d_min)) {
                idx = f;
                d_min = t;
            }
        }
    }
    bool ok = idx != -1;
    float rp[3] = {0.f, 0.f, 0.f}, rn[3] = {0.f, 0.f, 0.f}, t0 = 0.f, t1 = 0.f, dd = 0.f;
    if (ok) {
        float a[D], b[D];
        vtx<D>(s, idx, 0, a);
        vtx<D>(s, idx, 1, b);
        if (D == 2) {
            const float bx = b[0] - a[0], by = b[D - 1] - a[D - 1];
            const float inv = gq_rsqrt(gq_dot2(bx, by, bx, by));
            const float abx = bx * inv, aby = by * inv;
            rn[0] = aby;
            rn[1] = -abx;
            rp[0] = xo[0] + vd[0] * d_min;
            rp[1] = xo[D - 1] + vd[D - 1] * d_min;
            t0 = -1.f;
            dd = d_min;
        } else {
            float c[D];
            vtx<D>(s, idx, D - 1, c);
            float vv = __builtin_nanf(""), ww = 0.f;
            const float t = tri_ray(xo[0], xo[1], xo[D - 1], vd[0], vd[1], vd[D - 1], a[0], a[1], a[D - 1], b[0], b[1],
                                    b[D - 1], c[0], c[1], c[D - 1], r_max, &vv, &ww);
            ok = vv == vv;
            if (ok) {
                const float v1x = b[0] - a[0], v1y = b[1] - a[1], v1z = b[D - 1] - a[D - 1];
                const float v2x = c[0] - a[0], v2y = c[1] - a[1], v2z = c[D - 1] - a[D - 1];
                rp[0] = (a[0] + v1x * vv) + v2x * ww;
                rp[1] = (a[1] + v1y * vv) + v2y * ww;
                rp[2] = (a[D - 1] + v1z * vv) + v2z * ww;
                float cx, cy, cz;
                cross3(v1x, v1y, v1z, v2x, v2y, v2z, cx, cy, cz);
                const float inv = gq_rsqrt(gq_dot3(cx, cy, cz, cx, cy, cz));
                rn[0] = cx * inv;
                rn[1] = cy * inv;
                rn[2] = cz * inv;
                t0 = 1.f - vv - ww;
                t1 = vv;
                dd = t;
            }
        }
    }
    if (o.valid) o.valid[qi] = ok ? 1 : 0;
    if (o.p)
        for (int k = 0; k < D; ++k) o.p[k * n + qi] = ok ? rp[k] : 0.f;
    if (o.n)
        for (int k = 0; k < D; ++k) o.n[k * n + qi] = ok ? rn[k] : 0.f;
    if (D == 2)
        put1(o.t, qi, ok ? t0 : 0.f);
    else
        put2(o.t, n, qi, ok ? t0 : 0.f, ok ? t1 : 0.f);
    put1(o.d, qi, ok ? dd : 0.f);
    if (o.prim_id) o.prim_id[qi] = ok ? (int)idx : 0;
    if (o.on_boundary) o.on_boundary[qi] = ok ? 1 : 0;
}

// ===========================================================================
// closest_silhouette_baseline (mesh.py:124-135, polyline.py:212-223): every query
// tests the scene's silhouette list in order and keeps the first strictly nearest
// silhouette (the same per-silhouette test and acceptance as the SNCH traversal, so
// snch::test_silhouette does it; s.sils points at the baseline list here).
template <int D>
__global__ void __launch_bounds__(kBlock) k_sil_brute(DevScene s, int64_t n_sil, gq_vecs x, const float *rmax_in,
                                                      int64_t n, gq_sil_out o) {
    const int64_t qi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (qi >= n) return;
    snch::Lane<D> L;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        L.x[k] = qget(x, qi, k);
        L.bp[k] = 0.f;
    }
    L.r = rmax_in ? rmax_in[qi] : kInf;
    L.found = false;
    L.ovf = false;
    L.bd = 0.f;
    L.bid = 0;
    for (int64_t j = 0; j < n_sil; ++j) snch::test_silhouette<D>(s, L, (int)j);
    sil_write<D>(s, L, qi, n, o);
}

// FP64 brute force (error reference).  Primitives are staged through shared
// memory in tiles; one thread per query.
// ===========================================================================

constexpr int kTile = 256;

__device__ double d_cp_tri(const double *p, const double *a, const double *b, const double *c) {
    double ab[3], ac[3], ap[3], bp[3], cp[3];
    for (int k = 0; k < 3; ++k) {
        ab[k] = b[k] - a[k];
        ac[k] = c[k] - a[k];
        ap[k] = p[k] - a[k];
        bp[k] = p[k] - b[k];
        cp[k] = p[k] - c[k];
    }
    auto dot = [](const double *u, const double *v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; };
    auto dist = [&](double x, double y, double z) {
        const double ex = p[0] - x, ey = p[1] - y, ez = p[2] - z;
        return sqrt(ex * ex + ey * ey + ez * ez);
    };
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0 && d2 <= 0) return dist(a[0], a[1], a[2]);
    const double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0 && d4 <= d3) return dist(b[0], b[1], b[2]);
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) {
        const double v = d1 / (d1 - d3);
        return dist(a[0] + v * ab[0], a[1] + v * ab[1], a[2] + v * ab[2]);
    }
    const double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0 && d5 <= d6) return dist(c[0], c[1], c[2]);
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) {
        const double w = d2 / (d2 - d6);
        return dist(a[0] + w * ac[0], a[1] + w * ac[1], a[2] + w * ac[2]);
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        return dist(b[0] + w * (c[0] - b[0]), b[1] + w * (c[1] - b[1]), b[2] + w * (c[2] - b[2]));
    }
    const double den = 1.0 / (va + vb + vc);
    const double v = vb * den, w = vc * den;
    return dist(a[0] + ab[0] * v + ac[0] * w, a[1] + ab[1] * v + ac[1] * w, a[2] + ab[2] * v + ac[2] * w);
}

__device__ double d_ray_tri(const double *o, const double *d, const double *a, const double *b, const double *c) {
    double e1[3], e2[3], s[3];
    for (int k = 0; k < 3; ++k) {
        e1[k] = b[k] - a[k];
        e2[k] = c[k] - a[k];
        s[k] = o[k] - a[k];
    }
    const double p[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
    const double det = e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2];
    if (det == 0.0) return INFINITY;
    const double inv = 1.0 / det;
    const double u = (s[0] * p[0] + s[1] * p[1] + s[2] * p[2]) * inv;
    if (u < 0 || u > 1) return INFINITY;
    const double q[3] = {s[1] * e1[2] - s[2] * e1[1], s[2] * e1[0] - s[0] * e1[2], s[0] * e1[1] - s[1] * e1[0]};
    const double v = (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]) * inv;
    if (v < 0 || u + v > 1) return INFINITY;
    const double t = (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) * inv;
    return t >= 0 ? t : INFINITY;
}

template <int D>
__global__ void __launch_bounds__(kBlock) k_brute_f64(DevScene s, int kind, gq_vecs qa, gq_vecs qb, int64_t n,
                                                       double *out_d, int32_t *out_id) {
    __shared__ double tile[kTile][D * D];
    const int64_t qi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool active = qi < n;
    double a[D] = {}, b[D] = {};
    if (active)
        for (int k = 0; k < D; ++k) {
            a[k] = qget(qa, qi, k);
            if (kind == 1) b[k] = qget(qb, qi, k);
        }
    double best = INFINITY;
    int64_t bid = -1;
    for (int64_t base = 0; base < s.n_prims; base += kTile) {
        __syncthreads();
        for (int t = threadIdx.x; t < kTile; t += blockDim.x) {
            const int64_t f = base + t;
            if (f < s.n_prims)
                for (int k = 0; k < D; ++k) {
                    const int64_t vi = s.index[f * D + k];
                    for (int c = 0; c < D; ++c) tile[t][k * D + c] = (double)s.verts[vi * D + c];
                }
        }
        __syncthreads();
        const int lim = (int)min((int64_t)kTile, s.n_prims - base);
        if (active)
            for (int t = 0; t < lim; ++t) {
                double d;
                const double *pv = tile[t];
                if (D == 3) {
                    d = (kind == 0) ? d_cp_tri(a, pv, pv + 3, pv + 6) : d_ray_tri(a, b, pv, pv + 3, pv + 6);
                } else if (kind == 0) {
                    const double ux = pv[2] - pv[0], uy = pv[3] - pv[1], vx = a[0] - pv[0], vy = a[D - 1] - pv[1];
                    const double uu = ux * ux + uy * uy;
                    double tt = uu > 0 ? (vx * ux + vy * uy) / uu : 0.0;
                    tt = tt < 0 ? 0 : (tt > 1 ? 1 : tt);
                    const double ex = pv[0] + tt * ux - a[0], ey = pv[1] + tt * uy - a[D - 1];
                    d = sqrt(ex * ex + ey * ey);
                } else {
                    const double ux = pv[2] - pv[0], uy = pv[3] - pv[1], wx = a[0] - pv[0], wy = a[D - 1] - pv[1];
                    const double den = b[0] * uy - b[D - 1] * ux;
                    const double ss = (b[0] * wy - b[D - 1] * wx) / den, tt = (ux * wy - uy * wx) / den;
                    d = (den != 0.0 && tt > 0 && ss >= 0 && ss <= 1) ? tt : INFINITY;
                }
                if (d < best) {
                    best = d;
                    bid = base + t;
                }
            }
    }
    if (active) {
        out_d[qi] = best;
        out_id[qi] = (int32_t)bid;
    }
}

// FP64 nearest silhouette over the scene's raw silhouette list (the reference's
// SNCH list: one record per polyline vertex, one per unique mesh edge), the records as
// float positions: 2D a, b, c, flag (8 floats; flag 1 = both neighbours exist,
// silhouette_vertex.py:48), 3D a, b, c, d, flag (16 floats; flag 1 = boundary edge,
// always a silhouette, silhouette_edge.py:56-57).  The silhouette conditions of
// silhouette_vertex.py:27-28 and silhouette_edge.py:7-12 in double: the face normals
// are left unnormalised (the sign test does not depend on their length).  The first
// strictly nearest silhouette in list order is kept.
template <int D>
__global__ void __launch_bounds__(kBlock) k_sil_f64(const float *recs, int64_t n_sil, gq_vecs qx, int64_t n,
                                                    double *out_d, int32_t *out_id) {
    constexpr int W = (D == 3) ? 16 : 8;
    __shared__ double tile[kTile][W];
    const int64_t qi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool active = qi < n;
    double x[D] = {};
    if (active)
        for (int k = 0; k < D; ++k) x[k] = qget(qx, qi, k);
    double best = INFINITY;
    int64_t bid = -1;
    for (int64_t base = 0; base < n_sil; base += kTile) {
        __syncthreads();
        for (int t = threadIdx.x; t < kTile * W; t += blockDim.x) {
            const int64_t f = base + t / W;
            tile[t / W][t % W] = f < n_sil ? (double)recs[base * W + t] : 0.0;
        }
        __syncthreads();
        const int lim = (int)min((int64_t)kTile, n_sil - base);
        if (!active) continue;
        for (int t = 0; t < lim; ++t) {
            const double *r = tile[t];
            double d;
            bool sil;
            if (D == 3) {
                const double ux = r[3] - r[0], uy = r[4] - r[1], uz = r[5] - r[2];
                const double uu = ux * ux + uy * uy + uz * uz;
                double tt = uu > 0 ? ((x[0] - r[0]) * ux + (x[1] - r[1]) * uy + (x[D - 1] - r[2]) * uz) / uu : 0.0;
                tt = tt < 0 ? 0 : (tt > 1 ? 1 : tt);
                const double wx = r[0] + tt * ux - x[0], wy = r[1] + tt * uy - x[1], wz = r[2] + tt * uz - x[D - 1];
                d = sqrt(wx * wx + wy * wy + wz * wz);
                if (!(d < best)) continue;
                // n0 = (b - a) x (c - a), n1 = (d - a) x (b - a)
                const double cx = r[6] - r[0], cy = r[7] - r[1], cz = r[8] - r[2];
                const double ex = r[9] - r[0], ey = r[10] - r[1], ez = r[11] - r[2];
                const double n0x = uy * cz - uz * cy, n0y = uz * cx - ux * cz, n0z = ux * cy - uy * cx;
                const double n1x = ey * uz - ez * uy, n1y = ez * ux - ex * uz, n1z = ex * uy - ey * ux;
                sil = (r[12] != 0.0) ||
                      ((wx * n0x + wy * n0y + wz * n0z) * (wx * n1x + wy * n1y + wz * n1z) < 0.0);
            } else {
                const double bx = r[2] - x[0], by = r[3] - x[D - 1];
                d = sqrt(bx * bx + by * by);
                if (!(d < best) || r[6] == 0.0) continue;
                // cross(b - a, x - a) * cross(c - b, x - b) < 0
                const double c0 = (r[2] - r[0]) * (x[D - 1] - r[1]) - (r[3] - r[1]) * (x[0] - r[0]);
                const double c1 = (r[4] - r[2]) * (x[D - 1] - r[3]) - (r[5] - r[3]) * (x[0] - r[2]);
                sil = c0 * c1 < 0.0;
            }
            if (sil) {
                best = d;
                bid = base + t;
            }
        }
    }
    if (active) {
        out_d[qi] = best;
        out_id[qi] = (int32_t)bid;
    }
}

// ===========================================================================
// Reordering along a space-filling curve
// ===========================================================================

// Keys on a grid over the scene box grown to twice its extent about its centre: the
// cell's index along a Hilbert curve (1024 cells per axis in 3D, 32768 in 2D).
__global__ void k_point_keys(int dim, float lo0, float lo1, float lo2, float sc0, float sc1, float sc2, gq_vecs q,
                              int64_t n, uint32_t *keys, int32_t *vals) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float lo[3] = {lo0, lo1, lo2}, sc[3] = {sc0, sc1, sc2};
    uint32_t key;
    if (dim == 3) {
        uint32_t c[3];
        for (int k = 0; k < 3; ++k) {
            float f = (qget(q, i, k) - lo[k]) * sc[k];
            f = fminf(fmaxf(f, 0.f), 1023.f);
            c[k] = (uint32_t)f;
        }
        key = hilbert3(c[0], c[1], c[2]);
    } else {
        uint32_t c[2];
        for (int k = 0; k < 2; ++k) {
            float f = (qget(q, i, k) - lo[k]) * sc[k];
            f = fminf(fmaxf(f, 0.f), 32767.f);
            c[k] = (uint32_t)f;
        }
        key = hilbert2(c[0], c[1]);
    }
    keys[i] = key;
    vals[i] = (int32_t)i;
}

// Ray keys: the origin's cell on the same grid as k_point_keys and the direction.
// mode 1: the direction's octant (3 bits) above a 27-bit Morton code of the origin
//         (9 bits per axis): each warp of sorted rays shares an octant and a region.
// mode 2: the origin (6 bits per axis) and the direction's octahedral coordinates
//         (6 bits each) interleaved coarse to fine, 30 bits.
__device__ __forceinline__ uint32_t spread5(uint32_t v) {  // 6 bits -> every fifth bit
    uint32_t r = 0;
#pragma unroll
    for (int b = 0; b < 6; ++b) r |= ((v >> b) & 1u) << (5 * b);
    return r;
}

__global__ void k_ray_keys(int mode, float lo0, float lo1, float lo2, float sc0, float sc1, float sc2, gq_vecs o,
                           gq_vecs d, int64_t n, uint32_t *keys, int32_t *vals) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float lo[3] = {lo0, lo1, lo2}, sc[3] = {sc0, sc1, sc2};
    float dir[3];
    uint32_t c[3];
    for (int k = 0; k < 3; ++k) {
        float f = (qget(o, i, k) - lo[k]) * sc[k];  // 0 .. 1024 over the grid
        f = fminf(fmaxf(f, 0.f), 1023.f);
        c[k] = (uint32_t)f;
        dir[k] = qget(d, i, k);
    }
    uint32_t key;
    if (mode == 1) {
        const uint32_t oct = (dir[0] < 0.f ? 4u : 0u) | (dir[1] < 0.f ? 2u : 0u) | (dir[2] < 0.f ? 1u : 0u);
        key = (oct << 27) | (spread3(c[0] >> 1) << 2) | (spread3(c[1] >> 1) << 1) | spread3(c[2] >> 1);
    } else {
        // octahedral map of the direction onto [-1, 1]^2
        const float l1 = fabsf(dir[0]) + fabsf(dir[1]) + fabsf(dir[2]);
        float u = l1 > 0.f ? dir[0] / l1 : 0.f, v = l1 > 0.f ? dir[1] / l1 : 0.f;
        if (dir[2] < 0.f) {
            const float uu = (1.f - fabsf(v)) * (u < 0.f ? -1.f : 1.f);
            v = (1.f - fabsf(u)) * (v < 0.f ? -1.f : 1.f);
            u = uu;
        }
        const uint32_t qu = (uint32_t)fminf(fmaxf((u + 1.f) * 32.f, 0.f), 63.f);
        const uint32_t qv = (uint32_t)fminf(fmaxf((v + 1.f) * 32.f, 0.f), 63.f);
        key = (spread5(c[0] >> 4) << 4) | (spread5(c[1] >> 4) << 3) | (spread5(c[2] >> 4) << 2) | (spread5(qu) << 1) |
              spread5(qv);
    }
    keys[i] = key;
    vals[i] = (int32_t)i;
}

// Bandwidth probe: every thread reads its 16-byte words of the buffer `reps` times
// with loads that are cached in L2 only, folding them into one word so that the loads
// cannot be dropped; one word per warp goes to `sink`.
__global__ void __launch_bounds__(256) k_read_probe(const uint4 *buf, int64_t n16, int reps, unsigned *sink) {
    unsigned acc = 0;
    const int64_t step = (int64_t)gridDim.x * blockDim.x;
    for (int r = 0; r < reps; ++r)
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n16; i += step) {
            const uint4 v = __ldcg(buf + i);
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    acc = __reduce_xor_sync(0xffffffffu, acc);
    if ((threadIdx.x & 31u) == 0) atomicXor(sink, acc);
}

inline dim3 grid_for(int64_t n) { return dim3((unsigned)((n + kBlock - 1) / kBlock)); }
inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

size_t cub_temp_bytes(int64_t n) {
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                    (const int32_t *)nullptr, (int32_t *)nullptr, (int)n, 0, 32);
    return tb;
}

}  // namespace

size_t morton_scratch_bytes(int64_t n) {
    return 3 * align256((size_t)n * 4) + align256(cub_temp_bytes(n));
}

cudaError_t morton_order(const DevScene &s, gq_vecs q, int64_t n, int32_t *perm, void *scratch, size_t scratch_bytes,
                         cudaStream_t st, int ray_mode, gq_vecs ray_dir) {
    if (n <= 0) return cudaSuccess;
    if (scratch_bytes < morton_scratch_bytes(n)) return cudaErrorInvalidValue;
    char *p = (char *)scratch;
    uint32_t *k_in = (uint32_t *)p;
    p += align256((size_t)n * 4);
    uint32_t *k_out = (uint32_t *)p;
    p += align256((size_t)n * 4);
    int32_t *v_in = (int32_t *)p;
    p += align256((size_t)n * 4);
    size_t tb = cub_temp_bytes(n);
    float lo[3] = {0, 0, 0}, sc[3] = {1, 1, 1};
    const int bits = s.dim == 3 ? 1024 : 32768;
    for (int k = 0; k < s.dim; ++k) {
        const float c = 0.5f * (s.root_lo[k] + s.root_hi[k]);
        float ext = s.root_hi[k] - s.root_lo[k];
        if (!(ext > 0.f)) ext = 1.f;
        lo[k] = c - ext;
        sc[k] = (float)bits / (2.f * ext);
    }
    if (ray_mode > 0 && s.dim == 3)
        k_ray_keys<<<grid_for(n), kBlock, 0, st>>>(ray_mode, lo[0], lo[1], lo[2], sc[0], sc[1], sc[2], q, ray_dir, n,
                                                   k_in, v_in);
    else
        k_point_keys<<<grid_for(n), kBlock, 0, st>>>(s.dim, lo[0], lo[1], lo[2], sc[0], sc[1], sc[2], q, n, k_in,
                                                      v_in);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int end_bit = 30;
    return cub::DeviceRadixSort::SortPairs(p, tb, k_in, k_out, v_in, perm, (int)n, 0, end_bit, st);
}

cudaError_t launch_sil(const DevScene &s, int variant, const Tune &t, gq_vecs x, const float *r_max, int64_t n,
                       const int32_t *perm, const gq_sil_out &o, unsigned long long *counter, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    static int bps[2][2][3] = {}, n_sm = 0;
    const int di = s.dim == 3 ? 1 : 0;
    int slot = block_slot(t.block), block = t.block;
    if (slot < 0) slot = 1, block = 128;
    if (variant == GQ_VARIANT_WARP && counter) {
        const size_t smem = (size_t)(block / 32) * wsil::kWarpStack * sizeof(int2);
        using Fn = void (*)(DevScene, gq_vecs, const float *, int64_t, const int32_t *, gq_sil_out,
                            unsigned long long *);
        const Fn fn = s.dim == 3 ? k_sil_warp<3> : k_sil_warp<2>;
        static int wb[2][3] = {}, w_sm = 0;
        if (!wb[di][slot]) {
            int dev = 0, b = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&w_sm, cudaDevAttrMultiProcessorCount, dev);
            // up to 8 warps x 4 KB of stacks (the opt-in keeps larger stacks possible)
            const int most = (kMaxBlock / 32) * wsil::kWarpStack * (int)sizeof(int2);
            cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (const void *)fn, block, smem);
            wb[di][slot] = b < 1 ? 1 : b;
        }
        const int64_t want = std::min<int64_t>((int64_t)wb[di][slot] * w_sm, (n * 32 + block - 1) / block);
        cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
        if (e != cudaSuccess) return e;
        fn<<<dim3((unsigned)want), block, smem, st>>>(s, x, r_max, n, perm, o, counter);
        return cudaGetLastError();
    }
    const bool packet = variant == GQ_VARIANT_COHERENT && counter && n >= 32;
    const bool refill = !packet && t.persist && counter && n > 4096;
    if (packet || refill) {
        const int ki = packet ? 1 : 0;
        if (!bps[ki][di][slot]) {
            int dev = 0, b = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
            const void *fn = packet ? (s.dim == 3 ? (const void *)k_sil_packet<3> : (const void *)k_sil_packet<2>)
                                    : (s.dim == 3 ? (const void *)k_sil_persist<3> : (const void *)k_sil_persist<2>);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, block, 0);
            bps[ki][di][slot] = b < 1 ? 1 : b;
        }
        const int64_t want = std::min<int64_t>((int64_t)bps[ki][di][slot] * n_sm, (n + block - 1) / block);
        cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
        if (e != cudaSuccess) return e;
        const dim3 grid((unsigned)want);
        if (packet) {
            if (s.dim == 3)
                k_sil_packet<3><<<grid, block, 0, st>>>(s, x, r_max, n, perm, o, counter);
            else
                k_sil_packet<2><<<grid, block, 0, st>>>(s, x, r_max, n, perm, o, counter);
        } else {
            const int b = t.budget > 0 ? t.budget : 32;
            if (s.dim == 3)
                k_sil_persist<3><<<grid, block, 0, st>>>(s, x, r_max, n, perm, o, counter, b);
            else
                k_sil_persist<2><<<grid, block, 0, st>>>(s, x, r_max, n, perm, o, counter, b);
        }
        return cudaGetLastError();
    }
    if (s.dim == 3)
        k_sil_exact<3><<<grid_for(n), kBlock, 0, st>>>(s, x, r_max, n, perm, o);
    else
        k_sil_exact<2><<<grid_for(n), kBlock, 0, st>>>(s, x, r_max, n, perm, o);
    return cudaGetLastError();
}

cudaError_t launch_cp_brute(const DevScene &s, gq_vecs q, int64_t n, const gq_cp_out &o, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (s.dim == 3)
        k_cp_brute<3><<<grid_for(n), kBlock, 0, st>>>(s, q, n, o);
    else
        k_cp_brute<2><<<grid_for(n), kBlock, 0, st>>>(s, q, n, o);
    return cudaGetLastError();
}

cudaError_t launch_ray_brute(const DevScene &s, gq_vecs x, gq_vecs v, const float *r_max, int64_t n,
                             const gq_ray_out &o, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (s.dim == 3)
        k_ray_brute<3><<<grid_for(n), kBlock, 0, st>>>(s, x, v, r_max, n, o);
    else
        k_ray_brute<2><<<grid_for(n), kBlock, 0, st>>>(s, x, v, r_max, n, o);
    return cudaGetLastError();
}

cudaError_t launch_sil_brute(const DevScene &s, const void *sils, int64_t n_sil, gq_vecs x, const float *r_max,
                             int64_t n, const gq_sil_out &o, cudaStream_t st) {
    DevScene b = s;
    b.sils = sils;
    if (s.dim == 3)
        k_sil_brute<3><<<grid_for(n), kBlock, 0, st>>>(b, n_sil, x, r_max, n, o);
    else
        k_sil_brute<2><<<grid_for(n), kBlock, 0, st>>>(b, n_sil, x, r_max, n, o);
    return cudaGetLastError();
}

cudaError_t launch_read_probe(const void *buf, int64_t bytes, int reps, unsigned *sink, cudaStream_t st) {
    int dev = 0, n_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    k_read_probe<<<dim3((unsigned)(8 * n_sm)), 256, 0, st>>>((const uint4 *)buf, bytes / 16, reps, sink);
    return cudaGetLastError();
}

cudaError_t launch_sil_f64(int dim, const float *recs, int64_t n_sil, gq_vecs x, int64_t n, double *out_d,
                           int32_t *out_id, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (dim == 3)
        k_sil_f64<3><<<grid_for(n), kBlock, 0, st>>>(recs, n_sil, x, n, out_d, out_id);
    else
        k_sil_f64<2><<<grid_for(n), kBlock, 0, st>>>(recs, n_sil, x, n, out_d, out_id);
    return cudaGetLastError();
}

cudaError_t launch_brute_f64(const DevScene &s, int kind, gq_vecs a, gq_vecs b, int64_t n, double *out_d,
                             int32_t *out_id, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (s.dim == 3)
        k_brute_f64<3><<<grid_for(n), kBlock, 0, st>>>(s, kind, a, b, n, out_d, out_id);
    else
        k_brute_f64<2><<<grid_for(n), kBlock, 0, st>>>(s, kind, a, b, n, out_d, out_id);
    return cudaGetLastError();
}

}  // namespace gqd
