// Result-record writers shared by the binary and the wide kernels: the winner's
// record is recomputed with the reference formulas (line_segment.py:64-78,
// triangle.py:49-81, bvh.py:267-274).
#pragma once

#include "prim.cuh"

namespace gqd {

// Record writers (SoA, component stride n).  A miss writes zeros.
__device__ __forceinline__ void put1(float *p, int64_t i, float v) {
    if (p) p[i] = v;
}
__device__ __forceinline__ void put2(float *p, int64_t n, int64_t i, float a, float b) {
    if (p) {
        p[i] = a;
        p[n + i] = b;
    }
}
__device__ __forceinline__ void put3(float *p, int64_t n, int64_t i, float a, float b, float c) {
    if (p) {
        p[i] = a;
        p[n + i] = b;
        p[2 * n + i] = c;
    }
}

// Triangle.closest_point (triangle.py:76-81)
__device__ __forceinline__ void cp3_record(const void *prims, int idx, bool ok, float px, float py, float pz,
                                           const gq_cp_out &o, int64_t n, int64_t qi) {
    float pt[3] = {0.f, 0.f, 0.f}, nx = 0.f, ny = 0.f, nz = 0.f, u = 0.f, v = 0.f, d = 0.f;
    int pid = 0;
    if (ok) {
        const float4 t0 = ldg4(prims, 3 * (int64_t)idx), t1 = ldg4(prims, 3 * (int64_t)idx + 1),
                     t2 = ldg4(prims, 3 * (int64_t)idx + 2);
        d = tri_closest<true>(px, py, pz, t0.x, t0.y, t0.z, t0.w, t1.x, t1.y, t1.z, t1.w, t2.x, pt, &u, &v);
        float cx, cy, cz;
        cross3(t0.w - t0.x, t1.x - t0.y, t1.y - t0.z, t1.z - t0.x, t1.w - t0.y, t2.x - t0.z, cx, cy, cz);
        const float inv = gq_rsqrt(gq_dot3(cx, cy, cz, cx, cy, cz));
        nx = cx * inv;
        ny = cy * inv;
        nz = cz * inv;
        pid = fbits(t2.y);
    }
    if (o.valid) o.valid[qi] = ok ? 1 : 0;
    put3(o.p, n, qi, pt[0], pt[1], pt[2]);
    put3(o.n, n, qi, nx, ny, nz);
    put2(o.t, n, qi, u, v);
    put1(o.d, qi, d);
    if (o.prim_id) o.prim_id[qi] = pid;
}

// LineSegment.closest_point (line_segment.py:64-78)
__device__ __forceinline__ void cp2_record(const void *prims, int idx, bool ok, float px, float py,
                                           const gq_cp_out &o, int64_t n, int64_t qi) {
    float ix = 0.f, iy = 0.f, nx = 0.f, ny = 0.f, h = 0.f, d = 0.f;
    int pid = 0;
    if (ok) {
        const float4 a = ldg4(prims, 2 * (int64_t)idx);
        const int4 f = __ldg(reinterpret_cast<const int4 *>(prims) + 2 * (int64_t)idx + 1);
        const float pax = px - a.x, pay = py - a.y, bax = a.z - a.x, bay = a.w - a.y;
        const float inv = gq_rsqrt(gq_dot2(bax, bay, bax, bay));
        const float tx = bax * inv, ty = bay * inv;
        nx = ty;
        ny = -tx;
        h = gq_clamp(gq_div(gq_dot2(pax, pay, bax, bay), gq_dot2(bax, bay, bax, bay)), 0.f, 1.f);
        ix = a.x + bax * h;
        iy = a.y + bay * h;
        d = gq_norm2(ix - px, iy - py);
        pid = f.x;
    }
    if (o.valid) o.valid[qi] = ok ? 1 : 0;
    put2(o.p, n, qi, ix, iy);
    put2(o.n, n, qi, nx, ny);
    put1(o.t, qi, h);
    put1(o.d, qi, d);
    if (o.prim_id) o.prim_id[qi] = pid;
}

// Triangle.ray_intersect (triangle.py:49-73) re-run on the winner with r_max = its t.
__device__ __forceinline__ void ray3_record(const void *prims, int idx, bool found, float xx, float xy, float xz,
                                            float vx, float vy, float vz, float r_max, const gq_ray_out &o,
                                            int64_t n, int64_t qi) {
    float px = 0.f, py = 0.f, pz = 0.f, nx = 0.f, ny = 0.f, nz = 0.f, u = 0.f, w0 = 0.f, d = 0.f;
    int pid = 0;
    bool ok = false;
    if (found) {
        const float4 t0 = ldg4(prims, 3 * (int64_t)idx), t1 = ldg4(prims, 3 * (int64_t)idx + 1),
                     t2 = ldg4(prims, 3 * (int64_t)idx + 2);
        float vv = __builtin_nanf(""), ww = 0.f;
        const float t = tri_ray(xx, xy, xz, vx, vy, vz, t0.x, t0.y, t0.z, t0.w, t1.x, t1.y, t1.z, t1.w, t2.x, r_max,
                                &vv, &ww);
        ok = (vv == vv);
        if (ok) {
            const float v1x = t0.w - t0.x, v1y = t1.x - t0.y, v1z = t1.y - t0.z;
            const float v2x = t1.z - t0.x, v2y = t1.w - t0.y, v2z = t2.x - t0.z;
            px = (t0.x + v1x * vv) + v2x * ww;
            py = (t0.y + v1y * vv) + v2y * ww;
            pz = (t0.z + v1z * vv) + v2z * ww;
            float cx, cy, cz;
            cross3(v1x, v1y, v1z, v2x, v2y, v2z, cx, cy, cz);
            const float inv = gq_rsqrt(gq_dot3(cx, cy, cz, cx, cy, cz));
            nx = cx * inv;
            ny = cy * inv;
            nz = cz * inv;
            u = 1.f - vv - ww;
            w0 = vv;
            d = t;
            pid = fbits(t2.y);
        }
    }
    if (o.valid) o.valid[qi] = ok ? 1 : 0;
    put3(o.p, n, qi, px, py, pz);
    put3(o.n, n, qi, nx, ny, nz);
    put2(o.t, n, qi, u, w0);
    put1(o.d, qi, d);
    if (o.prim_id) o.prim_id[qi] = pid;
    if (o.on_boundary) o.on_boundary[qi] = ok ? 1 : 0;
}

// bvh.py:267-274
__device__ __forceinline__ void ray2_record(const void *prims, int idx, bool hit, float xx, float xy, float vx,
                                            float vy, float d_min, const gq_ray_out &o, int64_t n, int64_t qi) {
    float px = 0.f, py = 0.f, nx = 0.f, ny = 0.f, t = 0.f, d = 0.f;
    int pid = 0;
    if (hit) {
        const float4 a = ldg4(prims, 2 * (int64_t)idx);
        const int4 f = __ldg(reinterpret_cast<const int4 *>(prims) + 2 * (int64_t)idx + 1);
        px = xx + vx * d_min;
        py = xy + vy * d_min;
        const float tx = a.z - a.x, ty = a.w - a.y;  // LineSegment.normal (line_segment.py:14-16)
        const float inv = gq_rsqrt(gq_dot2(ty, -tx, ty, -tx));
        nx = ty * inv;
        ny = -tx * inv;
        t = -1.f;
        d = d_min;
        pid = f.x;
    }
    if (o.valid) o.valid[qi] = hit ? 1 : 0;
    put2(o.p, n, qi, px, py);
    put2(o.n, n, qi, nx, ny);
    put1(o.t, qi, t);
    put1(o.d, qi, d);
    if (o.prim_id) o.prim_id[qi] = pid;
    if (o.on_boundary) o.on_boundary[qi] = hit ? 1 : 0;
}


}  // namespace gqd
