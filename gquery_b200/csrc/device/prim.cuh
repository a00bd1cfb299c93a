// Device leaf tests and box tests, written to round exactly like gQuery's DrJit code
// under the fixed semantics of gq_fmath.h (this file is compiled with --fmad=false;
// every fused operation is spelled out).
#pragma once

#include <cuda_runtime.h>

#include "../gq_fmath.h"
#include "../layout.h"

namespace gqd {

constexpr float kInf = __builtin_inff();

__device__ __forceinline__ float4 ldg4(const void *base, int64_t idx) {
    return __ldg(reinterpret_cast<const float4 *>(base) + idx);
}
__device__ __forceinline__ int fbits(float f) { return __float_as_int(f); }

// BoundingBox.distance (bvh.py:22-27, bvh3d.py:19-24)
__device__ __forceinline__ void box_dist2(float lox, float loy, float hix, float hiy, float px, float py,
                                          float &dmin, float &dmax) {
    const float ux = lox - px, uy = loy - py;
    const float vx = px - hix, vy = py - hiy;
    dmin = gq_norm2(fmaxf(fmaxf(ux, vx), 0.f), fmaxf(fmaxf(uy, vy), 0.f));
    dmax = gq_norm2(fminf(ux, vx), fminf(uy, vy));
}
__device__ __forceinline__ void box_dist3(float lox, float loy, float loz, float hix, float hiy, float hiz, float px,
                                          float py, float pz, float &dmin, float &dmax) {
    const float ux = lox - px, uy = loy - py, uz = loz - pz;
    const float vx = px - hix, vy = py - hiy, vz = pz - hiz;
    dmin = gq_norm3(fmaxf(fmaxf(ux, vx), 0.f), fmaxf(fmaxf(uy, vy), 0.f), fmaxf(fmaxf(uz, vz), 0.f));
    dmax = gq_norm3(fminf(ux, vx), fminf(uy, vy), fminf(uz, vz));
}
__device__ __forceinline__ float box_dmin3(float lox, float loy, float loz, float hix, float hiy, float hiz, float px,
                                           float py, float pz) {
    const float ux = lox - px, uy = loy - py, uz = loz - pz;
    const float vx = px - hix, vy = py - hiy, vz = pz - hiz;
    return gq_norm3(fmaxf(fmaxf(ux, vx), 0.f), fmaxf(fmaxf(uy, vy), 0.f), fmaxf(fmaxf(uz, vz), 0.f));
}

// BoundingBox.intersect (bvh.py:33-50, bvh3d.py:30-47); returns t_min or +inf on a miss.
__device__ __forceinline__ bool box_ray2(float lox, float loy, float hix, float hiy, float xx, float xy, float vx,
                                         float vy, float r_max, float &t_min) {
    const float t0x = gq_div(lox - xx, vx), t0y = gq_div(loy - xy, vy);
    const float t1x = gq_div(hix - xx, vx), t1y = gq_div(hiy - xy, vy);
    const float tnm = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), 0.f);
    const float tfm = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), r_max);
    const bool hit = !(tnm > tfm);
    t_min = hit ? tnm : kInf;
    return hit;
}
__device__ __forceinline__ bool box_ray3(float lox, float loy, float loz, float hix, float hiy, float hiz, float xx,
                                         float xy, float xz, float vx, float vy, float vz, float r_max,
                                         float &t_min) {
    const float t0x = gq_div(lox - xx, vx), t0y = gq_div(loy - xy, vy), t0z = gq_div(loz - xz, vz);
    const float t1x = gq_div(hix - xx, vx), t1y = gq_div(hiy - xy, vy), t1z = gq_div(hiz - xz, vz);
    const float tnm = fmaxf(fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fminf(t0z, t1z)), 0.f);
    const float tfm = fminf(fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z)), r_max);
    const bool hit = !(tnm > tfm);
    t_min = hit ? tnm : kInf;
    return hit;
}

// closest_point_line_segment (math.py:15-21), distance only / with point and t
__device__ __forceinline__ float seg_dist(float px, float py, float ax, float ay, float bx, float by) {
    const float ux = bx - ax, uy = by - ay, vx = px - ax, vy = py - ay;
    const float t = gq_clamp(gq_div(gq_dot2(vx, vy, ux, uy), gq_dot2(ux, uy, ux, uy)), 0.f, 1.f);
    const float qx = gq_lerp(ax, bx, t), qy = gq_lerp(ay, by, t);
    return gq_norm2(qx - px, qy - py);
}
__device__ __forceinline__ float seg_dist3(float px, float py, float pz, float ax, float ay, float az, float bx,
                                           float by, float bz, float &qx, float &qy, float &qz) {
    const float ux = bx - ax, uy = by - ay, uz = bz - az;
    const float vx = px - ax, vy = py - ay, vz = pz - az;
    const float t = gq_clamp(gq_div(gq_dot3(vx, vy, vz, ux, uy, uz), gq_dot3(ux, uy, uz, ux, uy, uz)), 0.f, 1.f);
    qx = gq_lerp(ax, bx, t);
    qy = gq_lerp(ay, by, t);
    qz = gq_lerp(az, bz, t);
    return gq_norm3(qx - px, qy - py, qz - pz);
}

// ray_intersection (math.py:32-39): t of the hit, or +inf
__device__ __forceinline__ float seg_ray(float xx, float xy, float vx, float vy, float ax, float ay, float bx,
                                         float by) {
    const float ux = bx - ax, uy = by - ay, wx = xx - ax, wy = xy - ay;
    const float d = vx * uy - vy * ux;
    const float s = gq_div(vx * wy - vy * wx, d);
    const float t = gq_div(ux * wy - uy * wx, d);
    const bool valid = (t > 0.f) & (s >= 0.f) & (s <= 1.f);
    return valid ? t : kInf;
}

// closest_point_triangle (math.py:42-107).  Returns the distance; optionally the
// point and the remapped uv = (uv[1], 1 - uv[0] - uv[1]).
template <bool FULL>
__device__ __forceinline__ float tri_closest(float px, float py, float pz, float ax, float ay, float az, float bx,
                                             float by, float bz, float cx, float cy, float cz, float *pt = nullptr,
                                             float *u_out = nullptr, float *v_out = nullptr) {
    const float abx = bx - ax, aby = by - ay, abz = bz - az;
    const float acx = cx - ax, acy = cy - ay, acz = cz - az;
    const float apx = px - ax, apy = py - ay, apz = pz - az;
    const float d1 = gq_dot3(abx, aby, abz, apx, apy, apz);
    const float d2 = gq_dot3(acx, acy, acz, apx, apy, apz);
    const float bpx = px - bx, bpy = py - by, bpz = pz - bz;
    const float d3 = gq_dot3(abx, aby, abz, bpx, bpy, bpz);
    const float d4 = gq_dot3(acx, acy, acz, bpx, bpy, bpz);
    const float cpx = px - cx, cpy = py - cy, cpz = pz - cz;
    const float d5 = gq_dot3(abx, aby, abz, cpx, cpy, cpz);
    const float d6 = gq_dot3(acx, acy, acz, cpx, cpy, cpz);
    float qx, qy, qz, uv0, uv1;
    if ((d1 <= 0.f) & (d2 <= 0.f)) {
        qx = ax; qy = ay; qz = az; uv0 = 1.f; uv1 = 0.f;
    } else if ((d3 >= 0.f) & (d4 <= d3)) {
        qx = bx; qy = by; qz = bz; uv0 = 0.f; uv1 = 1.f;
    } else if ((d6 >= 0.f) & (d5 <= d6)) {
        qx = cx; qy = cy; qz = cz; uv0 = 0.f; uv1 = 0.f;
    } else {
        const float vc = d1 * d4 - d3 * d2;
        const float vb = d5 * d2 - d1 * d6;
        const float va = d3 * d6 - d5 * d4;
        if ((vc <= 0.f) & (d1 >= 0.f) & (d3 <= 0.f)) {
            const float v = gq_div(d1, d1 - d3);
            qx = ax + abx * v; qy = ay + aby * v; qz = az + abz * v;
            uv0 = 1.f - v; uv1 = v;
        } else if ((vb <= 0.f) & (d2 >= 0.f) & (d6 <= 0.f)) {
            const float w = gq_div(d2, d2 - d6);
            qx = ax + acx * w; qy = ay + acy * w; qz = az + acz * w;
            uv0 = 1.f - w; uv1 = 0.f;
        } else if ((va <= 0.f) & ((d4 - d3) >= 0.f) & ((d5 - d6) >= 0.f)) {
            const float w = gq_div(d4 - d3, (d4 - d3) + (d5 - d6));
            qx = bx + (cx - bx) * w; qy = by + (cy - by) * w; qz = bz + (cz - bz) * w;
            uv0 = 0.f; uv1 = 1.f - w;
        } else {
            const float denom = gq_div(1.f, va + vb + vc);
            const float v = vb * denom, w = vc * denom;
            qx = (ax + abx * v) + acx * w;
            qy = (ay + aby * v) + acy * w;
            qz = (az + abz * v) + acz * w;
            uv0 = 1.f - v - w; uv1 = v;
        }
    }
    if (FULL) {
        pt[0] = qx; pt[1] = qy; pt[2] = qz;
        *u_out = uv1;
        *v_out = 1.f - uv0 - uv1;
    }
    return gq_norm3(px - qx, py - qy, pz - qz);
}

// cross with the fused form of gq_fmath.h
__device__ __forceinline__ void cross3(float ax, float ay, float az, float bx, float by, float bz, float &cx,
                                       float &cy, float &cz) {
    cx = gq_fma(ay, bz, -(az * by));
    cy = gq_fma(az, bx, -(ax * bz));
    cz = gq_fma(ax, by, -(ay * bx));
}

// ray_triangle_intersect (math.py:110-128): returns t when it hits inside [0, r_max], else r_max.
__device__ __forceinline__ float tri_ray(float xx, float xy, float xz, float dx, float dy, float dz, float ax,
                                         float ay, float az, float bx, float by, float bz, float cx, float cy,
                                         float cz, float r_max, float *vv = nullptr, float *ww = nullptr) {
    const float v1x = bx - ax, v1y = by - ay, v1z = bz - az;
    const float v2x = cx - ax, v2y = cy - ay, v2z = cz - az;
    float px, py, pz;
    cross3(dx, dy, dz, v2x, v2y, v2z, px, py, pz);
    const float det = gq_dot3(v1x, v1y, v1z, px, py, pz);
    if (fabsf(det) > GQ_EPS_F) {
        const float inv_det = gq_div(1.f, det);
        const float sx = xx - ax, sy = xy - ay, sz = xz - az;
        const float v = gq_dot3(sx, sy, sz, px, py, pz) * inv_det;
        if ((v >= 0.f) & (v <= 1.f)) {
            float qx, qy, qz;
            cross3(sx, sy, sz, v1x, v1y, v1z, qx, qy, qz);
            const float w = gq_dot3(dx, dy, dz, qx, qy, qz) * inv_det;
            if ((w >= 0.f) & (v + w <= 1.f)) {
                const float t = gq_dot3(v2x, v2y, v2z, qx, qy, qz) * inv_det;
                if ((t >= 0.f) & (t <= r_max)) {
                    r_max = t;
                    if (vv) {
                        *vv = v;
                        *ww = w;
                    }
                }
            }
        }
    }
    return r_max;
}

__device__ __forceinline__ bool in_range(float x, float a, float b) { return (x >= a) & (x <= b); }

// SNCHNode.overlaps (snch.py:16-60 / snch3d.py:51-95), cone part.  `dmin` is the box
// distance already computed by the caller; the box test itself is dmin <= r_max.
template <int D>
__device__ __forceinline__ bool cone_overlaps(const float *lo, const float *hi, const float *axis, float half,
                                              float radius, const float *x, float dmin) {
    bool is_overlap = (half > GQ_PIO2_F) & (dmin < GQ_EPS_F);
    if (is_overlap) return true;
    float c[D], vca[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        c[k] = gq_div(lo[k] + hi[k], 2.f);
        vca[k] = c[k] - x[k];
    }
    float l;
    if (D == 2)
        l = gq_norm2(vca[0], vca[1]);
    else
        l = gq_norm3(vca[0], vca[1], vca[2]);
#pragma unroll
    for (int k = 0; k < D; ++k) vca[k] = gq_div(vca[k], l);
    float dt = (D == 2) ? gq_dot2(axis[0], axis[1], vca[0], vca[1])
                        : gq_dot3(axis[0], axis[1], axis[2], vca[0], vca[1], vca[2]);
    const float dA = gq_acos(gq_clamp(dt, -1.f, 1.f));
    if (in_range(GQ_PIO2_F, dA - half, dA + half)) return true;
    if (l > radius) {
        const float vch = gq_asin(gq_div(radius, l));
        const float hs = half + vch;
        return (hs > GQ_PIO2_F) | in_range(GQ_PIO2_F, dA - hs, dA + hs);
    }
    float e[D];
#pragma unroll
    for (int k = 0; k < D; ++k) e[k] = hi[k] - c[k];
    float dd = (D == 2) ? gq_dot2(e[0], e[1], fabsf(vca[0]), fabsf(vca[1]))
                        : gq_dot3(e[0], e[1], e[2], fabsf(vca[0]), fabsf(vca[1]), fabsf(vca[2]));
    const float s = l - dd;
    if (s < 0.f) return true;
    if (D == 2) {
        // project_to_plane (math.py:24-28): b = (-n.y, n.x), |dot(e, |b|)|
        dd = fabsf(gq_dot2(e[0], e[1], fabsf(-vca[1]), fabsf(vca[0])));
    } else {
        // project_to_plane_3D (snch3d.py:12-30)
        const float nx = vca[0], ny = vca[1], nz = vca[D - 1];
        const float sign = copysignf(1.f, nz);
        const float a = gq_div(-1.f, sign + nz);
        const float b = nx * ny * a;
        const float b1x = 1.f + sign * nx * nx * a, b1y = sign * b, b1z = -sign * nx;
        const float b2x = b, b2y = sign + ny * ny * a, b2z = -ny;
        const float r1 = gq_dot3(e[0], e[1], e[D - 1], fabsf(b1x), fabsf(b1y), fabsf(b1z));
        const float r2 = gq_dot3(e[0], e[1], e[D - 1], fabsf(b2x), fabsf(b2y), fabsf(b2z));
        dd = gq_sqrt(r1 * r1 + r2 * r2);
    }
    const float vch = gq_atan2(dd, s);
    const float hs = half + vch;
    return (hs > GQ_PIO2_F) | in_range(GQ_PIO2_F, dA - hs, dA + hs);
}

// The normal-cone test of cone_overlaps restated without inverse trigonometry, for the
// traversals that promise the reference's answers up to FP32 ties (not its exact visit
// order).  With dA the angle between the cone axis and the view direction v and h_v
// the view cone's half angle, the reference accepts when h + h_v >= pi/2 or
// |dA - pi/2| <= h + h_v, i.e. when |cos dA| = |axis . v| <= sin(h + h_v); the sine and
// cosine of h + h_v follow from sin h, cos h (hardware approximations) and those of h_v,
// which are ratios of lengths the reference already forms (radius / l, or d and s of
// its atan2).  Both comparisons carry a margin of kConeSlack, far above the few-ulp
// error of either form, so every node the reference admits is admitted here; a node it
// rejects by less than the margin may be visited too, which cannot change a correct
// answer.
constexpr float kConeSlack = 1e-5f;

template <int D>
__device__ __forceinline__ bool cone_overlaps_fast(const float *lo, const float *hi, const float *axis, float half,
                                                   float radius, const float *x, float dmin) {
    if (half >= GQ_PIO2_F) return true;  // |dA - pi/2| <= pi/2 <= h always holds
    float c[D], v[D], l2 = 0.f;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        c[k] = 0.5f * (lo[k] + hi[k]);
        v[k] = c[k] - x[k];
        l2 = __fmaf_rn(v[k], v[k], l2);
    }
    if (!(l2 > 1e-30f)) return true;
    const float il = rsqrtf(l2), l = l2 * il;
    float dt = 0.f;
#pragma unroll
    for (int k = 0; k < D; ++k) dt = __fmaf_rn(axis[k], v[k], dt);
    dt = fabsf(dt * il);
    float sv, cv;  // sine and cosine of the view cone's half angle
    if (l > radius) {
        sv = radius * il;
        cv = sqrtf(fmaxf(0.f, 1.f - sv * sv));
    } else {
        float e[D], u[D], dd = 0.f;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            e[k] = hi[k] - c[k];
            u[k] = v[k] * il;
            dd = __fmaf_rn(e[k], fabsf(u[k]), dd);
        }
        const float s = l - dd;
        if (s < kConeSlack * l) return true;
        float pd;
        if (D == 2) {
            pd = fabsf(__fmaf_rn(e[0], fabsf(u[D - 1]), e[D - 1] * fabsf(u[0])));
        } else {
            // project_to_plane_3D (snch3d.py:26-30) with the same orthonormal basis
            const float nx = u[0], ny = u[1], nz = u[D - 1];
            const float sign = copysignf(1.f, nz);
            const float a = -1.f / (sign + nz);
            const float b = nx * ny * a;
            const float r1 = __fmaf_rn(e[D - 1], fabsf(-sign * nx),
                                       __fmaf_rn(e[1], fabsf(sign * b), e[0] * fabsf(1.f + sign * nx * nx * a)));
            const float r2 = __fmaf_rn(e[D - 1], fabsf(-ny), __fmaf_rn(e[1], fabsf(sign + ny * ny * a), e[0] * fabsf(b)));
            pd = sqrtf(__fmaf_rn(r1, r1, r2 * r2));
        }
        const float ih = rsqrtf(__fmaf_rn(pd, pd, s * s));
        sv = pd * ih;
        cv = s * ih;
    }
    float sh, ch;
    __sincosf(half, &sh, &ch);
    const float cos_sum = ch * cv - sh * sv;  // cos(h + h_v)
    if (cos_sum <= kConeSlack) return true;   // h + h_v >= pi/2
    const float sin_sum = sh * cv + ch * sv;  // sin(h + h_v), h + h_v in [0, pi/2)
    (void)dmin;
    return dt <= sin_sum + kConeSlack;
}

}  // namespace gqd
