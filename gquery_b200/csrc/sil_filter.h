// Pre-test of the 3D silhouette-edge test that never changes its answer.
//
// SilhouetteEdge.closest_silhouette (silhouette_edge.py:50-64) takes q, the closest
// point of the edge [a, b] to x, w = q - x, and calls the edge a silhouette when
// (w . n0) * (w . n1) < 0 (is_silhouette_edge, silhouette_edge.py:7-12), n0 and n1
// being the unit normals of its two faces.  With u = b - a and q = a + t u for the
// t in [0, 1] the reference computes, w . n = n . (a - x) + t (n . u) lies in
// [A + min(0, U), A + max(0, U)] with A = n . (a - x) and U = n . u, which the host
// stores per edge.  When both intervals lie beyond a margin on the same side of
// zero, both of the reference's dot products have that sign and the edge is no
// silhouette for x, so the leaf test may skip it without computing q: skipping a
// non-silhouette never changes an answer or the order of the accepted ones.
//
// Margin.  With eps = 2^-24, M the largest |coordinate| of the scene, X that of x
// and |n|_1 <= kSilFilterNormMax, the reference's rounding (lerp for q, w = q - x,
// the fused dot product) moves w . n by at most 1.75 eps (6 M + 4 X), and the
// pre-test's own rounding (a - x, the dot products, U stored in FP32, the interval
// ends) moves the interval by at most 1.75 eps (15 M + 5 X): together below
// 2.2e-6 M + 1e-6 X.  The margin 1e-5 (2 M + X) is ten times that.  Edges whose
// normals are not finite or exceed the norm bound (degenerate faces) carry no
// GQ_SIL_FILTER flag and always take the full test, as do boundary edges.
#pragma once

#include "gq_fmath.h"

#define GQ_SIL_FILTER 4u  // gq_sile_t flag: span0 / span1 hold n0 . (b - a), n1 . (b - a)

constexpr float kSilFilterNormMax = 1.75f;

// normalize(cross(u, v)) with the FP32 operations of the per-edge test the device
// would otherwise repeat (cross in fused form, normalize = v * (1 / sqrt(dot(v, v)))).
GQ_HD void sil_face_normal(float ux, float uy, float uz, float vx, float vy, float vz, float &nx, float &ny,
                           float &nz) {
    const float cx = gq_fma(uy, vz, -(uz * vy));
    const float cy = gq_fma(uz, vx, -(ux * vz));
    const float cz = gq_fma(ux, vy, -(uy * vx));
    const float inv = gq_rsqrt(gq_dot3(cx, cy, cz, cx, cy, cz));
    nx = cx * inv;
    ny = cy * inv;
    nz = cz * inv;
}

// n . (b - a) as the pre-test's bound assumes it was computed.
GQ_HD float sil_span(float nx, float ny, float nz, float ax, float ay, float az, float bx, float by, float bz) {
    return gq_dot3(nx, ny, nz, bx - ax, by - ay, bz - az);
}

// Whether an edge with these normals and spans may use the pre-test.
GQ_HD bool sil_filter_usable(float n0x, float n0y, float n0z, float n1x, float n1y, float n1z, float s0, float s1) {
    const float l0 = fabsf(n0x) + fabsf(n0y) + fabsf(n0z), l1 = fabsf(n1x) + fabsf(n1y) + fabsf(n1z);
    // finite and bounded (NaN fails every comparison)
    return (l0 <= kSilFilterNormMax) & (l1 <= kSilFilterNormMax) & (fabsf(s0) <= 3.0e38f) & (fabsf(s1) <= 3.0e38f);
}

// Margin for a query at x (largest |coordinate| x_inf) in a scene whose vertices have
// |coordinate| <= coord_bound.
GQ_HD float sil_margin(float x_inf, float coord_bound) { return 1e-5f * (x_inf + 2.f * coord_bound); }

// True when the edge is certainly no silhouette for x.
GQ_HD bool sil_edge_excluded(float ax, float ay, float az, float n0x, float n0y, float n0z, float n1x, float n1y,
                             float n1z, float s0, float s1, float xx, float xy, float xz, float margin) {
    const float vx = ax - xx, vy = ay - xy, vz = az - xz;
    const float a0 = gq_dot3(n0x, n0y, n0z, vx, vy, vz);
    const float a1 = gq_dot3(n1x, n1y, n1z, vx, vy, vz);
    const float lo0 = a0 + fminf(0.f, s0), hi0 = a0 + fmaxf(0.f, s0);
    const float lo1 = a1 + fminf(0.f, s1), hi1 = a1 + fmaxf(0.f, s1);
    return ((lo0 > margin) & (lo1 > margin)) | ((hi0 < -margin) & (hi1 < -margin));
}
