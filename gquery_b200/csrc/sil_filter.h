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

// ---------------------------------------------------------------- node bound
//
// The same argument one level up.  For a node (a child of an SNCH pair) with box
// centre c, every silhouette edge of its subtree and each of its two faces, take the
// face normal n with the edge's orientation sign s (both normals of an edge may flip
// together: the test above is unchanged), and the points q of the edge.  Then
//   s n . (q - x) = s n . (q - c) + s n . (c - x),
// where s n . (q - c) lies in [lo, hi] (from the end points and the spans).  With
// v = c - x and l = |v|, the second term is bounded two ways from the spread of the
// unit vectors s n around the unit axis A:
//   delta form: s n . v in [A . v - delta l, A . v + delta l], delta = max |s n - A|;
//   cone form:  s n . v in [l cos(min(phi + theta, pi)), l cos(max(phi - theta, 0))],
//               theta the largest angle between s n and A, phi that between A and v,
//               from l cos phi = A . v and l sin phi = |A x v| (no trigonometry and no
//               cancellation near phi = 0).
// The cone form is never wider (l (cos(phi - theta) - cos phi) <= 2 sin(theta / 2) l =
// delta l) and skips a node seen head-on for spreads up to about 90 degrees where the
// delta form stops near 60; the delta form is about half the arithmetic.  The host
// computes lo, hi, delta and theta in double (delta rounded up, theta widened by
// 1e-6 rad, lo and hi rounded outward) and stores (A, delta, cos theta, sin theta, lo,
// hi).  When the interval lies beyond a margin on one side of zero, both dot products
// of every edge have the sign of that side and none is a silhouette for x, so the
// traversal may skip the child: the reference's visit order of the other nodes and its
// answers stay as they are.  With the orientation signs of a consistently wound mesh
// the axis gathers outward normals only, so the spread measures how much the surface
// bends inside the node rather than the pi of a cone that holds both orientations.
//
// Margin.  Besides the reference's rounding of each dot product (at most
// 1.75 eps (6 M + 4 X), see above), the FP32 evaluation of either form (c from the box,
// c - x, the dot and cross products, l, the products with delta or with the stored
// cosine and sine, the sums), and the rounding of A and n to unit length move the
// interval by at most about eps (40 M + 30 X); the margin 2e-5 (2 M + X) is eight times
// the total.  Nodes whose subtree holds a boundary edge or an edge without
// GQ_SIL_FILTER get lo = -inf, hi = +inf (never skipped); nodes without silhouettes get
// lo = hi = +inf (always skipped).

// Geometry of one 3D silhouette edge for the node bound: end points, stored face
// normals, orientation sign and whether the pre-test may be used on it.
struct SilEdgeGeom {
    float a[3], b[3], n0[3], n1[3];
    float orient;
    bool usable;
};

// Steps of the search for a narrow cone axis, and the largest node (in silhouette
// records) it runs on: above that the normals of a closed surface spread about pi
// around any axis.
constexpr int kSilAxisSteps = 8;
constexpr long long kSilAxisMaxRecords = 8192;

// Stored bound of a node: b[0..2] = A, b[3] = delta, b[4] = cos theta, b[5] = sin theta,
// b[6] = lo, b[7] = hi.
constexpr int kSilNodeBound = 8;

GQ_HD float sil_node_margin(float x_inf, float coord_bound) { return 2.f * sil_margin(x_inf, coord_bound); }

// The node's centre as the bound was computed with it: the middle of its box.
GQ_HD float sil_node_centre(float lo, float hi) { return 0.5f * (lo + hi); }

// cos and sin of the cone half-angle theta + 1e-6 (at most pi) from cmin = cos theta.
GQ_HD void sil_cone_of(double cmin, float &ct, float &st) {
    const double c = cmin > 1.0 ? 1.0 : (cmin < -1.0 ? -1.0 : cmin);
    const double s = sqrt((1.0 - c) * (1.0 + c));
    const double ce = 0.9999999999995, se = 1e-6;  // cos and sin of 1e-6
    double c2 = c * ce - s * se, s2 = s * ce + c * se;
    if (!(s2 >= 0.0) || c2 < -1.0) {  // widened past pi
        c2 = -1.0;
        s2 = 0.0;
    }
    ct = (float)c2;
    st = (float)s2;
}

// Delta form: true when the node (centre c, bound b) certainly holds no silhouette for x.
GQ_HD bool sil_node_excluded_delta(float cx, float cy, float cz, const float *b, float xx, float xy, float xz,
                                   float margin) {
    const float vx = cx - xx, vy = cy - xy, vz = cz - xz;
    const float g = gq_dot3(b[0], b[1], b[2], vx, vy, vz);
    const float dl = b[3] * gq_norm3(vx, vy, vz);
    return (g + b[6] - dl > margin) | (g + b[7] + dl < -margin);
}

// Cone form of the same test.
GQ_HD bool sil_node_excluded_cone(float cx, float cy, float cz, const float *b, float xx, float xy, float xz,
                                  float margin) {
    const float vx = cx - xx, vy = cy - xy, vz = cz - xz;
    const float ax = b[0], ay = b[1], az = b[2], ct = b[4], st = b[5];
    const float g = gq_dot3(ax, ay, az, vx, vy, vz);  // l cos phi
    const float wx = gq_fma(ay, vz, -(az * vy)), wy = gq_fma(az, vx, -(ax * vz)), wz = gq_fma(ax, vy, -(ay * vx));
    const float h = gq_norm3(wx, wy, wz);  // l sin phi
    const float l = gq_norm3(vx, vy, vz);
    const float up = g >= l * ct ? l : gq_fma(g, ct, h * st);         // phi <= theta: v inside the cone
    const float dn = g <= -(l * ct) ? -l : gq_fma(g, ct, -(h * st));  // phi >= pi - theta
    return (dn + b[6] > margin) | (up + b[7] < -margin);
}

#if !defined(__CUDA_ARCH__)
// Length of an edge's face normal f (0: n0, 1: n1) times its orientation sign, in double:
// sqrt((s0 * s0 + s1 * s1) + s2 * s2).
inline double sil_normal_len(const SilEdgeGeom &e, int f) {
    const float *n = f ? e.n1 : e.n0;
    const double s0 = (double)e.orient * n[0], s1 = (double)e.orient * n[1], s2 = (double)e.orient * n[2];
    return sqrt(s0 * s0 + s1 * s1 + s2 * s2);
}

// Node bound over the edges begin..end-1 (edge(j) returns their SilEdgeGeom) for a node
// whose box centre is c: out[kSilNodeBound] as above.  len(j, f, e) returns
// sil_normal_len(e, f) of edge j, computed here or read from a table filled once: a
// record's normals are read by the bound of every node above it, several times each.
template <class EdgeAt, class NormalLen>
inline void sil_node_bound(float cx, float cy, float cz, long long begin, long long end, EdgeAt edge,
                           NormalLen len, float out[kSilNodeBound]);

template <class EdgeAt>
inline void sil_node_bound(float cx, float cy, float cz, long long begin, long long end, EdgeAt edge,
                           float out[kSilNodeBound]) {
    sil_node_bound(cx, cy, cz, begin, end, edge,
                   [](long long, int f, const SilEdgeGeom &e) { return sil_normal_len(e, f); }, out);
}

template <class EdgeAt, class NormalLen>
inline void sil_node_bound(float cx, float cy, float cz, long long begin, long long end, EdgeAt edge,
                           NormalLen len, float out[kSilNodeBound]) {
    out[0] = out[1] = out[2] = 0.f;
    out[3] = 0.f;
    out[4] = 1.f;
    out[5] = 0.f;
    if (begin >= end) {  // no silhouettes: always skipped
        out[6] = out[7] = __builtin_inff();
        return;
    }
    double m[3] = {0.0, 0.0, 0.0};
    bool ok = true;
    for (long long j = begin; j < end && ok; ++j) {
        const SilEdgeGeom e = edge(j);
        ok = e.usable;
        for (int k = 0; k < 3; ++k) m[k] += (double)e.orient * ((double)e.n0[k] + (double)e.n1[k]);
    }
    const double ml = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    if (!ok || !(ml > 1e-30)) {  // never skipped
        out[3] = __builtin_inff();
        out[6] = -__builtin_inff();
        out[7] = __builtin_inff();
        return;
    }
    // axis: the mean direction, then steps toward the farthest normal (Badoiu-Clarkson
    // iterations for the smallest enclosing cone); the axis with the smallest spread wins
    double ax[3] = {m[0] / ml, m[1] / ml, m[2] / ml}, best[3] = {ax[0], ax[1], ax[2]}, best_c = -2.0;
    const int steps = end - begin <= kSilAxisMaxRecords ? kSilAxisSteps : 0;
    for (int it = 0; it <= steps; ++it) {
        double cmin_it = 2.0, far[3] = {0.0, 0.0, 0.0};
        for (long long j = begin; j < end; ++j) {
            const SilEdgeGeom e = edge(j);
            for (int f = 0; f < 2; ++f) {
                const float *n = f ? e.n1 : e.n0;
                const double sn[3] = {(double)e.orient * n[0], (double)e.orient * n[1], (double)e.orient * n[2]};
                const double nl = len(j, f, e);
                const double cs = (sn[0] * ax[0] + sn[1] * ax[1] + sn[2] * ax[2]) / nl;
                if (cs < cmin_it) {
                    cmin_it = cs;
                    for (int k = 0; k < 3; ++k) far[k] = sn[k] / nl;
                }
            }
        }
        if (cmin_it > best_c) {
            best_c = cmin_it;
            for (int k = 0; k < 3; ++k) best[k] = ax[k];
        }
        const double w = 1.0 / (it + 2);
        double nx[3], nn = 0.0;
        for (int k = 0; k < 3; ++k) {
            nx[k] = ax[k] + w * (far[k] - ax[k]);
            nn += nx[k] * nx[k];
        }
        nn = sqrt(nn);
        if (!(nn > 1e-12)) break;
        for (int k = 0; k < 3; ++k) ax[k] = nx[k] / nn;
    }
    float A[3];
    for (int k = 0; k < 3; ++k) A[k] = out[k] = (float)best[k];
    const double al = sqrt((double)A[0] * A[0] + (double)A[1] * A[1] + (double)A[2] * A[2]);
    const double c[3] = {cx, cy, cz};
    double dmax = 0.0, cmin = 1.0, lo = __builtin_inf(), hi = -__builtin_inf();
    for (long long j = begin; j < end; ++j) {
        const SilEdgeGeom e = edge(j);
        for (int f = 0; f < 2; ++f) {
            const float *n = f ? e.n1 : e.n0;
            double d2 = 0.0, cs = 0.0, ac = 0.0, sp = 0.0;
            for (int k = 0; k < 3; ++k) {
                const double sn = (double)e.orient * (double)n[k];
                d2 += (sn - A[k]) * (sn - A[k]);
                cs += sn * A[k];
                ac += sn * ((double)e.a[k] - c[k]);
                sp += sn * ((double)e.b[k] - (double)e.a[k]);
            }
            dmax = fmax(dmax, sqrt(d2));
            cmin = fmin(cmin, cs / (len(j, f, e) * al));  // the angle between the directions
            lo = fmin(lo, ac + fmin(0.0, sp));
            hi = fmax(hi, ac + fmax(0.0, sp));
        }
    }
    float fd = (float)(dmax * (1.0 + 1e-12));
    if ((double)fd < dmax) fd = nextafterf(fd, __builtin_inff());
    out[3] = fd;
    sil_cone_of(cmin, out[4], out[5]);
    // outward to FP32, with room for the double rounding above
    const double pad = 1e-12 * (fabs(lo) + fabs(hi) + 1.0);
    float fl = (float)(lo - pad), fh = (float)(hi + pad);
    if ((double)fl > lo - pad) fl = nextafterf(fl, -__builtin_inff());
    if ((double)fh < hi + pad) fh = nextafterf(fh, __builtin_inff());
    out[6] = fl;
    out[7] = fh;
}
#endif
