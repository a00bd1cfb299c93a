// ORACLE — test infrastructure only.  Nothing in the product links, imports or
// calls this file; tests/, the smoke check and bench.py's CPU-baseline leg use it
// as the checker.
//
// A scalar C++ restatement of gQuery's six traversals, statement for statement,
// over the reference's own float layouts (node/primitive/silhouette arrays with
// strides 7/9/13/16 and 5/10/10/19, integers stored as floats):
//   cp2d   gquery/shapes/bvh.py:127-198      ray2d  gquery/shapes/bvh.py:200-276
//   cp3d   gquery/shapes/bvh3d.py:108-174    ray3d  gquery/shapes/bvh3d.py:176-239
//   sil2d  gquery/shapes/snch.py:106-164     sil3d  gquery/shapes/snch3d.py:143-203
// with the leaf tests of gquery/core/math.py, line_segment.py, triangle.py,
// silhouette_vertex.py and silhouette_edge.py.  Every function cites its source.
//
// Parity status: the traversal control flow is checked against the reference's
// own Python traversal executed under a scalar stand-in for DrJit (fixtures in
// tests/golden/), and against FP64 brute force and hand-derived known answers.
// The rounding of DrJit's array-library calls (dot, norm, lerp, acos, ...) cannot
// be pinned: DrJit is not installable here and the reference ships no golden
// vectors.  Those choices are fixed in gquery_b200/csrc/gq_fmath.h.
//
// Also: FP64 brute force for the three query kinds (the structure of the
// reference's *_baseline methods, polyline.py:137-223, mesh.py:287-362).
//
// Build: see oracle/Makefile (-O2 -ffp-contract=off).
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "../gquery_b200/csrc/gq_fmath.h"

namespace {

const float INF = GQ_INF_F;

struct V2 {
    float x, y;
};
struct V3 {
    float x, y, z;
};
static inline V2 sub(V2 a, V2 b) { return {a.x - b.x, a.y - b.y}; }
static inline V2 add(V2 a, V2 b) { return {a.x + b.x, a.y + b.y}; }
static inline V2 mul(V2 a, float s) { return {a.x * s, a.y * s}; }
static inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 mul(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
static inline float dot(V2 a, V2 b) { return gq_dot2(a.x, a.y, b.x, b.y); }
static inline float dot(V3 a, V3 b) { return gq_dot3(a.x, a.y, a.z, b.x, b.y, b.z); }
static inline float norm(V2 a) { return gq_sqrt(dot(a, a)); }
static inline float norm(V3 a) { return gq_sqrt(dot(a, a)); }
static inline V2 normalize(V2 a) { return mul(a, gq_rsqrt(dot(a, a))); }
static inline V3 normalize(V3 a) { return mul(a, gq_rsqrt(dot(a, a))); }
static inline V3 cross(V3 a, V3 b) {
    return {gq_fma(a.y, b.z, -(a.z * b.y)), gq_fma(a.z, b.x, -(a.x * b.z)), gq_fma(a.x, b.y, -(a.y * b.x))};
}
static inline V2 vmax(V2 a, V2 b) { return {gq_max(a.x, b.x), gq_max(a.y, b.y)}; }
static inline V2 vmin(V2 a, V2 b) { return {gq_min(a.x, b.x), gq_min(a.y, b.y)}; }
static inline V3 vmax(V3 a, V3 b) { return {gq_max(a.x, b.x), gq_max(a.y, b.y), gq_max(a.z, b.z)}; }
static inline V3 vmin(V3 a, V3 b) { return {gq_min(a.x, b.x), gq_min(a.y, b.y), gq_min(a.z, b.z)}; }
static inline V2 vabs(V2 a) { return {fabsf(a.x), fabsf(a.y)}; }
static inline V3 vabs(V3 a) { return {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
static inline int I(float f) { return (int)f; }  // DrJit Int(Float): truncation
static inline float cross2(V2 a, V2 b) { return a.x * b.y - a.y * b.x; }  // math.py:10-12

struct Stack {
    int index[64];
    float dist[64];
};

// ---- bounding boxes (bvh.py:22-50, bvh3d.py:19-47) ----
template <typename V>
static inline void box_distance(V lo, V hi, V p, float *dmin, float *dmax) {
    V u = sub(lo, p), v = sub(p, hi);
    V z;
    memset(&z, 0, sizeof z);
    *dmin = norm(vmax(vmax(u, v), z));
    *dmax = norm(vmin(u, v));
}
static inline float hmax(V2 a) { return gq_max(a.x, a.y); }
static inline float hmin(V2 a) { return gq_min(a.x, a.y); }
static inline float hmax(V3 a) { return gq_max(gq_max(a.x, a.y), a.z); }
static inline float hmin(V3 a) { return gq_min(gq_min(a.x, a.y), a.z); }
static inline V2 vdiv(V2 a, V2 b) { return {a.x / b.x, a.y / b.y}; }
static inline V3 vdiv(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }

template <typename V>
static inline bool box_intersect(V lo, V hi, V x, V v, float r_max, float *t_min) {
    V t0 = vdiv(sub(lo, x), v), t1 = vdiv(sub(hi, x), v);
    V tn = vmin(t0, t1), tf = vmax(t0, t1);
    float tnm = gq_max(hmax(tn), 0.f);
    float tfm = gq_min(hmin(tf), r_max);
    if (tnm > tfm) {
        *t_min = INF;
        return false;
    }
    *t_min = tnm;
    return true;
}

// ---- reference node views ----
struct Node2 {
    V2 lo, hi;
    int off, sco, n;
};
static inline Node2 node2(const float *d, int i) {
    const float *p = d + 7 * (int64_t)i;
    return {{p[0], p[1]}, {p[2], p[3]}, I(p[4]), I(p[5]), I(p[6])};
}
struct Node3 {
    V3 lo, hi;
    int off, sco, n;
};
static inline Node3 node3(const float *d, int i) {
    const float *p = d + 9 * (int64_t)i;
    return {{p[0], p[1], p[2]}, {p[3], p[4], p[5]}, I(p[6]), I(p[7]), I(p[8])};
}
struct SNode2 {
    V2 lo, hi, axis;
    float half, radius;
    int off, sco, n, soff, ns;
};
static inline SNode2 snode2(const float *d, int i) {
    const float *p = d + 13 * (int64_t)i;
    return {{p[0], p[1]}, {p[2], p[3]}, {p[4], p[5]}, p[6], p[7], I(p[8]), I(p[9]), I(p[10]), I(p[11]), I(p[12])};
}
struct SNode3 {
    V3 lo, hi, axis;
    float half, radius;
    int off, sco, n, soff, ns;
};
static inline SNode3 snode3(const float *d, int i) {
    const float *p = d + 16 * (int64_t)i;
    return {{p[0], p[1], p[2]}, {p[3], p[4], p[5]}, {p[6], p[7], p[8]}, p[9], p[10],
            I(p[11]), I(p[12]), I(p[13]), I(p[14]), I(p[15])};
}

// ---- primitive math (core/math.py) ----
// closest_point_line_segment, math.py:15-21
template <typename V>
static inline float cp_segment(V x, V a, V b, V *pt, float *tt) {
    V u = sub(b, a), v = sub(x, a);
    float t = gq_clamp(gq_div(dot(v, u), dot(u, u)), 0.f, 1.f);
    V p;
    if constexpr (sizeof(V) == sizeof(V2)) {
        p = V{gq_lerp(a.x, b.x, t), gq_lerp(a.y, b.y, t)};
    } else {
        p = V{gq_lerp(a.x, b.x, t), gq_lerp(a.y, b.y, t), gq_lerp(a.z, b.z, t)};
    }
    if (pt) *pt = p;
    if (tt) *tt = t;
    return norm(sub(p, x));
}

// ray_intersection, math.py:32-39
static inline float ray_segment(V2 x, V2 v, V2 a, V2 b) {
    V2 u = sub(b, a), w = sub(x, a);
    float d = cross2(v, u);
    float s = cross2(v, w) / d;
    float t = cross2(u, w) / d;
    bool valid = (t > 0.f) & (s >= 0.f) & (s <= 1.f);
    return valid ? t : INF;
}

// closest_point_triangle, math.py:42-107
static inline float cp_triangle(V3 p, V3 a, V3 b, V3 c, V3 *pt_out, float *u_out, float *v_out) {
    V3 ab = sub(b, a), ac = sub(c, a);
    V3 ax = sub(p, a);
    float d1 = dot(ab, ax), d2 = dot(ac, ax);
    V3 pt;
    float uv0, uv1;
    V3 bx = sub(p, b);
    float d3 = dot(ab, bx), d4 = dot(ac, bx);
    V3 cx = sub(p, c);
    float d5 = dot(ab, cx), d6 = dot(ac, cx);
    if ((d1 <= 0.f) & (d2 <= 0.f)) {
        pt = a; uv0 = 1.f; uv1 = 0.f;
    } else if ((d3 >= 0.f) & (d4 <= d3)) {
        pt = b; uv0 = 0.f; uv1 = 1.f;
    } else if ((d6 >= 0.f) & (d5 <= d6)) {
        pt = c; uv0 = 0.f; uv1 = 0.f;
    } else {
        float vc = d1 * d4 - d3 * d2;
        float vb = d5 * d2 - d1 * d6;
        float va = d3 * d6 - d5 * d4;
        if ((vc <= 0.f) & (d1 >= 0.f) & (d3 <= 0.f)) {
            float v = d1 / (d1 - d3);
            pt = add(a, mul(ab, v)); uv0 = 1.f - v; uv1 = v;
        } else if ((vb <= 0.f) & (d2 >= 0.f) & (d6 <= 0.f)) {
            float w = d2 / (d2 - d6);
            pt = add(a, mul(ac, w)); uv0 = 1.f - w; uv1 = 0.f;
        } else if ((va <= 0.f) & ((d4 - d3) >= 0.f) & ((d5 - d6) >= 0.f)) {
            float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
            pt = add(b, mul(sub(c, b), w)); uv0 = 0.f; uv1 = 1.f - w;
        } else {
            float denom = 1.f / (va + vb + vc);
            float v = vb * denom, w = vc * denom;
            pt = add(add(a, mul(ab, v)), mul(ac, w)); uv0 = 1.f - v - w; uv1 = v;
        }
    }
    if (pt_out) {
        *pt_out = pt;
        *u_out = uv1;
        *v_out = 1.f - uv0 - uv1;
    }
    return norm(sub(p, pt));
}

// ray_triangle_intersect, math.py:110-128 (returns r_max when missed)
static inline float ray_triangle(V3 x, V3 d, V3 a, V3 b, V3 c, float r_max, float *vv, float *ww) {
    V3 v1 = sub(b, a), v2 = sub(c, a);
    V3 p = cross(d, v2);
    float det = dot(v1, p);
    if (fabsf(det) > GQ_EPS_F) {
        float inv_det = 1.f / det;
        V3 s = sub(x, a);
        float v = dot(s, p) * inv_det;
        if ((v >= 0.f) & (v <= 1.f)) {
            V3 q = cross(s, v1);
            float w = dot(d, q) * inv_det;
            if ((w >= 0.f) & (v + w <= 1.f)) {
                float t = dot(v2, q) * inv_det;
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

// ---- SNCH cone tests (snch.py:16-60, snch3d.py:12-30, 51-95) ----
static inline bool in_range(float x, float a, float b) { return (x >= a) & (x <= b); }

static inline float project_to_plane(V2 n, V2 e) {  // math.py:24-28
    V2 b = {-n.y, n.x};
    float r = dot(e, vabs(b));
    return fabsf(r);
}
static inline float project_to_plane(V3 n, V3 e) {  // snch3d.py:12-30
    float sign = copysignf(1.f, n.z);
    float a = -1.f / (sign + n.z);
    float b = n.x * n.y * a;
    V3 b1 = {1.f + sign * n.x * n.x * a, sign * b, -sign * n.x};
    V3 b2 = {b, sign + n.y * n.y * a, -n.y};
    float r1 = dot(e, vabs(b1));
    float r2 = dot(e, vabs(b2));
    return gq_sqrt(r1 * r1 + r2 * r2);
}

template <typename V, typename N>
static inline bool snch_overlaps(const N &nd, V x, float r_max, float *d_min_out) {
    float d_min, d_max;
    box_distance(nd.lo, nd.hi, x, &d_min, &d_max);
    bool is_overlap = d_min <= r_max;
    if ((nd.half >= 0.f) & is_overlap) {
        is_overlap = (nd.half > GQ_PIO2_F) & (d_min < GQ_EPS_F);
        if (!is_overlap) {
            V c = mul(add(nd.lo, nd.hi), 0.5f);  // (p_min + p_max) / 2
            V vca = sub(c, x);
            float l = norm(vca);
            if constexpr (sizeof(V) == sizeof(V2))
                vca = V{vca.x / l, vca.y / l};
            else
                vca = V{vca.x / l, vca.y / l, vca.z / l};
            float dA = gq_acos(gq_clamp(dot(nd.axis, vca), -1.f, 1.f));
            is_overlap = in_range(GQ_PIO2_F, dA - nd.half, dA + nd.half);
            if (!is_overlap) {
                if (l > nd.radius) {
                    float vch = gq_asin(nd.radius / l);
                    float hs = nd.half + vch;
                    is_overlap = (hs > GQ_PIO2_F) | in_range(GQ_PIO2_F, dA - hs, dA + hs);
                } else {
                    V e = sub(nd.hi, c);
                    float dd = dot(e, vabs(vca));
                    float s = l - dd;
                    is_overlap = s < 0.f;
                    if (!is_overlap) {
                        dd = project_to_plane(vca, e);
                        float vch = gq_atan2(dd, s);
                        float hs = nd.half + vch;
                        is_overlap = (hs > GQ_PIO2_F) | in_range(GQ_PIO2_F, dA - hs, dA + hs);
                    }
                }
            }
        }
    }
    *d_min_out = d_min;
    return is_overlap;
}

// ---------------------------------------------------------------------------
// Output rows.  f rows: cp2d [px py nx ny t d], cp3d [px py pz nx ny nz u v d],
// ray2d [px py nx ny t d], ray3d [px py pz nx ny nz u v d], sil2d [px py d],
// sil3d [px py pz d].  i rows: [valid prim_id on_boundary].  Misses are all zero.
// counts rows (optional): [interior nodes expanded, primitives/silhouettes tested].
// ---------------------------------------------------------------------------

struct Out {
    float *f;
    int32_t *i;
    int32_t *cnt;
    int kf;
};

// BVH.closest_point, bvh.py:127-198
static void cp2d_one(const float *N, const float *P, V2 p, Out o, int64_t q) {
    float r_max = INF;
    Stack st;
    int sp = 0;
    st.index[0] = 0;
    st.dist[0] = r_max;
    int idx = -1;
    int ni_exp = 0, np_test = 0;
    bool ovf = false;
    while (sp >= 0) {
        int ni = st.index[sp];
        float cd = st.dist[sp];
        sp -= 1;
        if (cd <= r_max) {
            Node2 nd = node2(N, ni);
            if (nd.n > 0) {
                for (int j = 0; j < nd.n; ++j) {
                    int ri = nd.off + j;
                    const float *s = P + 5 * (int64_t)ri;
                    float d = cp_segment(p, V2{s[0], s[1]}, V2{s[2], s[3]}, (V2 *)nullptr, nullptr);
                    np_test++;
                    if (d < r_max) {
                        r_max = d;
                        idx = ri;
                    }
                }
            } else {
                ni_exp++;
                Node2 L = node2(N, ni + 1), R = node2(N, ni + nd.sco);
                float dminl, dmaxl, dminr, dmaxr;
                box_distance(L.lo, L.hi, p, &dminl, &dmaxl);
                bool hl = dminl <= r_max;
                r_max = gq_min(r_max, dmaxl);
                box_distance(R.lo, R.hi, p, &dminr, &dmaxr);
                bool hr = dminr <= r_max;
                r_max = gq_min(r_max, dmaxr);
                if (hl & hr) {
                    int closer = ni + 1, other = ni + nd.sco;
                    if (dminr < dminl) {
                        std::swap(closer, other);
                        std::swap(dminl, dminr);
                    }
                    if (sp + 2 >= 64) {
                        ovf = true;
                        break;
                    }
                    st.index[++sp] = other;
                    st.dist[sp] = dminr;
                    st.index[++sp] = closer;
                    st.dist[sp] = dminl;
                } else if (hl) {
                    st.index[++sp] = ni + 1;
                    st.dist[sp] = dminl;
                } else if (hr) {
                    st.index[++sp] = ni + nd.sco;
                    st.dist[sp] = dminr;
                }
            }
        }
    }
    float *f = o.f + q * o.kf;
    int32_t *ii = o.i + q * 3;
    memset(f, 0, sizeof(float) * o.kf);
    ii[0] = ii[1] = ii[2] = 0;
    if (idx != -1) {  // LineSegment.closest_point, line_segment.py:64-78
        const float *s = P + 5 * (int64_t)idx;
        V2 a{s[0], s[1]}, b{s[2], s[3]};
        V2 pa = sub(p, a), ba = sub(b, a);
        V2 t = normalize(ba);
        float h = gq_clamp(gq_div(dot(pa, ba), dot(ba, ba)), 0.f, 1.f);
        V2 i = add(a, mul(ba, h));
        f[0] = i.x;
        f[1] = i.y;
        f[2] = t.y;
        f[3] = -t.x;
        f[4] = h;
        f[5] = norm(sub(i, p));
        ii[0] = 1;
        ii[1] = I(s[4]);
    }
    if (ovf) ii[0] = -1;  // stack overflow (deeper than the reference's 64-entry stack)
    if (o.cnt) {
        o.cnt[2 * q] = ni_exp;
        o.cnt[2 * q + 1] = np_test;
    }
}

// BVH3D.closest_point, bvh3d.py:108-174
static void cp3d_one(const float *N, const float *P, V3 p, Out o, int64_t q) {
    float r_max = INF;
    int idx = -1;
    Stack st;
    int sp = 0;
    st.index[0] = 0;
    st.dist[0] = r_max;
    int ni_exp = 0, np_test = 0;
    bool ovf = false;
    while (sp >= 0) {
        int ni = st.index[sp];
        float cd = st.dist[sp];
        sp -= 1;
        if (cd <= r_max) {
            Node3 nd = node3(N, ni);
            if (nd.n > 0) {
                for (int j = 0; j < nd.n; ++j) {
                    int ri = nd.off + j;
                    const float *t = P + 10 * (int64_t)ri;
                    float d = cp_triangle(p, V3{t[0], t[1], t[2]}, V3{t[3], t[4], t[5]}, V3{t[6], t[7], t[8]},
                                          nullptr, nullptr, nullptr);
                    np_test++;
                    if (d < r_max) {
                        r_max = d;
                        idx = ri;
                    }
                }
            } else {
                ni_exp++;
                Node3 L = node3(N, ni + 1), R = node3(N, ni + nd.sco);
                float dminl, dmaxl, dminr, dmaxr;
                box_distance(L.lo, L.hi, p, &dminl, &dmaxl);
                bool hl = dminl <= r_max;
                r_max = gq_min(r_max, dmaxl);
                box_distance(R.lo, R.hi, p, &dminr, &dmaxr);
                bool hr = dminr <= r_max;
                r_max = gq_min(r_max, dmaxr);
                if (hl & hr) {
                    int closer = ni + 1, other = ni + nd.sco;
                    if (dminr < dminl) {
                        std::swap(closer, other);
                        std::swap(dminl, dminr);
                    }
                    if (sp + 2 >= 64) {
                        ovf = true;
                        break;
                    }
                    st.index[++sp] = other;
                    st.dist[sp] = dminr;
                    st.index[++sp] = closer;
                    st.dist[sp] = dminl;
                } else if (hl) {
                    st.index[++sp] = ni + 1;
                    st.dist[sp] = dminl;
                } else if (hr) {
                    st.index[++sp] = ni + nd.sco;
                    st.dist[sp] = dminr;
                }
            }
        }
    }
    float *f = o.f + q * o.kf;
    int32_t *ii = o.i + q * 3;
    memset(f, 0, sizeof(float) * o.kf);
    ii[0] = ii[1] = ii[2] = 0;
    if (idx >= 0) {  // Triangle.closest_point, triangle.py:76-81
        const float *t = P + 10 * (int64_t)idx;
        V3 a{t[0], t[1], t[2]}, b{t[3], t[4], t[5]}, c{t[6], t[7], t[8]};
        V3 pt;
        float u, v;
        float d = cp_triangle(p, a, b, c, &pt, &u, &v);
        V3 n = normalize(cross(sub(b, a), sub(c, a)));
        f[0] = pt.x; f[1] = pt.y; f[2] = pt.z;
        f[3] = n.x; f[4] = n.y; f[5] = n.z;
        f[6] = u; f[7] = v; f[8] = d;
        ii[0] = 1;
        ii[1] = I(t[9]);
    }
    if (ovf) ii[0] = -1;  // stack overflow (deeper than the reference's 64-entry stack)
    if (o.cnt) {
        o.cnt[2 * q] = ni_exp;
        o.cnt[2 * q + 1] = np_test;
    }
}

// BVH.intersect, bvh.py:200-276
static void ray2d_one(const float *N, const float *P, V2 x, V2 v, float r_max, Out o, int64_t q) {
    Node2 root = node2(N, 0);
    float t_min;
    bool hit = box_intersect(root.lo, root.hi, x, v, r_max, &t_min);
    float d_min = r_max;
    int idx = -1;
    bool is_hit = false;
    int ni_exp = 0, np_test = 0;
    bool ovf = false;
    if (hit) {
        Stack st;
        int sp = 0;
        st.index[0] = 0;
        st.dist[0] = t_min;
        while (sp >= 0) {
            int ni = st.index[sp];
            float cd = st.dist[sp];
            sp -= 1;
            if (cd <= r_max) {
                Node2 nd = node2(N, ni);
                if (nd.n > 0) {
                    for (int j = 0; j < nd.n; ++j) {
                        int ri = nd.off + j;
                        const float *s = P + 5 * (int64_t)ri;
                        float d = ray_segment(x, v, V2{s[0], s[1]}, V2{s[2], s[3]});
                        np_test++;
                        if (d < d_min) {
                            d_min = d;
                            idx = ri;
                            is_hit = true;
                        }
                    }
                } else {
                    ni_exp++;
                    Node2 L = node2(N, ni + 1), R = node2(N, ni + nd.sco);
                    float t0, t1;
                    bool h0 = box_intersect(L.lo, L.hi, x, v, r_max, &t0);
                    bool h1 = box_intersect(R.lo, R.hi, x, v, r_max, &t1);
                    if (h0 & h1) {
                        int closer = ni + 1, other = ni + nd.sco;
                        if (t1 < t0) {
                            std::swap(closer, other);
                            std::swap(t0, t1);
                        }
                        if (sp + 2 >= 64) {
                        ovf = true;
                        break;
                    }
                        st.index[++sp] = other;
                        st.dist[sp] = t1;
                        st.index[++sp] = closer;
                        st.dist[sp] = t0;
                    } else if (h0) {
                        st.index[++sp] = ni + 1;
                        st.dist[sp] = t0;
                    } else if (h1) {
                        st.index[++sp] = ni + nd.sco;
                        st.dist[sp] = t1;
                    }
                }
            }
        }
    }
    float *f = o.f + q * o.kf;
    int32_t *ii = o.i + q * 3;
    memset(f, 0, sizeof(float) * o.kf);
    ii[0] = ii[1] = ii[2] = 0;
    if (is_hit) {
        const float *s = P + 5 * (int64_t)idx;
        V2 p = add(x, mul(v, d_min));
        V2 t = sub(V2{s[2], s[3]}, V2{s[0], s[1]});  // LineSegment.normal, line_segment.py:14-16
        V2 n = normalize(V2{t.y, -t.x});
        f[0] = p.x; f[1] = p.y; f[2] = n.x; f[3] = n.y;
        f[4] = -1.f;
        f[5] = d_min;
        ii[0] = 1;
        ii[1] = I(s[4]);
        ii[2] = 1;
    }
    if (ovf) ii[0] = -1;  // stack overflow (deeper than the reference's 64-entry stack)
    if (o.cnt) {
        o.cnt[2 * q] = ni_exp;
        o.cnt[2 * q + 1] = np_test;
    }
}

// BVH3D.intersect, bvh3d.py:176-239
static void ray3d_one(const float *N, const float *P, V3 x, V3 v, float r_max, Out o, int64_t q) {
    int idx = -1;
    Node3 root = node3(N, 0);
    float t_min;
    bool hit = box_intersect(root.lo, root.hi, x, v, r_max, &t_min);
    int ni_exp = 0, np_test = 0;
    bool ovf = false;
    if (hit) {
        Stack st;
        int sp = 0;
        st.index[0] = 0;
        st.dist[0] = t_min;
        while (sp >= 0) {
            int ni = st.index[sp];
            float cd = st.dist[sp];
            sp -= 1;
            if (cd <= r_max) {
                Node3 nd = node3(N, ni);
                if (nd.n > 0) {
                    for (int j = 0; j < nd.n; ++j) {
                        int ri = nd.off + j;
                        const float *t = P + 10 * (int64_t)ri;
                        float d = ray_triangle(x, v, V3{t[0], t[1], t[2]}, V3{t[3], t[4], t[5]},
                                               V3{t[6], t[7], t[8]}, INF, nullptr, nullptr);
                        np_test++;
                        if (d < r_max) {
                            r_max = d;
                            idx = ri;
                        }
                    }
                } else {
                    ni_exp++;
                    Node3 L = node3(N, ni + 1), R = node3(N, ni + nd.sco);
                    float t0, t1;
                    bool h0 = box_intersect(L.lo, L.hi, x, v, r_max, &t0);
                    bool h1 = box_intersect(R.lo, R.hi, x, v, r_max, &t1);
                    if (h0 & h1) {
                        int closer = ni + 1, other = ni + nd.sco;
                        if (t1 < t0) {
                            std::swap(closer, other);
                            std::swap(t0, t1);
                        }
                        if (sp + 2 >= 64) {
                        ovf = true;
                        break;
                    }
                        st.index[++sp] = other;
                        st.dist[sp] = t1;
                        st.index[++sp] = closer;
                        st.dist[sp] = t0;
                    } else if (h0) {
                        st.index[++sp] = ni + 1;
                        st.dist[sp] = t0;
                    } else if (h1) {
                        st.index[++sp] = ni + nd.sco;
                        st.dist[sp] = t1;
                    }
                }
            }
        }
    }
    float *f = o.f + q * o.kf;
    int32_t *ii = o.i + q * 3;
    memset(f, 0, sizeof(float) * o.kf);
    ii[0] = ii[1] = ii[2] = 0;
    if (idx >= 0) {  // Triangle.ray_intersect, triangle.py:49-73
        const float *t = P + 10 * (int64_t)idx;
        V3 a{t[0], t[1], t[2]}, b{t[3], t[4], t[5]}, c{t[6], t[7], t[8]};
        float vv = 0, ww = 0;
        float tt = ray_triangle(x, v, a, b, c, r_max, &vv, &ww);
        (void)tt;
        V3 v1 = sub(b, a), v2 = sub(c, a);
        V3 p = add(add(a, mul(v1, vv)), mul(v2, ww));
        V3 n = normalize(cross(v1, v2));
        f[0] = p.x; f[1] = p.y; f[2] = p.z;
        f[3] = n.x; f[4] = n.y; f[5] = n.z;
        f[6] = 1.f - vv - ww;
        f[7] = vv;
        f[8] = tt;
        ii[0] = 1;
        ii[1] = I(t[9]);
        ii[2] = 1;
    }
    if (ovf) ii[0] = -1;  // stack overflow (deeper than the reference's 64-entry stack)
    if (o.cnt) {
        o.cnt[2 * q] = ni_exp;
        o.cnt[2 * q + 1] = np_test;
    }
}

// SilhouetteVertex.closest_silhouette, silhouette_vertex.py:40-53
static inline bool sil_vertex(const float *s, V2 x, float r_max, V2 *p_out, float *d_out) {
    V2 a{s[0], s[1]}, b{s[2], s[3]}, c{s[4], s[5]};
    V2 p = b;
    float d = norm(sub(x, p));
    if ((I(s[6]) != -1) & (I(s[8]) != -1)) {
        if (d < r_max) {
            if (cross2(sub(b, a), sub(x, a)) * cross2(sub(c, b), sub(x, b)) < 0.f) {
                *p_out = p;
                *d_out = d;
                return true;
            }
        }
    }
    return false;
}

// SilhouetteEdge.closest_silhouette, silhouette_edge.py:50-64 (field order c, a, b, d)
static inline bool sil_edge(const float *s, V3 x, float r_max, V3 *p_out, float *d_out) {
    V3 c{s[0], s[1], s[2]}, a{s[3], s[4], s[5]}, b{s[6], s[7], s[8]}, dd{s[9], s[10], s[11]};
    V3 pt;
    float d = cp_segment(x, a, b, &pt, nullptr);
    if (d < r_max) {
        bool is_sil = (I(s[12]) == -1) | (I(s[15]) == -1);
        if (!is_sil) {
            V3 n0 = normalize(cross(sub(b, a), sub(c, a)));
            V3 n1 = normalize(cross(sub(dd, a), sub(b, a)));
            V3 view = sub(pt, x);
            float dot0 = dot(view, n0), dot1 = dot(view, n1);
            is_sil = dot0 * dot1 < 0.f;
        }
        if (is_sil) {
            *p_out = pt;
            *d_out = d;
            return true;
        }
    }
    return false;
}

// SNCH.closest_silhouette (snch.py:106-164) and SNCH3D.closest_silhouette (snch3d.py:143-203)
template <int D>
static void sil_one(const float *N, const float *S, const float *xq, float r_max, Out o, int64_t q) {
    using V = std::conditional_t<D == 2, V2, V3>;
    V x;
    memcpy(&x, xq, sizeof(V));
    bool found = false;
    V best_p;
    memset(&best_p, 0, sizeof best_p);
    float best_d = 0.f;
    int best_id = 0;
    int ni_exp = 0, np_test = 0;
    bool ovf = false;
    auto load = [&](int i) {
        if constexpr (D == 2)
            return snode2(N, i);
        else
            return snode3(N, i);
    };
    auto root = load(0);
    float d_min, d_max;
    box_distance(root.lo, root.hi, x, &d_min, &d_max);
    if (d_min <= r_max) {
        Stack st;
        int sp = 0;
        st.index[0] = 0;
        st.dist[0] = d_min;
        while (sp >= 0) {
            int ni = st.index[sp];
            float cd = st.dist[sp];
            sp -= 1;
            if (cd <= r_max) {
                auto nd = load(ni);
                if (nd.n > 0) {
                    for (int j = 0; j < nd.ns; ++j) {
                        int ri = nd.soff + j;
                        V p;
                        float d;
                        bool ok;
                        if constexpr (D == 2)
                            ok = sil_vertex(S + 10 * (int64_t)ri, x, r_max, &p, &d);
                        else
                            ok = sil_edge(S + 19 * (int64_t)ri, x, r_max, &p, &d);
                        np_test++;
                        if (ok && (d < r_max)) {
                            r_max = gq_min(r_max, d);
                            found = true;
                            best_p = p;
                            best_d = d;
                            best_id = (D == 2) ? I(S[10 * (int64_t)ri + 9]) : I(S[19 * (int64_t)ri + 18]);
                        }
                    }
                } else {
                    ni_exp++;
                    auto L = load(ni + 1), R = load(ni + nd.sco);
                    float d0, d1;
                    bool h0 = snch_overlaps<V>(L, x, r_max, &d0);
                    bool h1 = snch_overlaps<V>(R, x, r_max, &d1);
                    if (h0 & h1) {
                        int closer = ni + 1, other = ni + nd.sco;
                        if (d1 < d0) {
                            std::swap(closer, other);
                            std::swap(d0, d1);
                        }
                        if (sp + 2 >= 64) {
                        ovf = true;
                        break;
                    }
                        st.index[++sp] = other;
                        st.dist[sp] = d1;
                        st.index[++sp] = closer;
                        st.dist[sp] = d0;
                    } else if (h0) {
                        st.index[++sp] = ni + 1;
                        st.dist[sp] = d0;
                    } else if (h1) {
                        st.index[++sp] = ni + nd.sco;
                        st.dist[sp] = d1;
                    }
                }
            }
        }
    }
    float *f = o.f + q * o.kf;
    int32_t *ii = o.i + q * 3;
    memset(f, 0, sizeof(float) * o.kf);
    ii[0] = ii[1] = ii[2] = 0;
    if (found) {
        memcpy(f, &best_p, sizeof(V));
        f[D] = best_d;
        ii[0] = 1;
        ii[1] = best_id;
    }
    if (ovf) ii[0] = -1;  // stack overflow (deeper than the reference's 64-entry stack)
    if (o.cnt) {
        o.cnt[2 * q] = ni_exp;
        o.cnt[2 * q + 1] = np_test;
    }
}

template <typename F>
static void parallel_for(int64_t n, int nthreads, F fn) {
    if (nthreads <= 1 || n < 64) {
        for (int64_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::vector<std::thread> pool;
    const int64_t chunk = 256;
    std::atomic<int64_t> next{0};
    for (int t = 0; t < nthreads; ++t)
        pool.emplace_back([&]() {
            for (;;) {
                int64_t s = next.fetch_add(chunk);
                if (s >= n) break;
                int64_t e = std::min(n, s + chunk);
                for (int64_t i = s; i < e; ++i) fn(i);
            }
        });
    for (auto &th : pool) th.join();
}

// ---- FP64 brute force ----
struct D2 {
    double x, y;
};
struct D3 {
    double x, y, z;
};
static inline double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline D3 dsub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline D3 dcross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

static double d_cp_triangle(D3 p, D3 a, D3 b, D3 c) {
    D3 ab = dsub(b, a), ac = dsub(c, a), ap = dsub(p, a);
    double d1 = ddot(ab, ap), d2 = ddot(ac, ap);
    auto dist = [&](D3 q) { D3 e = dsub(p, q); return sqrt(ddot(e, e)); };
    if (d1 <= 0 && d2 <= 0) return dist(a);
    D3 bp = dsub(p, b);
    double d3 = ddot(ab, bp), d4 = ddot(ac, bp);
    if (d3 >= 0 && d4 <= d3) return dist(b);
    double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) {
        double v = d1 / (d1 - d3);
        return dist(D3{a.x + v * ab.x, a.y + v * ab.y, a.z + v * ab.z});
    }
    D3 cp = dsub(p, c);
    double d5 = ddot(ab, cp), d6 = ddot(ac, cp);
    if (d6 >= 0 && d5 <= d6) return dist(c);
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) {
        double w = d2 / (d2 - d6);
        return dist(D3{a.x + w * ac.x, a.y + w * ac.y, a.z + w * ac.z});
    }
    double va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
        double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        return dist(D3{b.x + w * (c.x - b.x), b.y + w * (c.y - b.y), b.z + w * (c.z - b.z)});
    }
    double den = 1.0 / (va + vb + vc);
    double v = vb * den, w = vc * den;
    return dist(D3{a.x + ab.x * v + ac.x * w, a.y + ab.y * v + ac.y * w, a.z + ab.z * v + ac.z * w});
}

// ---- FP32 brute force: the reference's *_baseline scans over the raw primitives ----
// Records are written in the row layout of the traversals (Out.kf floats, 3 ints);
// a scan that keeps no primitive leaves the zeroed record.
static inline V2 vtx2(const float *V, const int32_t *E, int64_t e, int k) {
    const int64_t i = E[2 * e + k];
    return V2{V[2 * i], V[2 * i + 1]};
}
static inline V3 vtx3(const float *V, const int32_t *F, int64_t f, int k) {
    const int64_t i = F[3 * f + k];
    return V3{V[3 * i], V[3 * i + 1], V[3 * i + 2]};
}

// Polyline.closest_point_baseline, polyline.py:175-209
static void cp_brute2d_one(const float *V, const int32_t *E, int64_t ne, V2 p, Out o, int64_t q) {
    float d_min = INF;
    int64_t idx = -1;
    for (int64_t i = 0; i < ne; ++i) {
        const V2 a = vtx2(V, E, i, 0), b = vtx2(V, E, i, 1);
        const V2 pa = sub(p, a), ba = sub(b, a);
        const float h = gq_clamp(gq_div(dot(pa, ba), dot(ba, ba)), 0.f, 1.f);
        const float d = norm(sub(pa, mul(ba, h)));
        if (d < d_min) {
            d_min = d;
            idx = i;
        }
    }
    float *f = o.f + q * o.kf;
    int32_t *ii = o.i + q * 3;
    memset(f, 0, sizeof(float) * o.kf);
    ii[0] = ii[1] = ii[2] = 0;
    if (idx == -1) return;
    const V2 a = vtx2(V, E, idx, 0), b = vtx2(V, E, idx, 1);
    const V2 pa = sub(p, a), ba = sub(b, a);
    const float h = gq_clamp(gq_div(dot(pa, ba), dot(ba, ba)), 0.f, 1.f);  // dr.clip
    const V2 n = normalize(V2{ba.y, -ba.x});
    f[0] = gq_lerp(a.x, b.x, h);
    f[1] = gq_lerp(a.y, b.y, h);
    f[2] = n.x;
    f[3] = n.y;
    f[4] = h;
    f[5] = d_min;
    ii[0] = 1;
    ii[1] = (int32_t)idx;
}

// Mesh.closest_point_baseline, mesh.py:91-117; the normal is the face normal of
// Mesh.configure_normal (mesh.py:35-40), normalize(cross(b - a, c - a)).
static void cp_brute3d_one(const float *V, const int32_t *F, int64_t nf, V3 x, Out o, int64_t q) {
    float d_min = INF;
    int64_t idx = -1;
    for (int64_t i = 0; i < nf; ++i) {
        const float d = cp_triangle(x, vtx3(V, F, i, 0), vtx3(V, F, i, 1), vtx3(V, F, i, 2), nullptr, nullptr, nullptr);
        if (d < d_min) {
            d_min = d;
            idx = i;
        }
    }
    float *f = o.f + q * o.kf;
    int32_t *ii = o.i + q * 3;
    memset(f, 0, sizeof(float) * o.kf);
    ii[0] = ii[1] = ii[2] = 0;
    if (idx == -1) return;
    const V3 a = vtx3(V, F, idx, 0), b = vtx3(V, F, idx, 1), c = vtx3(V, F, idx, 2);
    V3 pt;
    float u, v;
    cp_triangle(x, a, b, c, &pt, &u, &v);
    const V3 n = normalize(cross(sub(b, a), sub(c, a)));
    f[0] = pt.x, f[1] = pt.y, f[2] = pt.z;
    f[3] = n.x, f[4] = n.y, f[5] = n.z;
    f[6] = u, f[7] = v;
    f[8] = d_min;
    ii[0] = 1;
    ii[1] = (int32_t)idx;
}

// Polyline.intersect_baseline, polyline.py:137-169: d_min starts at r_max, the first
// strictly nearest hit is kept; the record has p = x + v d, t = -1, on_boundary set.
static void ray_brute2d_one(const float *V, const int32_t *E, int64_t ne, V2 x, V2 v, float r_max, Out o, int64_t q) {
    float d_min = r_max;
    int64_t idx = -1;
    for (int64_t i = 0; i < ne; ++i) {
        const float d = ray_segment(x, v, vtx2(V, E, i, 0), vtx2(V, E, i, 1));
        if (d < d_min) {
            d_min = d;
            idx = i;
        }
    }
    float *f = o.f + q * o.kf;
    int32_t *ii = o.i + q * 3;
    memset(f, 0, sizeof(float) * o.kf);
    ii[0] = ii[1] = ii[2] = 0;
    if (idx == -1) return;
    const V2 a = vtx2(V, E, idx, 0), b = vtx2(V, E, idx, 1);
    const V2 ab = normalize(sub(b, a));
    const V2 p = add(x, mul(v, d_min));
    f[0] = p.x, f[1] = p.y;
    f[2] = ab.y, f[3] = -ab.x;
    f[4] = -1.f;
    f[5] = d_min;
    ii[0] = 1;
    ii[1] = (int32_t)idx;
    ii[2] = 1;
}

// Triangle.ray_intersect, triangle.py:48-73: whether the ray hits within [0, r_max],
// with the barycentric v, w and the parameter t of the hit.
static inline bool tri_hit(V3 x, V3 d, V3 a, V3 b, V3 c, float r_max, float *t, float *v, float *w) {
    float vv = NAN, ww = 0.f;
    const float tt = ray_triangle(x, d, a, b, c, r_max, &vv, &ww);
    if (vv != vv) return false;
    *t = tt, *v = vv, *w = ww;
    return true;
}

// Mesh.intersect_baseline, mesh.py:60-84: every triangle is tested against the
// caller's r_max, a hit is kept when nearer than the best so far, and the record is
// the kept triangle's ray_intersect at the caller's r_max again.
static void ray_brute3d_one(const float *V, const int32_t *F, int64_t nf, V3 x, V3 dir, float r_max, Out o,
                            int64_t q) {
    float d_min = r_max;
    int64_t idx = -1;
    for (int64_t i = 0; i < nf; ++i) {
        float t, v, w;
        if (tri_hit(x, dir, vtx3(V, F, i, 0), vtx3(V, F, i, 1), vtx3(V, F, i, 2), r_max, &t, &v, &w) && t < d_min) {
            idx = i;
            d_min = t;
        }
    }
    float *f = o.f + q * o.kf;
    int32_t *ii = o.i + q * 3;
    memset(f, 0, sizeof(float) * o.kf);
    ii[0] = ii[1] = ii[2] = 0;
    if (idx == -1) return;
    const V3 a = vtx3(V, F, idx, 0), b = vtx3(V, F, idx, 1), c = vtx3(V, F, idx, 2);
    float t, v, w;
    if (!tri_hit(x, dir, a, b, c, r_max, &t, &v, &w)) return;
    const V3 v1 = sub(b, a), v2 = sub(c, a);
    const V3 p = add(add(a, mul(v1, v)), mul(v2, w));
    const V3 n = normalize(cross(v1, v2));
    f[0] = p.x, f[1] = p.y, f[2] = p.z;
    f[3] = n.x, f[4] = n.y, f[5] = n.z;
    f[6] = 1.f - v - w, f[7] = v;
    f[8] = t;
    ii[0] = 1;
    ii[1] = (int32_t)idx;
    ii[2] = 1;
}

}  // namespace

// closest_silhouette_baseline (mesh.py:124-135, polyline.py:212-223): the shape's
// silhouette list in order, the first strictly nearest silhouette kept.  The per-
// silhouette test is called with the current minimum as its r_max, which accepts
// exactly what "valid and d < d_min" accepts.
template <int D>
static void sil_brute_one(const float *S, int64_t n_sil, const float *xq, float r_max, Out o, int64_t q) {
    using V = std::conditional_t<D == 2, V2, V3>;
    V x;
    memcpy(&x, xq, sizeof(V));
    float d_min = r_max;
    bool found = false;
    V best_p;
    memset(&best_p, 0, sizeof best_p);
    float best_d = 0.f;
    int best_id = 0;
    for (int64_t j = 0; j < n_sil; ++j) {
        V p;
        float d;
        bool ok;
        if constexpr (D == 2)
            ok = sil_vertex(S + 10 * j, x, d_min, &p, &d);
        else
            ok = sil_edge(S + 19 * j, x, d_min, &p, &d);
        if (ok && d < d_min) {
            d_min = d;
            found = true;
            best_p = p;
            best_d = d;
            best_id = (D == 2) ? I(S[10 * j + 9]) : I(S[19 * j + 18]);
        }
    }
    float *f = o.f + q * o.kf;
    int32_t *ii = o.i + q * 3;
    memset(f, 0, sizeof(float) * o.kf);
    ii[0] = ii[1] = ii[2] = 0;
    if (found) {
        memcpy(f, &best_p, sizeof(V));
        f[D] = best_d;
        ii[0] = 1;
        ii[1] = best_id;
    }
}

// Polyline.configure_silhouette (polyline.py:44-122) as 10-float SilhouetteVertex
// records (a, b, c, indices, index): vertices in order of first appearance in the edge
// list with both a predecessor and a successor, nearly collinear ones dropped.
static std::vector<float> polyline_silhouettes(const float *V, int64_t nv, const int32_t *E, int64_t ne) {
    std::vector<int64_t> prev((size_t)nv, -1), next((size_t)nv, -1), order;
    std::vector<char> seen((size_t)nv, 0);
    for (int64_t e = 0; e < ne; ++e) {
        const int64_t a = E[2 * e], b = E[2 * e + 1];
        if (!seen[(size_t)a]) seen[(size_t)a] = 1, order.push_back(a);
        if (!seen[(size_t)b]) seen[(size_t)b] = 1, order.push_back(b);
        next[(size_t)a] = b;
        prev[(size_t)b] = a;
    }
    std::vector<float> r;
    for (size_t i = 0; i < order.size(); ++i) {
        const int64_t c = order[i], p = prev[(size_t)c], n = next[(size_t)c];
        if (p == -1 || n == -1) continue;
        const V2 p0{V[2 * p], V[2 * p + 1]}, p1{V[2 * c], V[2 * c + 1]}, p2{V[2 * n], V[2 * n + 1]};
        const float col = fabsf(dot(normalize(sub(p1, p0)), normalize(sub(p2, p1))));
        if (!(col < 0.99999f)) continue;
        const float rec[10] = {p0.x, p0.y, p1.x, p1.y, p2.x, p2.y, (float)p, (float)c, (float)n, (float)i};
        r.insert(r.end(), rec, rec + 10);
    }
    return r;
}

extern "C" {

int orc_version(void) { return 1; }

// The shared fixed-semantics math of gq_fmath.h, for accuracy tests.
// which: 0 acos(x), 1 asin(x), 2 atan2(x, y)
void orc_fmath(int which, const float *x, const float *y, float *out, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        if (which == 0)
            out[i] = gq_acos(x[i]);
        else if (which == 1)
            out[i] = gq_asin(x[i]);
        else
            out[i] = gq_atan2(x[i], y[i]);
    }
}

// Reference-layout traversals.  q: [nq][D] (AoS).  r_max: nullable (+inf).
// f_out: [nq][kf], i_out: [nq][3], counts: nullable [nq][2].
void orc_cp2d(const float *N, const float *P, const float *q, int64_t nq, float *f_out, int32_t *i_out,
              int32_t *counts, int nthreads) {
    Out o{f_out, i_out, counts, 6};
    parallel_for(nq, nthreads, [&](int64_t i) { cp2d_one(N, P, V2{q[2 * i], q[2 * i + 1]}, o, i); });
}
void orc_cp3d(const float *N, const float *P, const float *q, int64_t nq, float *f_out, int32_t *i_out,
              int32_t *counts, int nthreads) {
    Out o{f_out, i_out, counts, 9};
    parallel_for(nq, nthreads,
                 [&](int64_t i) { cp3d_one(N, P, V3{q[3 * i], q[3 * i + 1], q[3 * i + 2]}, o, i); });
}
void orc_ray2d(const float *N, const float *P, const float *x, const float *v, const float *rmax, int64_t nq,
               float *f_out, int32_t *i_out, int32_t *counts, int nthreads) {
    Out o{f_out, i_out, counts, 6};
    parallel_for(nq, nthreads, [&](int64_t i) {
        ray2d_one(N, P, V2{x[2 * i], x[2 * i + 1]}, V2{v[2 * i], v[2 * i + 1]}, rmax ? rmax[i] : INF, o, i);
    });
}
void orc_ray3d(const float *N, const float *P, const float *x, const float *v, const float *rmax, int64_t nq,
               float *f_out, int32_t *i_out, int32_t *counts, int nthreads) {
    Out o{f_out, i_out, counts, 9};
    parallel_for(nq, nthreads, [&](int64_t i) {
        ray3d_one(N, P, V3{x[3 * i], x[3 * i + 1], x[3 * i + 2]}, V3{v[3 * i], v[3 * i + 1], v[3 * i + 2]},
                  rmax ? rmax[i] : INF, o, i);
    });
}
void orc_sil2d(const float *N, const float *S, const float *x, const float *rmax, int64_t nq, float *f_out,
               int32_t *i_out, int32_t *counts, int nthreads) {
    Out o{f_out, i_out, counts, 3};
    parallel_for(nq, nthreads, [&](int64_t i) { sil_one<2>(N, S, x + 2 * i, rmax ? rmax[i] : INF, o, i); });
}
void orc_sil3d(const float *N, const float *S, const float *x, const float *rmax, int64_t nq, float *f_out,
               int32_t *i_out, int32_t *counts, int nthreads) {
    Out o{f_out, i_out, counts, 4};
    parallel_for(nq, nthreads, [&](int64_t i) { sil_one<3>(N, S, x + 3 * i, rmax ? rmax[i] : INF, o, i); });
}

void orc_sil_brute2d(const float *V, int64_t nv, const int32_t *E, int64_t ne, const float *x, const float *rmax,
                     int64_t nq, float *f_out, int32_t *i_out, int nthreads) {
    const std::vector<float> S = polyline_silhouettes(V, nv, E, ne);
    const int64_t n_sil = (int64_t)S.size() / 10;
    Out o{f_out, i_out, nullptr, 3};
    parallel_for(nq, nthreads,
                 [&](int64_t i) { sil_brute_one<2>(S.data(), n_sil, x + 2 * i, rmax ? rmax[i] : INF, o, i); });
}
void orc_sil_brute3d(const float *S, int64_t n_sil, const float *x, const float *rmax, int64_t nq, float *f_out,
                     int32_t *i_out, int nthreads) {
    Out o{f_out, i_out, nullptr, 4};
    parallel_for(nq, nthreads, [&](int64_t i) { sil_brute_one<3>(S, n_sil, x + 3 * i, rmax ? rmax[i] : INF, o, i); });
}

// FP32 *_baseline scans over the raw primitives (verts [nv][D], idx [np][D]), records in
// the traversal row layout.  rmax: nullable (+inf).
void orc_cp_brute2d(const float *verts, const int32_t *idx, int64_t np, const float *q, int64_t nq, float *f_out,
                    int32_t *i_out, int nthreads) {
    Out o{f_out, i_out, nullptr, 6};
    parallel_for(nq, nthreads, [&](int64_t i) { cp_brute2d_one(verts, idx, np, V2{q[2 * i], q[2 * i + 1]}, o, i); });
}
void orc_cp_brute3d(const float *verts, const int32_t *idx, int64_t np, const float *q, int64_t nq, float *f_out,
                    int32_t *i_out, int nthreads) {
    Out o{f_out, i_out, nullptr, 9};
    parallel_for(nq, nthreads, [&](int64_t i) {
        cp_brute3d_one(verts, idx, np, V3{q[3 * i], q[3 * i + 1], q[3 * i + 2]}, o, i);
    });
}
void orc_ray_brute2d(const float *verts, const int32_t *idx, int64_t np, const float *x, const float *v,
                     const float *rmax, int64_t nq, float *f_out, int32_t *i_out, int nthreads) {
    Out o{f_out, i_out, nullptr, 6};
    parallel_for(nq, nthreads, [&](int64_t i) {
        ray_brute2d_one(verts, idx, np, V2{x[2 * i], x[2 * i + 1]}, V2{v[2 * i], v[2 * i + 1]}, rmax ? rmax[i] : INF,
                        o, i);
    });
}
void orc_ray_brute3d(const float *verts, const int32_t *idx, int64_t np, const float *x, const float *v,
                     const float *rmax, int64_t nq, float *f_out, int32_t *i_out, int nthreads) {
    Out o{f_out, i_out, nullptr, 9};
    parallel_for(nq, nthreads, [&](int64_t i) {
        ray_brute3d_one(verts, idx, np, V3{x[3 * i], x[3 * i + 1], x[3 * i + 2]},
                        V3{v[3 * i], v[3 * i + 1], v[3 * i + 2]}, rmax ? rmax[i] : INF, o, i);
    });
}

// FP64 brute force over the raw (unordered) primitives.  verts [nv][D], idx [np][D].
// out_d: nearest distance (cp) / nearest ray parameter (ray, +inf if none);
// out_id: original primitive index (-1 if none).
void orc_brute_cp3d(const float *verts, const int32_t *idx, int64_t np, const float *q, int64_t nq,
                    double *out_d, int32_t *out_id, int nthreads) {
    parallel_for(nq, nthreads, [&](int64_t i) {
        D3 p{q[3 * i], q[3 * i + 1], q[3 * i + 2]};
        double best = INFINITY;
        int32_t bid = -1;
        for (int64_t f = 0; f < np; ++f) {
            auto V = [&](int k) {
                int64_t vi = idx[3 * f + k];
                return D3{verts[3 * vi], verts[3 * vi + 1], verts[3 * vi + 2]};
            };
            double d = d_cp_triangle(p, V(0), V(1), V(2));
            if (d < best) {
                best = d;
                bid = (int32_t)f;
            }
        }
        out_d[i] = best;
        out_id[i] = bid;
    });
}

void orc_brute_cp2d(const float *verts, const int32_t *idx, int64_t np, const float *q, int64_t nq,
                    double *out_d, int32_t *out_id, int nthreads) {
    parallel_for(nq, nthreads, [&](int64_t i) {
        D2 p{q[2 * i], q[2 * i + 1]};
        double best = INFINITY;
        int32_t bid = -1;
        for (int64_t e = 0; e < np; ++e) {
            int64_t i0 = idx[2 * e], i1 = idx[2 * e + 1];
            D2 a{verts[2 * i0], verts[2 * i0 + 1]}, b{verts[2 * i1], verts[2 * i1 + 1]};
            double ux = b.x - a.x, uy = b.y - a.y, vx = p.x - a.x, vy = p.y - a.y;
            double uu = ux * ux + uy * uy;
            double t = uu > 0 ? (vx * ux + vy * uy) / uu : 0.0;
            t = t < 0 ? 0 : (t > 1 ? 1 : t);
            double dx = a.x + t * ux - p.x, dy = a.y + t * uy - p.y;
            double d = sqrt(dx * dx + dy * dy);
            if (d < best) {
                best = d;
                bid = (int32_t)e;
            }
        }
        out_d[i] = best;
        out_id[i] = bid;
    });
}

void orc_brute_ray3d(const float *verts, const int32_t *idx, int64_t np, const float *x, const float *v,
                     int64_t nq, double *out_t, int32_t *out_id, int nthreads) {
    parallel_for(nq, nthreads, [&](int64_t i) {
        D3 o{x[3 * i], x[3 * i + 1], x[3 * i + 2]}, d{v[3 * i], v[3 * i + 1], v[3 * i + 2]};
        double best = INFINITY;
        int32_t bid = -1;
        for (int64_t f = 0; f < np; ++f) {
            auto V = [&](int k) {
                int64_t vi = idx[3 * f + k];
                return D3{verts[3 * vi], verts[3 * vi + 1], verts[3 * vi + 2]};
            };
            D3 a = V(0), b = V(1), c = V(2);
            D3 e1 = dsub(b, a), e2 = dsub(c, a);
            D3 p = dcross(d, e2);
            double det = ddot(e1, p);
            if (fabs(det) <= 1e-300) continue;
            double inv = 1.0 / det;
            D3 s = dsub(o, a);
            double uu = ddot(s, p) * inv;
            if (uu < 0 || uu > 1) continue;
            D3 qv = dcross(s, e1);
            double vv = ddot(d, qv) * inv;
            if (vv < 0 || uu + vv > 1) continue;
            double t = ddot(e2, qv) * inv;
            if (t >= 0 && t < best) {
                best = t;
                bid = (int32_t)f;
            }
        }
        out_t[i] = best;
        out_id[i] = bid;
    });
}

}  // extern "C"
