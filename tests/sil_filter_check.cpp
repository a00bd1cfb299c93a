// Soundness check of the silhouette-edge pre-test (gquery_b200/csrc/sil_filter.h):
// over random and adversarial edges and query points, the pre-test must never
// exclude an edge that the reference's test (silhouette_edge.py:7-12, 50-64, in the
// FP32 operations the kernels use) calls a silhouette.  Prints one JSON line with the
// counts per regime; a non-zero "unsound" is a failure.  The node regimes check the
// node bound the same way over whole patches of edges.  An optional second argument
// scales the margin (0 removes it: the check must then find unsound exclusions, which
// shows that its cases reach the rounding boundary the margin covers).
//
// Build: g++ -O2 -ffp-contract=off -I gquery_b200/csrc tests/sil_filter_check.cpp
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <utility>
#include <vector>

#include "gq_fmath.h"
#include "sil_filter.h"
#include "sil_ref.h"

namespace {

struct Rng {
    uint64_t s;
    uint64_t next() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return s;
    }
    float uni(float lo, float hi) { return lo + (hi - lo) * (float)((next() >> 11) * (1.0 / 9007199254740992.0)); }
    float logu(float lo, float hi) { return std::exp(uni(std::log(lo), std::log(hi))); }
    float sgn() { return (next() & 1) ? 1.f : -1.f; }
};

V add(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V sub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V mul(V a, float s) { return {a.x * s, a.y * s, a.z * s}; }
float amax(V a) { return std::fmax(std::fabs(a.x), std::fmax(std::fabs(a.y), std::fabs(a.z))); }
V rand_in(Rng &r, float s) { return {r.uni(-s, s), r.uni(-s, s), r.uni(-s, s)}; }
V unit(V a) {
    const double l = std::sqrt((double)a.x * a.x + (double)a.y * a.y + (double)a.z * a.z);
    return {(float)(a.x / l), (float)(a.y / l), (float)(a.z / l)};
}
V cross(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

struct Count {
    long long cases = 0, usable = 0, excluded = 0, silhouettes = 0, unsound = 0;
};

// Edge (a, b) with faces (a, b, c) and (a, d, b), queried at x; `bound` is the scene's
// largest |coordinate| (at least that of a, b, c, d).
float g_margin_scale = 1.f;

void check(V a, V b, V c, V d, V x, float bound, Count &k) {
    V n0, n1;
    sil_face_normal(b.x - a.x, b.y - a.y, b.z - a.z, c.x - a.x, c.y - a.y, c.z - a.z, n0.x, n0.y, n0.z);
    sil_face_normal(d.x - a.x, d.y - a.y, d.z - a.z, b.x - a.x, b.y - a.y, b.z - a.z, n1.x, n1.y, n1.z);
    const float s0 = sil_span(n0.x, n0.y, n0.z, a.x, a.y, a.z, b.x, b.y, b.z);
    const float s1 = sil_span(n1.x, n1.y, n1.z, a.x, a.y, a.z, b.x, b.y, b.z);
    const bool sil = reference_silhouette(a, b, n0, n1, x);
    ++k.cases;
    k.silhouettes += sil;
    if (!sil_filter_usable(n0.x, n0.y, n0.z, n1.x, n1.y, n1.z, s0, s1)) return;
    ++k.usable;
    const float m = g_margin_scale * sil_margin(amax(x), bound);
    const bool ex = sil_edge_excluded(a.x, a.y, a.z, n0.x, n0.y, n0.z, n1.x, n1.y, n1.z, s0, s1, x.x, x.y, x.z, m);
    k.excluded += ex;
    if (ex && sil) {
        if (k.unsound < 3 && g_margin_scale == 1.f)
            std::fprintf(stderr, "unsound: a=(%a %a %a) b=(%a %a %a) c=(%a %a %a) d=(%a %a %a) x=(%a %a %a)\n", a.x,
                         a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z, d.x, d.y, d.z, x.x, x.y, x.z);
        ++k.unsound;
    }
}

float bound_of(V a, V b, V c, V d) { return std::fmax(std::fmax(amax(a), amax(b)), std::fmax(amax(c), amax(d))); }

void print(const char *name, const Count &k, bool last) {
    std::printf("\"%s\": {\"cases\": %lld, \"usable\": %lld, \"excluded\": %lld, \"silhouettes\": %lld, "
                "\"unsound\": %lld}%s",
                name, k.cases, k.usable, k.excluded, k.silhouettes, k.unsound, last ? "" : ", ");
}


// Node bound: a patch of a height field z = h(x, y) (smooth waves plus noise of a
// chosen amplitude, or steep waves whose slopes reach `steep` radians), or a spherical
// cap (normals spread up to `cap` radians from its axis), triangulated consistently; every interior edge is a silhouette
// record whose end points are stored in winding order (orientation +1) or swapped
// (both stored normals point the other way, orientation -1), as the reference's
// records come.  The patch is placed with a random rotation, scale and offset.
struct Patch {
    std::vector<SilEdgeGeom> edges;
    float c[3];
    float bound;  // largest |coordinate|
    V sphere;     // centre of the cap's sphere (cap patches)
    V axis;       // the patch's unit z axis
};

V rot(V v, const float R[9]) {
    return {R[0] * v.x + R[1] * v.y + R[2] * v.z, R[3] * v.x + R[4] * v.y + R[5] * v.z,
            R[6] * v.x + R[7] * v.y + R[8] * v.z};
}

Patch make_patch(Rng &r, int g, float rough, float cap = 0.f, float steep = 0.f) {
    // random rotation from a random unit quaternion
    float q0 = r.uni(-1, 1), q1 = r.uni(-1, 1), q2 = r.uni(-1, 1), q3 = r.uni(-1, 1);
    const float qn = std::sqrt(q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3);
    q0 /= qn; q1 /= qn; q2 /= qn; q3 /= qn;
    const float R[9] = {1 - 2 * (q2 * q2 + q3 * q3), 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2),
                        2 * (q1 * q2 + q0 * q3), 1 - 2 * (q1 * q1 + q3 * q3), 2 * (q2 * q3 - q0 * q1),
                        2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), 1 - 2 * (q1 * q1 + q2 * q2)};
    const float s = r.logu(1e-2f, 1e2f);
    const V off = mul(rand_in(r, 1.f), s * r.uni(0.f, 3.f));
    const float w1 = r.uni(0.5f, 4.f), w2 = r.uni(0.5f, 4.f), amp = r.uni(0.f, 0.3f);
    std::vector<V> p((size_t)(g + 1) * (g + 1));
    const float tc = std::tan(cap) / std::sqrt(2.f);  // the cap's corners lie `cap` off its axis
    for (int i = 0; i <= g; ++i)
        for (int j = 0; j <= g; ++j) {
            const float u = (float)i / g, v = (float)j / g;
            V q;
            if (cap > 0.f) {
                q = unit(V{2.f * (u - 0.5f) * tc, 2.f * (v - 0.5f) * tc, 1.f});
            } else if (steep > 0.f) {  // slope up to tan(steep) along u
                const float w = 2.f * (float)g;
                q = V{u - 0.5f, v - 0.5f, std::tan(steep) / w * std::sin(w * u + 1.3f)};
            } else {
                const float z = amp * std::sin(w1 * u + 1.3f) * std::cos(w2 * v) + rough * r.uni(-1.f, 1.f) / g;
                q = V{u - 0.5f, v - 0.5f, z};
            }
            p[(size_t)i * (g + 1) + j] = add(mul(rot(q, R), s), off);
        }
    auto at = [&](int i, int j) { return p[(size_t)i * (g + 1) + j]; };
    Patch P;
    P.sphere = off;
    P.axis = rot(V{0.f, 0.f, 1.f}, R);
    // triangles (i,j),(i+1,j),(i+1,j+1) and (i,j),(i+1,j+1),(i,j+1); interior diagonal and
    // grid edges with their two faces in winding order: edge a->b of face (a, b, c), the
    // other face (b, a, d)
    auto add_edge = [&](V a, V b, V c, V d) {
        SilEdgeGeom e;
        const bool swap = r.next() & 1;
        if (swap) std::swap(a, b);
        e.a[0] = a.x; e.a[1] = a.y; e.a[2] = a.z;
        e.b[0] = b.x; e.b[1] = b.y; e.b[2] = b.z;
        sil_face_normal(b.x - a.x, b.y - a.y, b.z - a.z, c.x - a.x, c.y - a.y, c.z - a.z, e.n0[0], e.n0[1], e.n0[2]);
        sil_face_normal(d.x - a.x, d.y - a.y, d.z - a.z, b.x - a.x, b.y - a.y, b.z - a.z, e.n1[0], e.n1[1], e.n1[2]);
        e.orient = swap ? -1.f : 1.f;
        const float s0 = sil_span(e.n0[0], e.n0[1], e.n0[2], a.x, a.y, a.z, b.x, b.y, b.z);
        const float s1 = sil_span(e.n1[0], e.n1[1], e.n1[2], a.x, a.y, a.z, b.x, b.y, b.z);
        e.usable = sil_filter_usable(e.n0[0], e.n0[1], e.n0[2], e.n1[0], e.n1[1], e.n1[2], s0, s1);
        P.edges.push_back(e);
    };
    for (int i = 0; i < g; ++i)
        for (int j = 0; j < g; ++j) {
            // diagonal (i,j)-(i+1,j+1) between the two triangles of the cell
            add_edge(at(i, j), at(i + 1, j + 1), at(i, j + 1), at(i + 1, j));
            if (i + 1 < g) add_edge(at(i + 1, j), at(i + 1, j + 1), at(i, j), at(i + 2, j + 1));
            if (j + 1 < g) add_edge(at(i, j + 1), at(i + 1, j + 1), at(i + 1, j + 2), at(i, j));
        }
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    P.bound = 0.f;
    for (const V &v : p) {
        const float w[3] = {v.x, v.y, v.z};
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::fmin(lo[k], w[k]);
            hi[k] = std::fmax(hi[k], w[k]);
        }
        P.bound = std::fmax(P.bound, amax(v));
    }
    for (int k = 0; k < 3; ++k) P.c[k] = sil_node_centre(lo[k], hi[k]);
    return P;
}

struct NodeCount {
    long long cases = 0, excluded = 0, unsound = 0, delta = 0, cone = 0;  // excluded by either / each form
};

void check_node(Rng &r, int g, float rough, NodeCount &k, float cap = 0.f, float steep = 0.f) {
    Patch P = make_patch(r, g, rough, cap, steep);
    float b[kSilNodeBound];
    sil_node_bound(P.c[0], P.c[1], P.c[2], 0, (long long)P.edges.size(),
                   [&](long long j) { return P.edges[(size_t)j]; }, b);
    const float s = std::fmax(P.bound, 1e-6f);
    for (int t = 0; t < 64; ++t) {
        // queries: near the patch (within 1e-6 .. 2 of its size), and far
        V x;
        const V c{P.c[0], P.c[1], P.c[2]};
        const int kind = (int)(r.next() % (cap > 0.f || steep > 0.f ? 4 : 3));
        if (kind == 3 && steep > 0.f) {  // head-on, far along the patch's axis (either side)
            x = add(add(c, mul(P.axis, r.sgn() * r.logu(3.f, 100.f) * s)), mul(rand_in(r, 1.f), 0.05f * s));
        } else if (kind == 3) {  // near the centre of the cap's sphere
            x = add(P.sphere, mul(unit(rand_in(r, 1.f)), r.logu(1e-4f, 0.3f) * s));
        } else if (kind == 0) {
            const SilEdgeGeom &e = P.edges[r.next() % P.edges.size()];
            x = add(V{e.a[0], e.a[1], e.a[2]}, mul(unit(rand_in(r, 1.f)), r.logu(1e-7f, 1.f) * s));
        } else if (kind == 1) {
            x = add(c, rand_in(r, 2.f * s));
        } else {
            x = add(c, mul(unit(rand_in(r, 1.f)), r.logu(2.f, 1e3f) * s));
        }
        const float m = g_margin_scale * sil_node_margin(amax(x), P.bound);
        const bool ed = sil_node_excluded_delta(P.c[0], P.c[1], P.c[2], b, x.x, x.y, x.z, m);
        const bool ec = sil_node_excluded_cone(P.c[0], P.c[1], P.c[2], b, x.x, x.y, x.z, m);
        ++k.cases;
        k.delta += ed;
        k.cone += ec;
        if (!(ed || ec)) continue;
        ++k.excluded;
        for (const SilEdgeGeom &e : P.edges)
            if (reference_silhouette(V{e.a[0], e.a[1], e.a[2]}, V{e.b[0], e.b[1], e.b[2]},
                                     V{e.n0[0], e.n0[1], e.n0[2]}, V{e.n1[0], e.n1[1], e.n1[2]}, x)) {
                ++k.unsound;
                break;
            }
    }
}

void print_node(const char *name, const NodeCount &k, bool last) {
    std::printf("\"%s\": {\"cases\": %lld, \"usable\": %lld, \"excluded\": %lld, \"silhouettes\": 0, "
                "\"unsound\": %lld, \"delta\": %lld, \"cone\": %lld}%s",
                name, k.cases, k.cases, k.excluded, k.unsound, k.delta, k.cone, last ? "" : ", ");
}

}  // namespace

int main(int argc, char **argv) {
    const long long n = argc > 1 ? std::atoll(argv[1]) : 1000000;
    if (argc > 2) g_margin_scale = (float)std::atof(argv[2]);
    Rng r{0x9e3779b97f4a7c15ull};
    Count generic, coplanar, near_plane, sliver, zero_len, far, on_edge;
    for (long long i = 0; i < n; ++i) {
        const float s = r.logu(1e-3f, 1e3f);
        const V o = mul(rand_in(r, 1.f), s * r.uni(0.f, 4.f));  // edges away from the origin too
        // generic: random faces, x anywhere around them
        {
            V a = add(o, rand_in(r, s)), b = add(o, rand_in(r, s)), c = add(o, rand_in(r, s)), d = add(o, rand_in(r, s));
            V x = add(o, rand_in(r, 3.f * s));
            check(a, b, c, d, x, bound_of(a, b, c, d), generic);
        }
        // nearly coplanar faces (dihedral angle down to 1e-7 rad), x near the planes
        {
            V a = add(o, rand_in(r, s)), b = add(o, rand_in(r, s));
            V u = sub(b, a), w = unit(cross(u, rand_in(r, 1.f))), nrm = unit(cross(u, w));
            const float h = r.logu(1e-7f, 1e-1f) * s;
            V c = add(add(a, mul(u, r.uni(0.f, 1.f))), mul(w, s * r.uni(0.1f, 1.f)));
            V d = add(add(add(a, mul(u, r.uni(0.f, 1.f))), mul(w, -s * r.uni(0.1f, 1.f))), mul(nrm, r.sgn() * h));
            V x = add(add(a, mul(u, r.uni(-0.5f, 1.5f))), add(mul(w, r.uni(-2.f, 2.f) * s),
                                                              mul(nrm, r.sgn() * r.logu(1e-9f, 1.f) * s)));
            check(a, b, c, d, x, bound_of(a, b, c, d), coplanar);
            // x exactly in the plane of face 0, up to rounding
            V x2 = add(add(a, mul(u, r.uni(-0.5f, 1.5f))), mul(w, r.uni(-2.f, 2.f) * s));
            check(a, b, c, d, x2, bound_of(a, b, c, d), near_plane);
        }
        // sliver faces: c and d within 1e-6 .. 1e-2 of the edge's line
        {
            V a = add(o, rand_in(r, s)), b = add(o, rand_in(r, s));
            V u = sub(b, a);
            V c = add(add(a, mul(u, r.uni(-1.f, 2.f))), mul(unit(rand_in(r, 1.f)), r.logu(1e-6f, 1e-2f) * s));
            V d = add(add(a, mul(u, r.uni(-1.f, 2.f))), mul(unit(rand_in(r, 1.f)), r.logu(1e-6f, 1e-2f) * s));
            V x = add(o, rand_in(r, 2.f * s));
            check(a, b, c, d, x, bound_of(a, b, c, d), sliver);
        }
        // zero-length edge
        {
            V a = add(o, rand_in(r, s)), c = add(o, rand_in(r, s)), d = add(o, rand_in(r, s));
            V x = add(o, rand_in(r, 2.f * s));
            check(a, a, c, d, x, bound_of(a, a, c, d), zero_len);
        }
        // far queries: |x| up to 1e4 times the scene
        {
            V a = add(o, rand_in(r, s)), b = add(o, rand_in(r, s)), c = add(o, rand_in(r, s)), d = add(o, rand_in(r, s));
            V x = mul(unit(rand_in(r, 1.f)), s * r.logu(10.f, 1e4f));
            check(a, b, c, d, x, bound_of(a, b, c, d), far);
        }
        // x on or next to the edge
        {
            V a = add(o, rand_in(r, s)), b = add(o, rand_in(r, s)), c = add(o, rand_in(r, s)), d = add(o, rand_in(r, s));
            V x = add(add(a, mul(sub(b, a), r.uni(-0.2f, 1.2f))), mul(unit(rand_in(r, 1.f)), r.logu(1e-9f, 1e-2f) * s));
            check(a, b, c, d, x, bound_of(a, b, c, d), on_edge);
        }
    }
    NodeCount smooth, rough, flat, capn, steepn;
    for (long long i = 0; i < n / 200; ++i) {
        check_node(r, 2 + (int)(r.next() % 7), 0.f, smooth);
        check_node(r, 2 + (int)(r.next() % 7), r.logu(1e-3f, 2.f), rough);
        check_node(r, 2 + (int)(r.next() % 7), 1e-6f, flat);
        check_node(r, 2 + (int)(r.next() % 7), 0.f, capn, r.uni(0.35f, 1.48f));  // 20 .. 85 degrees
        check_node(r, 3 + (int)(r.next() % 6), 0.f, steepn, 0.f, r.uni(1.05f, 1.48f));  // 60 .. 85 degrees
    }
    std::printf("{");
    print("generic", generic, false);
    print("coplanar", coplanar, false);
    print("near_plane", near_plane, false);
    print("sliver", sliver, false);
    print("zero_length", zero_len, false);
    print("far", far, false);
    print("on_edge", on_edge, false);
    print_node("node_smooth", smooth, false);
    print_node("node_rough", rough, false);
    print_node("node_flat", flat, false);
    print_node("node_cap", capn, false);
    print_node("node_steep", steepn, true);
    std::printf("}\n");
    const long long bad = generic.unsound + coplanar.unsound + near_plane.unsound + sliver.unsound +
                          zero_len.unsound + far.unsound + on_edge.unsound + smooth.unsound + rough.unsound +
                          flat.unsound + capn.unsound + steepn.unsound;
    return bad ? 1 : 0;
}
