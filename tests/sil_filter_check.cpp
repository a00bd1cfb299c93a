// Soundness check of the silhouette-edge pre-test (gquery_b200/csrc/sil_filter.h):
// over random and adversarial edges and query points, the pre-test must never
// exclude an edge that the reference's test (silhouette_edge.py:7-12, 50-64, in the
// FP32 operations the kernels use) calls a silhouette.  Prints one JSON line with the
// counts per regime; a non-zero "unsound" is a failure.  An optional second argument
// scales the margin (0 removes it: the check must then find unsound exclusions, which
// shows that its cases reach the rounding boundary the margin covers).
//
// Build: g++ -O2 -ffp-contract=off -I gquery_b200/csrc tests/sil_filter_check.cpp
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "gq_fmath.h"
#include "sil_filter.h"

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

struct V {
    float x, y, z;
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

// The kernels' per-edge test: closest point q (closest_point_line_segment, math.py),
// w = q - x, silhouette when (w . n0) * (w . n1) < 0.
bool reference_silhouette(V a, V b, V n0, V n1, V x) {
    const float ux = b.x - a.x, uy = b.y - a.y, uz = b.z - a.z;
    const float vx = x.x - a.x, vy = x.y - a.y, vz = x.z - a.z;
    const float t = gq_clamp(gq_div(gq_dot3(vx, vy, vz, ux, uy, uz), gq_dot3(ux, uy, uz, ux, uy, uz)), 0.f, 1.f);
    const float qx = gq_lerp(a.x, b.x, t), qy = gq_lerp(a.y, b.y, t), qz = gq_lerp(a.z, b.z, t);
    const float wx = qx - x.x, wy = qy - x.y, wz = qz - x.z;
    const float d0 = gq_dot3(wx, wy, wz, n0.x, n0.y, n0.z);
    const float d1 = gq_dot3(wx, wy, wz, n1.x, n1.y, n1.z);
    return d0 * d1 < 0.f;
}

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
    std::printf("{");
    print("generic", generic, false);
    print("coplanar", coplanar, false);
    print("near_plane", near_plane, false);
    print("sliver", sliver, false);
    print("zero_length", zero_len, false);
    print("far", far, false);
    print("on_edge", on_edge, true);
    std::printf("}\n");
    const long long bad = generic.unsound + coplanar.unsound + near_plane.unsound + sliver.unsound +
                          zero_len.unsound + far.unsound + on_edge.unsound;
    return bad ? 1 : 0;
}
