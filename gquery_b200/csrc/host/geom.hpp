// Fixed-size float vectors and axis-aligned boxes for the CPU scene builders.
//
// The builders must produce bit-identical trees to gQuery's Eigen-based C++
// builder, so every reduction here evaluates in the order Eigen 3.4 uses for
// fixed-size float vectors of size 2 and 3 (no SIMD for these sizes):
//   sum over 2 entries : e0 + e1
//   sum over 3 entries : e0 + (e1 + e2)          (redux split in halves)
//   cwiseMin/cwiseMax  : std::min / std::max      ((b < a) ? b : a, ...)
//   maxCoeff(&i)       : first index holding the strict maximum
//   normalized()       : v / sqrt(|v|^2) when |v|^2 > 0, else v unchanged
//   cross              : (a1 b2 - a2 b1, a2 b0 - a0 b2, a0 b1 - a1 b0)
// This file must be compiled without floating-point contraction
// (-ffp-contract=off) so that a*b+c is never fused.
//
// Reference: include/shapes/bounding_box.h:10-72 (BoundingBox), include/core/fwd.h:9-10
// (Float = float, Epsilon = FLT_EPSILON).
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>

namespace gqb {

constexpr float kEps = FLT_EPSILON;            // fwd.h:10  std::numeric_limits<float>::epsilon()
constexpr float kPiF = (float)3.14159265358979323846;  // fwd.h:13 M_PI narrowed to float

template <int D>
struct Vec {
    float v[D];
    float &operator[](int i) { return v[i]; }
    float operator[](int i) const { return v[i]; }
    static Vec splat(float c) {
        Vec r;
        for (int i = 0; i < D; ++i) r.v[i] = c;
        return r;
    }
};

using Vec2 = Vec<2>;
using Vec3 = Vec<3>;

template <int D>
inline Vec<D> operator+(const Vec<D> &a, const Vec<D> &b) {
    Vec<D> r;
    for (int i = 0; i < D; ++i) r.v[i] = a.v[i] + b.v[i];
    return r;
}
template <int D>
inline Vec<D> operator-(const Vec<D> &a, const Vec<D> &b) {
    Vec<D> r;
    for (int i = 0; i < D; ++i) r.v[i] = a.v[i] - b.v[i];
    return r;
}
template <int D>
inline Vec<D> operator*(const Vec<D> &a, float s) {
    Vec<D> r;
    for (int i = 0; i < D; ++i) r.v[i] = a.v[i] * s;
    return r;
}
template <int D>
inline Vec<D> operator/(const Vec<D> &a, float s) {
    Vec<D> r;
    for (int i = 0; i < D; ++i) r.v[i] = a.v[i] / s;
    return r;
}

// Eigen's fixed-size reduction order (see header comment).
inline float eigen_sum(const Vec2 &e) { return e.v[0] + e.v[1]; }
inline float eigen_sum(const Vec3 &e) { return e.v[0] + (e.v[1] + e.v[2]); }

template <int D>
inline float dot(const Vec<D> &a, const Vec<D> &b) {
    Vec<D> p;
    for (int i = 0; i < D; ++i) p.v[i] = a.v[i] * b.v[i];
    return eigen_sum(p);
}
template <int D>
inline float norm(const Vec<D> &a) { return std::sqrt(dot(a, a)); }

template <int D>
inline Vec<D> normalized(const Vec<D> &a) {
    float z = dot(a, a);
    if (z > 0.f) return a / std::sqrt(z);
    return a;
}

inline Vec3 cross(const Vec3 &a, const Vec3 &b) {
    Vec3 r;
    r.v[0] = a.v[1] * b.v[2] - a.v[2] * b.v[1];
    r.v[1] = a.v[2] * b.v[0] - a.v[0] * b.v[2];
    r.v[2] = a.v[0] * b.v[1] - a.v[1] * b.v[0];
    return r;
}

template <int D>
inline Vec<D> cmin(const Vec<D> &a, const Vec<D> &b) {
    Vec<D> r;
    for (int i = 0; i < D; ++i) r.v[i] = std::min(a.v[i], b.v[i]);
    return r;
}
template <int D>
inline Vec<D> cmax(const Vec<D> &a, const Vec<D> &b) {
    Vec<D> r;
    for (int i = 0; i < D; ++i) r.v[i] = std::max(a.v[i], b.v[i]);
    return r;
}

// Axis-aligned box with gQuery's semantics: the default box is empty
// (lo = +FLT_MAX, hi = -FLT_MAX) and growing by a point pads it by FLT_EPSILON.
template <int D>
struct Box {
    Vec<D> lo = Vec<D>::splat(FLT_MAX);
    Vec<D> hi = Vec<D>::splat(-FLT_MAX);

    void grow_point(const Vec<D> &p) {               // bounding_box.h:22-26
        Vec<D> e = Vec<D>::splat(kEps);
        lo = cmin(lo, p - e);
        hi = cmax(hi, p + e);
    }
    void grow_box(const Box &b) {                    // bounding_box.h:28-31
        lo = cmin(lo, b.lo);
        hi = cmax(hi, b.hi);
    }
    Vec<D> extent() const { return hi - lo; }
    Vec<D> centroid() const { return (lo + hi) * 0.5f; }

    // Perimeter in 2D, surface area in 3D (bounding_box.h:37-50).
    float area() const {
        Vec<D> e = extent();
        if constexpr (D == 2) {
            return 2.0f * (e.v[0] + e.v[1]);
        } else {
            return 2.0f * (e.v[0] * e.v[1] + e.v[0] * e.v[2] + e.v[1] * e.v[2]);
        }
    }
    int widest_axis() const {                         // bounding_box.h:52-56 (maxCoeff)
        Vec<D> e = extent();
        int best = 0;
        for (int i = 1; i < D; ++i)
            if (e.v[i] > e.v[best]) best = i;
        return best;
    }
    // Relative position of p inside the box along `axis`, with the extent floored at
    // FLT_EPSILON (bounding_box.h:58-62; only one component is ever consumed).
    float rel(const Vec<D> &p, int axis) const {
        float ext = hi.v[axis] - lo.v[axis];
        ext = std::max(ext, kEps);
        return (p.v[axis] - lo.v[axis]) / ext;
    }
};

}  // namespace gqb
