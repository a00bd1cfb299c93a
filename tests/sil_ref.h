// The kernels' per-edge silhouette test in FP32, shared by the soundness checkers:
// closest point q of [a, b] to x (closest_point_line_segment, math.py), w = q - x, a
// silhouette when (w . n0) * (w . n1) < 0 (silhouette_edge.py:7-12, 50-64).
#pragma once

#include "gq_fmath.h"

struct V {
    float x, y, z;
};

inline bool reference_silhouette(V a, V b, V n0, V n1, V x) {
    const float ux = b.x - a.x, uy = b.y - a.y, uz = b.z - a.z;
    const float vx = x.x - a.x, vy = x.y - a.y, vz = x.z - a.z;
    const float t = gq_clamp(gq_div(gq_dot3(vx, vy, vz, ux, uy, uz), gq_dot3(ux, uy, uz, ux, uy, uz)), 0.f, 1.f);
    const float qx = gq_lerp(a.x, b.x, t), qy = gq_lerp(a.y, b.y, t), qz = gq_lerp(a.z, b.z, t);
    const float wx = qx - x.x, wy = qy - x.y, wz = qz - x.z;
    const float d0 = gq_dot3(wx, wy, wz, n0.x, n0.y, n0.z);
    const float d1 = gq_dot3(wx, wy, wz, n1.x, n1.y, n1.z);
    return d0 * d1 < 0.f;
}
