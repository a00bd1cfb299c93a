// Flattening pass (see flatten.hpp).  Compile with -ffp-contract=off.
#include "flatten.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "../gq_fmath.h"
#include "../sil_filter.h"

namespace gqb {

namespace {

// Preorder rank of every interior node (the index of its pair record), -1 for leaves.
template <int D>
std::vector<int32_t> interior_ranks(const BvhTree<D> &t) {
    std::vector<int32_t> rank(t.nodes.size(), -1);
    int32_t r = 0;
    for (size_t i = 0; i < t.nodes.size(); ++i)
        if (t.nodes[i].n_prims == 0) rank[i] = r++;
    return rank;
}

// Deepest leaf (root at depth 0).
template <int D>
int max_leaf_depth(const BvhTree<D> &t) {
    std::vector<std::pair<uint32_t, int>> st{{0u, 0}};
    int best = 0;
    while (!st.empty()) {
        auto [i, d] = st.back();
        st.pop_back();
        const auto &n = t.nodes[i];
        if (n.n_prims > 0) {
            best = std::max(best, d);
        } else {
            st.push_back({i + 1, d + 1});
            st.push_back({i + (uint32_t)n.second_child, d + 1});
        }
    }
    return best;
}

template <int D>
void put_box(const Box<D> &b, float *lo, float *hi) {
    for (int k = 0; k < D; ++k) {
        lo[k] = b.lo.v[k];
        hi[k] = b.hi.v[k];
    }
}

}  // namespace

template <int D>
void flatten_bvh(const PrimSource<D> &src, const BvhTree<D> &t, DeviceImage<D> &img) {
    const auto rank = interior_ranks(t);
    auto ref_of = [&](uint32_t i) -> int32_t {
        const auto &n = t.nodes[i];
        return n.n_prims > 0 ? ~n.prim_offset : rank[i];
    };
    // every node's run of ordered primitives, children after parents in preorder; a
    // subtree of at most GQ_COLLAPSE_MAX primitives is also written as one run
    std::vector<int64_t> first(t.nodes.size()), count(t.nodes.size());
    for (size_t i = t.nodes.size(); i-- > 0;) {
        const auto &n = t.nodes[i];
        if (n.n_prims > 0) {
            first[i] = n.prim_offset;
            count[i] = n.n_prims;
        } else {
            const size_t l = i + 1, r = i + (size_t)n.second_child;
            first[i] = first[l];
            // contiguous runs (always so in this preorder; -1 turns the collapse off above)
            count[i] = (count[l] >= 0 && count[r] >= 0 && first[r] == first[l] + count[l]) ? count[l] + count[r] : -1;
        }
    }
    auto sub_of = [&](uint32_t i) -> int32_t {
        if (count[i] < 1 || count[i] > GQ_COLLAPSE_MAX || first[i] + count[i] > (int64_t(1) << 24)) return 0;
        return (int32_t)(first[i] | (count[i] << 24));
    };
    img.pairs.clear();
    for (uint32_t i = 0; i < t.nodes.size(); ++i) {
        const auto &n = t.nodes[i];
        if (n.n_prims > 0) continue;
        const uint32_t l = i + 1, r = i + (uint32_t)n.second_child;
        typename DeviceImage<D>::Pair p;
        std::memset(&p, 0, sizeof p);
        if constexpr (D == 2) {
            p.l_lox = t.nodes[l].box.lo.v[0];
            p.l_loy = t.nodes[l].box.lo.v[1];
            p.l_hix = t.nodes[l].box.hi.v[0];
            p.l_hiy = t.nodes[l].box.hi.v[1];
            p.r_lox = t.nodes[r].box.lo.v[0];
            p.r_loy = t.nodes[r].box.lo.v[1];
            p.r_hix = t.nodes[r].box.hi.v[0];
            p.r_hiy = t.nodes[r].box.hi.v[1];
        } else {
            p.l_lox = t.nodes[l].box.lo.v[0];
            p.l_loy = t.nodes[l].box.lo.v[1];
            p.l_loz = t.nodes[l].box.lo.v[2];
            p.l_hix = t.nodes[l].box.hi.v[0];
            p.l_hiy = t.nodes[l].box.hi.v[1];
            p.l_hiz = t.nodes[l].box.hi.v[2];
            p.r_lox = t.nodes[r].box.lo.v[0];
            p.r_loy = t.nodes[r].box.lo.v[1];
            p.r_loz = t.nodes[r].box.lo.v[2];
            p.r_hix = t.nodes[r].box.hi.v[0];
            p.r_hiy = t.nodes[r].box.hi.v[1];
            p.r_hiz = t.nodes[r].box.hi.v[2];
        }
        p.ref_l = ref_of(l);
        p.ref_r = ref_of(r);
        p.sub_l = sub_of(l);
        p.sub_r = sub_of(r);
        img.pairs.push_back(p);
    }
    img.root_ref = ref_of(0);
    put_box(t.nodes[0].box, img.root_lo, img.root_hi);
    img.exact_stack = max_leaf_depth(t) + 1;

    // ordered primitives with end-of-leaf flags
    img.prims.assign(t.order.size(), typename DeviceImage<D>::Prim{});
    for (size_t s = 0; s < t.order.size(); ++s) {
        const int64_t p = t.order[s];
        auto &r = img.prims[s];
        std::memset(&r, 0, sizeof r);
        if constexpr (D == 2) {
            Vec2 a = vert2(src, src.index[2 * p]), b = vert2(src, src.index[2 * p + 1]);
            r.ax = a.v[0];
            r.ay = a.v[1];
            r.bx = b.v[0];
            r.by = b.v[1];
        } else {
            Vec3 a = vert3(src, src.index[3 * p]), b = vert3(src, src.index[3 * p + 1]),
                 c = vert3(src, src.index[3 * p + 2]);
            r.ax = a.v[0];
            r.ay = a.v[1];
            r.az = a.v[2];
            r.bx = b.v[0];
            r.by = b.v[1];
            r.bz = b.v[2];
            r.cx = c.v[0];
            r.cy = c.v[1];
            r.cz = c.v[2];
        }
        // The reference stores the original index as a float (line_segment.h:104-108);
        // reading it back with Int() gives the same value for every index below 2^24.
        r.index = (int32_t)(float)p;
        r.flags = 0;
    }
    for (const auto &n : t.nodes)
        if (n.n_prims > 0) img.prims[(size_t)(n.prim_offset + n.n_prims - 1)].flags |= GQ_ITEM_LAST;

    if constexpr (D == 3) {
        // Bounding spheres: centre = fp32 centroid, radius = largest vertex distance in
        // double, rounded up and widened by 2^-20 relative so the fp32 sphere contains
        // the triangle exactly.
        img.spheres.resize(img.prims.size());
        for (size_t s = 0; s < img.prims.size(); ++s) {
            const auto &r = img.prims[s];
            const float cx = (r.ax + r.bx + r.cx) / 3.f, cy = (r.ay + r.by + r.cy) / 3.f,
                        cz = (r.az + r.bz + r.cz) / 3.f;
            auto dist = [&](float x, float y, float z) {
                const double dx = (double)x - cx, dy = (double)y - cy, dz = (double)z - cz;
                return std::sqrt(dx * dx + dy * dy + dz * dz);
            };
            double rad = std::max(dist(r.ax, r.ay, r.az), std::max(dist(r.bx, r.by, r.bz), dist(r.cx, r.cy, r.cz)));
            float rf = (float)(rad * (1.0 + std::ldexp(1.0, -20)));
            if ((double)rf < rad) rf = std::nextafter(rf, INFINITY);
            img.spheres[s] = gq_tsph_t{cx, cy, cz, (r.flags & GQ_ITEM_LAST) ? -rf : rf};
            if (rf == 0.f && (r.flags & GQ_ITEM_LAST)) img.spheres[s].r = -0.f;
        }
    }
}

// ---------------------------------------------------------------------------
// Quantised 8-wide collapse
// ---------------------------------------------------------------------------

int quant_exponent(float lo, float hi, int qmax) {
    double ext = (double)hi - (double)lo;
    if (!(ext > 0.0)) return -126;
    int e = (int)std::ceil(std::log2(ext / qmax));
    while (qmax * std::ldexp(1.0, e) < ext) ++e;
    while (e > -126 && qmax * std::ldexp(1.0, e - 1) >= ext) --e;
    if (e < -126) e = -126;
    if (e > 127) e = 127;
    return e;
}

// Decoding used by the kernels.  `biased` is the node's stored origin
// fma(-2^23, 2^e, lo); the kernels build the float 2^23 + q from the byte with one
// byte-permute and decode with one fma.
float dequant(float biased, int e, int q) {
    float s = std::ldexp(1.0f, e);
    return std::fma((float)(8388608 + q), s, biased);
}

// Biased origin and exponent for the parent box [lo, hi] such that decode(0) <= lo
// and decode(qmax) >= hi hold exactly in fp32.
void quant_axis(float lo, float hi, int qmax, float *biased, int *e_out) {
    int e = quant_exponent(lo, hi, qmax);
    for (;;) {
        float s = std::ldexp(1.0f, e);
        float b = std::fma(-8388608.0f, s, lo);
        int guard = 0;
        while (!(dequant(b, e, 0) <= lo) && guard++ < 64) b = std::nextafter(b, -INFINITY);
        if (dequant(b, e, qmax) >= hi || e >= 127) {
            *biased = b;
            *e_out = e;
            return;
        }
        ++e;
    }
}

// Outward rounding on a grid of qmax steps: the largest q with decode(q) <= clo and the
// smallest with decode(q) >= chi, checked in the kernels' fp32 decode.
static void quantise_steps(float origin, int e, float clo, float chi, int qmax, int *qlo, int *qhi) {
    const double base = (double)dequant(origin, e, 0);
    int a = (int)std::floor(((double)clo - base) / std::ldexp(1.0, e));
    a = std::max(0, std::min(qmax, a));
    while (a > 0 && !(dequant(origin, e, a) <= clo)) --a;
    while (a < qmax && dequant(origin, e, a + 1) <= clo) ++a;
    int b = (int)std::ceil(((double)chi - base) / std::ldexp(1.0, e));
    b = std::max(0, std::min(qmax, b));
    while (b < qmax && !(dequant(origin, e, b) >= chi)) ++b;
    while (b > 0 && dequant(origin, e, b - 1) >= chi) --b;
    *qlo = a;
    *qhi = b;
}

void quantise_bounds(float origin, int e, float clo, float chi, uint8_t *qlo, uint8_t *qhi) {
    int a, b;
    quantise_steps(origin, e, clo, chi, 255, &a, &b);
    *qlo = (uint8_t)a;
    *qhi = (uint8_t)b;
}

void quantise_bounds16(float origin, int e, float clo, float chi, uint16_t *qlo, uint16_t *qhi) {
    int a, b;
    quantise_steps(origin, e, clo, chi, 65535, &a, &b);
    *qlo = (uint16_t)a;
    *qhi = (uint16_t)b;
}

namespace {

template <int D>
struct WideBuilder {
    const BvhTree<D> &t;
    DeviceImage<D> &img;
    bool with16 = false;
    // every binary node's run of ordered primitives (children after parents in preorder);
    // a subtree of at most GQ_COLLAPSE_MAX primitives becomes one run child (GQ_RUN_REF)
    std::vector<int64_t> sfirst, scount;
    bool small(uint32_t i) const {
        return scount[i] >= 1 && scount[i] <= GQ_COLLAPSE_MAX && sfirst[i] + scount[i] <= (int64_t(1) << 24);
    }

    // Returns the stack entries a traversal of this subtree needs once its node is popped.
    int build(uint32_t b, int32_t *ref_out) {
        const auto &bn = t.nodes[b];
        std::vector<uint32_t> kids{b + 1, b + (uint32_t)bn.second_child};
        while (kids.size() < GQ_WIDTH) {
            int pick = -1;
            float best = -1.f;
            for (size_t k = 0; k < kids.size(); ++k) {
                const auto &kn = t.nodes[kids[k]];
                if (kn.n_prims == 0 && !small(kids[k])) {  // runs are not expanded
                    float a = kn.box.area();
                    if (a > best) {
                        best = a;
                        pick = (int)k;
                    }
                }
            }
            if (pick < 0) break;
            uint32_t c = kids[(size_t)pick];
            kids[(size_t)pick] = c + 1;
            kids.insert(kids.begin() + pick + 1, c + (uint32_t)t.nodes[c].second_child);
        }
        const size_t me = img.wnodes.size();
        img.wnodes.emplace_back();
        if (with16) img.wq16.emplace_back();
        *ref_out = (int32_t)me;

        int e[D];
        float org[D];
        for (int k = 0; k < D; ++k) quant_axis(bn.box.lo.v[k], bn.box.hi.v[k], 255, &org[k], &e[k]);
        if (with16) {
            // the same children's bounds on a grid of 65,535 steps over the node's box
            typename DeviceImage<D>::WQ16 w16;
            std::memset(&w16, 0, sizeof w16);
            int e16[D];
            float o16[D];
            for (int k = 0; k < D; ++k) quant_axis(bn.box.lo.v[k], bn.box.hi.v[k], 65535, &o16[k], &e16[k]);
            w16.ox = o16[0];
            w16.oy = o16[1];
            uint32_t meta = (uint32_t)(e16[0] + 127) | ((uint32_t)(e16[1] + 127) << 8) | ((uint32_t)kids.size() << 24);
            if constexpr (D == 3) {
                w16.oz = o16[2];
                meta |= (uint32_t)(e16[2] + 127) << 16;
            }
            w16.meta = meta;
            for (size_t k = 0; k < kids.size(); ++k) {
                const auto &kn = t.nodes[kids[k]];
                for (int ax = 0; ax < D; ++ax)
                    quantise_bounds16(o16[ax], e16[ax], kn.box.lo.v[ax], kn.box.hi.v[ax], &w16.q[ax][k],
                                      &w16.q[D + ax][k]);
            }
            img.wq16[me] = w16;
        }
        typename DeviceImage<D>::WNode w;
        std::memset(&w, 0, sizeof w);
        if constexpr (D == 2) {
            w.ox = org[0];
            w.oy = org[1];
            w.meta = (uint32_t)(e[0] + 127) | ((uint32_t)(e[1] + 127) << 8) | ((uint32_t)kids.size() << 24);
        } else {
            w.ox = org[0];
            w.oy = org[1];
            w.oz = org[2];
            w.meta = (uint32_t)(e[0] + 127) | ((uint32_t)(e[1] + 127) << 8) | ((uint32_t)(e[2] + 127) << 16) |
                     ((uint32_t)kids.size() << 24);
        }
        for (int k = 0; k < GQ_WIDTH; ++k) w.ref[k] = kEmptyLeaf;
        int deepest = 0;
        for (size_t k = 0; k < kids.size(); ++k) {
            const auto &kn = t.nodes[kids[k]];
            for (int ax = 0; ax < D; ++ax)
                quantise_bounds(org[ax], e[ax], kn.box.lo.v[ax], kn.box.hi.v[ax], &w.q[ax][k], &w.q[D + ax][k]);
            if (kn.n_prims > 0) {
                w.ref[k] = ~kn.prim_offset;
            } else if (small(kids[k])) {
                w.ref[k] = (int32_t)(0x80000000u | (uint32_t)(sfirst[kids[k]] | (scount[kids[k]] << 24)));
            } else {
                int32_t r;
                int need = build(kids[k], &r);
                w.ref[k] = r;
                deepest = std::max(deepest, need);
            }
        }
        img.wnodes[me] = w;
        const int k = (int)kids.size();
        return std::max(k, (k - 1) + deepest);
    }
};

}  // namespace

template <int D>
void flatten_wide(const BvhTree<D> &t, DeviceImage<D> &img, bool with16) {
    img.wnodes.clear();
    img.wq16.clear();
    if (t.nodes[0].n_prims > 0) {
        img.wroot_ref = ~t.nodes[0].prim_offset;
        img.wide_stack = 1;
        return;
    }
    WideBuilder<D> wb{t, img, with16};
    wb.sfirst.assign(t.nodes.size(), 0);
    wb.scount.assign(t.nodes.size(), 0);
    for (size_t i = t.nodes.size(); i-- > 0;) {
        const auto &n = t.nodes[i];
        if (n.n_prims > 0) {
            wb.sfirst[i] = n.prim_offset;
            wb.scount[i] = n.n_prims;
        } else {
            const size_t l = i + 1, r = i + (size_t)n.second_child;
            wb.sfirst[i] = wb.sfirst[l];
            const bool joined = wb.scount[l] >= 0 && wb.scount[r] >= 0 && wb.sfirst[r] == wb.sfirst[l] + wb.scount[l];
            wb.scount[i] = joined ? wb.scount[l] + wb.scount[r] : -1;
        }
    }
    int32_t r;
    img.wide_stack = wb.build(0, &r);
    img.wroot_ref = r;
}

// ---------------------------------------------------------------------------
// Binary SNCH
// ---------------------------------------------------------------------------

namespace {

// Node bounds of sil_filter.h for both children of every 3D pair.  The silhouettes of
// a subtree are one contiguous run of the leaf-ordered list (depth-first layout); a
// subtree whose run is not contiguous gets a bound that never skips it.
template <int D>
void snch_node_bounds(const BvhTree<D> &t, const SnchTree<D> &s, DeviceImage<D> &img, int n_threads) {
    const size_t nn = t.nodes.size();
    std::vector<int64_t> beg(nn, 0), end(nn, 0);
    std::vector<uint8_t> split(nn, 0);  // 1: run not contiguous
    for (size_t i = nn; i-- > 0;) {
        const auto &n = t.nodes[i];
        if (n.n_prims > 0) {
            beg[i] = s.nodes[i].n_sil > 0 ? s.nodes[i].sil_offset : 0;
            end[i] = s.nodes[i].n_sil > 0 ? s.nodes[i].sil_offset + s.nodes[i].n_sil : 0;
            continue;
        }
        const size_t l = i + 1, r = i + (size_t)n.second_child;
        const bool el = beg[l] == end[l], er = beg[r] == end[r];
        split[i] = split[l] | split[r];
        if (el) {
            beg[i] = beg[r];
            end[i] = end[r];
        } else if (er) {
            beg[i] = beg[l];
            end[i] = end[l];
        } else if (end[l] == beg[r]) {
            beg[i] = beg[l];
            end[i] = end[r];
        } else if (end[r] == beg[l]) {
            beg[i] = beg[r];
            end[i] = end[l];
        } else {
            beg[i] = std::min(beg[l], beg[r]);
            end[i] = std::max(end[l], end[r]);
            split[i] = 1;
        }
    }
    // each record's orientation, read once in record order (a node's bound reads its
    // records up to ten times, and the raw edges lie in another order)
    std::vector<float> orient(img.sils.size());
    for (size_t j = 0; j < orient.size(); ++j) orient[j] = (float)s.raw[s.ordered[j]].orient;
    auto edge = [&](long long j) {
        const gq_sile_t &r = img.sils[(size_t)j];
        SilEdgeGeom g;
        g.a[0] = r.ax; g.a[1] = r.ay; g.a[2] = r.az;
        g.b[0] = r.bx; g.b[1] = r.by; g.b[2] = r.bz;
        g.n0[0] = r.n0x; g.n0[1] = r.n0y; g.n0[2] = r.n0z;
        g.n1[0] = r.n1x; g.n1[1] = r.n1y; g.n1[2] = r.n1z;
        g.orient = orient[(size_t)j];
        g.usable = (r.flags & (GQ_ITEM_VALID | GQ_SIL_FILTER)) == GQ_SIL_FILTER;
        return g;
    };
    // each record's two normal lengths, computed once (every enclosing node's bound reads them)
    std::vector<double> nlen(2 * img.sils.size());
    for (size_t j = 0; j < img.sils.size(); ++j) {
        const SilEdgeGeom g = edge((long long)j);
        nlen[2 * j] = sil_normal_len(g, 0);
        nlen[2 * j + 1] = sil_normal_len(g, 1);
    }
    auto len = [&](long long j, int f, const SilEdgeGeom &) { return nlen[2 * (size_t)j + (size_t)f]; };
    auto bound = [&](size_t i, float out[kSilNodeBound]) {
        const auto &bx = t.nodes[i].box;
        const float cx = sil_node_centre(bx.lo.v[0], bx.hi.v[0]), cy = sil_node_centre(bx.lo.v[1], bx.hi.v[1]),
                    cz = sil_node_centre(bx.lo.v[2], bx.hi.v[2]);
        if (split[i]) {
            // never skipped (delta = +inf, lo = -inf, hi = +inf)
            const float open[kSilNodeBound] = {0.f, 0.f, 0.f, __builtin_inff(), 1.f, 0.f, -__builtin_inff(),
                                               __builtin_inff()};
            std::memcpy(out, open, sizeof open);
        } else {
            sil_node_bound(cx, cy, cz, beg[i], end[i], edge, len, out);
        }
    };
    std::vector<uint32_t> interior;  // pair k belongs to interior node interior[k]
    for (size_t i = 0; i < nn; ++i)
        if (t.nodes[i].n_prims == 0) interior.push_back((uint32_t)i);
    auto pair_bounds = [&](size_t k) {
        const size_t i = interior[k];
        auto &p = img.spairs[k];
        bound(i + 1, p.l_b);
        bound(i + (size_t)t.nodes[i].second_child, p.r_b);
    };
    const int nt = std::max(1, n_threads);
    if (nt == 1 || interior.size() < 4096) {
        for (size_t k = 0; k < interior.size(); ++k) pair_bounds(k);
    } else {  // each pair is independent: the result does not depend on the thread count
        std::vector<std::thread> pool;
        for (int th = 0; th < nt; ++th)
            pool.emplace_back([&, th]() {
                for (size_t k = (size_t)th; k < interior.size(); k += (size_t)nt) pair_bounds(k);
            });
        for (auto &th : pool) th.join();
    }
}

}  // namespace

void device_silhouette(const SilVertex &x, gq_silv_t &r) {
    std::memset(&r, 0, sizeof r);
    r.ax = x.v[0].v[0]; r.ay = x.v[0].v[1];
    r.bx = x.v[1].v[0]; r.by = x.v[1].v[1];
    r.cx = x.v[2].v[0]; r.cy = x.v[2].v[1];
    r.prim = (int32_t)(float)x.prim;
    // silhouette_vertex.py:48: Int(Float(index)) != -1 for both neighbours
    const bool ok = ((int64_t)(float)x.idx[0] != -1) && ((int64_t)(float)x.idx[2] != -1);
    r.flags = ok ? GQ_ITEM_VALID : 0;
}

void device_silhouette(const SilEdge &x, gq_sile_t &r) {
    std::memset(&r, 0, sizeof r);
    // SilhouetteEdges view (silhouette_edge.py:75-86): c = v[0], a = v[1], b = v[2], d = v[3]
    r.ax = x.v[1].v[0]; r.ay = x.v[1].v[1]; r.az = x.v[1].v[2];
    r.bx = x.v[2].v[0]; r.by = x.v[2].v[1]; r.bz = x.v[2].v[2];
    const float cx = x.v[0].v[0], cy = x.v[0].v[1], cz = x.v[0].v[2];
    const float dx = x.v[3].v[0], dy = x.v[3].v[1], dz = x.v[3].v[2];
    // n0 = normalize(cross(b - a, c - a)), n1 = normalize(cross(d - a, b - a))
    sil_face_normal(r.bx - r.ax, r.by - r.ay, r.bz - r.az, cx - r.ax, cy - r.ay, cz - r.az, r.n0x, r.n0y, r.n0z);
    sil_face_normal(dx - r.ax, dy - r.ay, dz - r.az, r.bx - r.ax, r.by - r.ay, r.bz - r.az, r.n1x, r.n1y, r.n1z);
    r.prim = (int32_t)(float)x.prim;
    // silhouette_edge.py:56-57: boundary marker index == -1 never occurs (size_t storage)
    const bool boundary = ((int64_t)(float)x.idx[0] == -1) || ((int64_t)(float)x.idx[3] == -1);
    r.flags = boundary ? GQ_ITEM_VALID : 0;  // for edges the bit means "always a silhouette"
    // spans of the pre-test that skips edges which are certainly no silhouette
    r.span0 = sil_span(r.n0x, r.n0y, r.n0z, r.ax, r.ay, r.az, r.bx, r.by, r.bz);
    r.span1 = sil_span(r.n1x, r.n1y, r.n1z, r.ax, r.ay, r.az, r.bx, r.by, r.bz);
    if (!boundary && sil_filter_usable(r.n0x, r.n0y, r.n0z, r.n1x, r.n1y, r.n1z, r.span0, r.span1))
        r.flags |= GQ_SIL_FILTER;
}

template <int D>
void flatten_snch(const BvhTree<D> &t, const SnchTree<D> &s, DeviceImage<D> &img, int n_threads) {
    const auto rank = interior_ranks(t);
    auto ref_of = [&](uint32_t i) -> int32_t {
        const auto &n = t.nodes[i];
        if (n.n_prims == 0) return rank[i];
        return s.nodes[i].n_sil > 0 ? ~s.nodes[i].sil_offset : kEmptyLeaf;
    };
    img.spairs.clear();
    for (uint32_t i = 0; i < t.nodes.size(); ++i) {
        const auto &n = t.nodes[i];
        if (n.n_prims > 0) continue;
        const uint32_t l = i + 1, r = i + (uint32_t)n.second_child;
        const auto &L = t.nodes[l], &R = t.nodes[r];
        const auto &Lc = s.nodes[l].cone, &Rc = s.nodes[r].cone;
        typename DeviceImage<D>::SPair p;
        std::memset(&p, 0, sizeof p);
        if constexpr (D == 2) {
            p.l_lox = L.box.lo.v[0]; p.l_loy = L.box.lo.v[1]; p.l_hix = L.box.hi.v[0]; p.l_hiy = L.box.hi.v[1];
            p.l_ax = Lc.axis.v[0]; p.l_ay = Lc.axis.v[1]; p.l_half = Lc.half_angle; p.l_rad = Lc.radius;
            p.r_lox = R.box.lo.v[0]; p.r_loy = R.box.lo.v[1]; p.r_hix = R.box.hi.v[0]; p.r_hiy = R.box.hi.v[1];
            p.r_ax = Rc.axis.v[0]; p.r_ay = Rc.axis.v[1]; p.r_half = Rc.half_angle; p.r_rad = Rc.radius;
        } else {
            p.l_lox = L.box.lo.v[0]; p.l_loy = L.box.lo.v[1]; p.l_loz = L.box.lo.v[2];
            p.l_hix = L.box.hi.v[0]; p.l_hiy = L.box.hi.v[1]; p.l_hiz = L.box.hi.v[2];
            p.l_ax = Lc.axis.v[0]; p.l_ay = Lc.axis.v[1]; p.l_az = Lc.axis.v[2];
            p.l_half = Lc.half_angle; p.l_rad = Lc.radius;
            p.r_lox = R.box.lo.v[0]; p.r_loy = R.box.lo.v[1]; p.r_loz = R.box.lo.v[2];
            p.r_hix = R.box.hi.v[0]; p.r_hiy = R.box.hi.v[1]; p.r_hiz = R.box.hi.v[2];
            p.r_ax = Rc.axis.v[0]; p.r_ay = Rc.axis.v[1]; p.r_az = Rc.axis.v[2];
            p.r_half = Rc.half_angle; p.r_rad = Rc.radius;
        }
        p.ref_l = ref_of(l);
        p.ref_r = ref_of(r);
        img.spairs.push_back(p);
    }
    img.sroot_ref = ref_of(0);

    img.sils.assign(s.ordered.size(), typename DeviceImage<D>::Sil{});
    for (size_t k = 0; k < s.ordered.size(); ++k) device_silhouette(s.raw[s.ordered[k]], img.sils[k]);
    for (size_t i = 0; i < t.nodes.size(); ++i) {
        const auto &sn = s.nodes[i];
        if (t.nodes[i].n_prims > 0 && sn.n_sil > 0) img.sils[(size_t)(sn.sil_offset + sn.n_sil - 1)].flags |= GQ_ITEM_LAST;
    }
    if constexpr (D == 3) snch_node_bounds(t, s, img, n_threads);
}

// The same collapse over a binary tree given as pair records (a device-built tree: pair
// i holds both child boxes of interior node i and their references, leaf = ~record).
// The top levels are built first; the interior children found at depth kDeferDepth are
// built as separate subtrees on threads and appended with their indices shifted.
template <int D>
struct PairWideBuilder {
    using Pair = typename DeviceImage<D>::Pair;
    using WNode = typename DeviceImage<D>::WNode;
    struct Deferred {
        int32_t node;
        Box<D> box;
        size_t wnode;
        int slot;
    };
    const std::vector<Pair> &pairs;
    std::vector<WNode> &out;
    int defer_depth;                   // < 0: build everything here
    std::vector<Deferred> *deferred;

    static Box<D> child_box(const Pair &p, int c) {
        Box<D> b;
        if constexpr (D == 2) {
            b.lo.v[0] = c ? p.r_lox : p.l_lox; b.lo.v[1] = c ? p.r_loy : p.l_loy;
            b.hi.v[0] = c ? p.r_hix : p.l_hix; b.hi.v[1] = c ? p.r_hiy : p.l_hiy;
        } else {
            b.lo.v[0] = c ? p.r_lox : p.l_lox; b.lo.v[1] = c ? p.r_loy : p.l_loy; b.lo.v[2] = c ? p.r_loz : p.l_loz;
            b.hi.v[0] = c ? p.r_hix : p.l_hix; b.hi.v[1] = c ? p.r_hiy : p.l_hiy; b.hi.v[2] = c ? p.r_hiz : p.l_hiz;
        }
        return b;
    }

    int32_t build(int32_t node, const Box<D> &box, int depth) {
        struct Kid {
            int32_t ref;
            Box<D> box;
        };
        const Pair &pn = pairs[(size_t)node];
        std::vector<Kid> kids{{pn.ref_l, child_box(pn, 0)}, {pn.ref_r, child_box(pn, 1)}};
        while (kids.size() < GQ_WIDTH) {  // open the interior child with the largest area
            int pick = -1;
            float best = -1.f;
            for (size_t k = 0; k < kids.size(); ++k) {
                if (kids[k].ref >= 0) {
                    const float a = kids[k].box.area();
                    if (a > best) {
                        best = a;
                        pick = (int)k;
                    }
                }
            }
            if (pick < 0) break;
            const Pair &pc = pairs[(size_t)kids[(size_t)pick].ref];
            kids[(size_t)pick] = Kid{pc.ref_l, child_box(pc, 0)};
            kids.insert(kids.begin() + pick + 1, Kid{pc.ref_r, child_box(pc, 1)});
        }
        const size_t me = out.size();
        out.emplace_back();
        int e[D];
        float org[D];
        for (int k = 0; k < D; ++k) quant_axis(box.lo.v[k], box.hi.v[k], 255, &org[k], &e[k]);
        WNode w;
        std::memset(&w, 0, sizeof w);
        if constexpr (D == 2) {
            w.ox = org[0];
            w.oy = org[1];
            w.meta = (uint32_t)(e[0] + 127) | ((uint32_t)(e[1] + 127) << 8) | ((uint32_t)kids.size() << 24);
        } else {
            w.ox = org[0];
            w.oy = org[1];
            w.oz = org[2];
            w.meta = (uint32_t)(e[0] + 127) | ((uint32_t)(e[1] + 127) << 8) | ((uint32_t)(e[2] + 127) << 16) |
                     ((uint32_t)kids.size() << 24);
        }
        for (int k = 0; k < GQ_WIDTH; ++k) w.ref[k] = kEmptyLeaf;
        for (size_t k = 0; k < kids.size(); ++k)
            for (int ax = 0; ax < D; ++ax)
                quantise_bounds(org[ax], e[ax], kids[k].box.lo.v[ax], kids[k].box.hi.v[ax], &w.q[ax][k],
                                &w.q[D + ax][k]);
        out[me] = w;
        for (size_t k = 0; k < kids.size(); ++k) {
            if (kids[k].ref < 0) {
                out[me].ref[k] = kids[k].ref;  // one primitive per leaf: ~record
            } else if (defer_depth >= 0 && depth + 1 >= defer_depth) {
                deferred->push_back(Deferred{kids[k].ref, kids[k].box, me, (int)k});
            } else {
                const int32_t r = build(kids[k].ref, kids[k].box, depth + 1);
                out[me].ref[k] = r;
            }
        }
        return (int32_t)me;
    }
};

// Stack entries a traversal of wide node w needs once it is popped (as flatten_wide
// computes while building).
template <int D>
static int wide_need(const std::vector<typename DeviceImage<D>::WNode> &w, int32_t i) {
    const int k = (int)(w[(size_t)i].meta >> 24);
    int deepest = 0;
    for (int c = 0; c < k; ++c)
        if (w[(size_t)i].ref[c] >= 0) deepest = std::max(deepest, wide_need<D>(w, w[(size_t)i].ref[c]));
    return std::max(k, (k - 1) + deepest);
}

template <int D>
void flatten_wide_from_pairs(const std::vector<typename DeviceImage<D>::Pair> &pairs, int32_t root_ref,
                             const float *root_lo, const float *root_hi, DeviceImage<D> &img, int n_threads) {
    using WNode = typename DeviceImage<D>::WNode;
    img.wnodes.clear();
    if (root_ref < 0) {
        img.wroot_ref = root_ref;
        img.wide_stack = 1;
        return;
    }
    Box<D> box;
    for (int k = 0; k < D; ++k) box.lo.v[k] = root_lo[k], box.hi.v[k] = root_hi[k];
    constexpr int kDeferDepth = 3;  // up to 8^3 subtrees for the threads
    std::vector<typename PairWideBuilder<D>::Deferred> deferred;
    PairWideBuilder<D> top{pairs, img.wnodes, kDeferDepth, &deferred};
    img.wroot_ref = top.build(root_ref, box, 0);
    std::vector<std::vector<WNode>> parts(deferred.size());
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t i; (i = next.fetch_add(1)) < deferred.size();) {
            PairWideBuilder<D> sub{pairs, parts[i], -1, nullptr};
            sub.build(deferred[i].node, deferred[i].box, 0);
        }
    };
    const int nt = std::max(1, std::min<int>(n_threads, (int)deferred.size()));
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (auto &th : pool) th.join();
    for (size_t i = 0; i < deferred.size(); ++i) {  // append, shifting the subtree's own indices
        const int32_t base = (int32_t)img.wnodes.size();
        for (WNode &w : parts[i])
            for (int k = 0; k < GQ_WIDTH; ++k)
                if (w.ref[k] >= 0) w.ref[k] += base;
        img.wnodes.insert(img.wnodes.end(), parts[i].begin(), parts[i].end());
        img.wnodes[deferred[i].wnode].ref[deferred[i].slot] = base;
    }
    img.wide_stack = wide_need<D>(img.wnodes, img.wroot_ref);
}

template void flatten_bvh<2>(const PrimSource<2> &, const BvhTree<2> &, DeviceImage<2> &);
template void flatten_bvh<3>(const PrimSource<3> &, const BvhTree<3> &, DeviceImage<3> &);
template void flatten_wide<2>(const BvhTree<2> &, DeviceImage<2> &, bool);
template void flatten_wide<3>(const BvhTree<3> &, DeviceImage<3> &, bool);
template void flatten_wide_from_pairs<2>(const std::vector<gq_pair2_t> &, int32_t, const float *, const float *,
                                         DeviceImage<2> &, int);
template void flatten_wide_from_pairs<3>(const std::vector<gq_pair3_t> &, int32_t, const float *, const float *,
                                         DeviceImage<3> &, int);
template void flatten_snch<2>(const BvhTree<2> &, const SnchTree<2> &, DeviceImage<2> &, int);
template void flatten_snch<3>(const BvhTree<3> &, const SnchTree<3> &, DeviceImage<3> &, int);

}  // namespace gqb
