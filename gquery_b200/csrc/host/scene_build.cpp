// CPU scene builders (see scene_build.hpp).  Compile with -ffp-contract=off.
#include "scene_build.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <unordered_set>

#include "../gq_fmath.h"

namespace gqb {

Vec2 vert2(const PrimSource<2> &src, int64_t i) {
    Vec2 r;
    r.v[0] = src.verts[2 * i + 0];
    r.v[1] = src.verts[2 * i + 1];
    return r;
}
Vec3 vert3(const PrimSource<3> &src, int64_t i) {
    Vec3 r;
    r.v[0] = src.verts[3 * i + 0];
    r.v[1] = src.verts[3 * i + 1];
    r.v[2] = src.verts[3 * i + 2];
    return r;
}

template <int D>
static Vec<D> vert(const PrimSource<D> &src, int64_t i) {
    if constexpr (D == 2)
        return vert2(src, i);
    else
        return vert3(src, i);
}

template <int D>
std::string validate_source(const PrimSource<D> &src) {
    if (src.np <= 0) return "scene has no primitives";
    if (src.nv <= 0) return "scene has no vertices";
    if (src.np > (int64_t(1) << 30)) return "too many primitives (limit 2^30)";
    for (int64_t i = 0; i < src.np * D; ++i) {
        int32_t k = src.index[i];
        if (k < 0 || k >= src.nv) return "primitive index out of range";
    }
    // the SAH bins centroids with int(12 * offset), which a NaN or an infinite
    // coordinate turns into an out-of-range bucket (bvh.cpp:44-46 has no guard)
    for (int64_t i = 0; i < src.nv * D; ++i)
        if (!std::isfinite(src.verts[i])) return "vertex coordinates must be finite";
    return std::string();
}

// ---------------------------------------------------------------------------
// Binned SAH BVH (src/shapes/bvh.cpp:29-88, 182-327)
// ---------------------------------------------------------------------------

namespace {

constexpr int kBuckets = 12;  // bvh.cpp:91

template <int D>
struct BuildPrim {
    uint32_t index;  // original primitive index
    Box<D> box;
};

template <int D>
inline int bucket_of(const Box<D> &cbox, const Vec<D> &c, int dim) {
    // bvh.cpp:44-46 and 258-260: int(12 * offset[dim]), the top edge folds into the last bucket.
    int b = (int)((float)kBuckets * cbox.rel(c, dim));
    if (b == kBuckets) b = kBuckets - 1;
    return b;
}

struct SahChoice {
    int bucket;
    float cost;
};

// Sweep of the 11 candidate split planes between the 12 buckets (bvh.cpp:29-88).
template <int D>
SahChoice sah_choose(const BuildPrim<D> *p, size_t n, const Box<D> &cbox, int dim) {
    Box<D> bbox[kBuckets];
    int bcount[kBuckets] = {};
    for (size_t i = 0; i < n; ++i) {
        int b = bucket_of(cbox, p[i].box.centroid(), dim);
        bcount[b] += 1;
        bbox[b].grow_box(p[i].box);
    }
    constexpr int kSplits = kBuckets - 1;
    float cost[kSplits] = {};
    int below = 0;
    Box<D> acc;
    for (int s = 0; s < kSplits; ++s) {
        acc.grow_box(bbox[s]);
        below += bcount[s];
        cost[s] = (float)below * acc.area();
    }
    int above = 0;
    Box<D> acc2;
    for (int s = kSplits - 1; s >= 0; --s) {
        acc2.grow_box(bbox[s + 1]);
        above += bcount[s + 1];
        cost[s] += (float)above * acc2.area();
    }
    SahChoice best{0, cost[0]};
    for (int s = 1; s < kSplits; ++s) {
        if (cost[s] < best.cost) {
            best.cost = cost[s];
            best.bucket = s;
        }
    }
    return best;
}

template <int D>
struct BvhBuilder {
    BuildPrim<D> *prims;
    int max_leaf;
    int par_depth;  // subtrees at depth < par_depth may be built on another thread
    int max_depth = 0;

    // Appends the subtree over prims[begin, end) to `out` in preorder.
    void build(size_t begin, size_t end, std::vector<FlatNode<D>> &out, int depth) {
        if (depth > max_depth) max_depth = depth;
        const size_t n = end - begin;
        const size_t me = out.size();
        out.emplace_back();

        Box<D> box;
        for (size_t i = begin; i < end; ++i) box.grow_box(prims[i].box);

        auto make_leaf = [&]() {
            FlatNode<D> &nd = out[me];
            nd.box = box;
            nd.prim_offset = (int32_t)begin;  // slot of the leaf's first ordered primitive
            nd.n_prims = (int32_t)n;
            nd.second_child = 0;
        };

        if (box.area() == 0.f || n == 1) {  // bvh.cpp:200
            make_leaf();
            return;
        }
        Box<D> cbox;
        for (size_t i = begin; i < end; ++i) cbox.grow_point(prims[i].box.centroid());
        const int dim = cbox.widest_axis();
        if (cbox.hi.v[dim] == cbox.lo.v[dim]) {  // bvh.cpp:218
            make_leaf();
            return;
        }

        size_t mid;
        if (n <= 2) {  // bvh.cpp:233-239
            mid = begin + n / 2;
            std::nth_element(prims + begin, prims + mid, prims + end,
                             [dim](const BuildPrim<D> &a, const BuildPrim<D> &b) {
                                 return a.box.centroid().v[dim] < b.box.centroid().v[dim];
                             });
        } else {
            SahChoice ch = sah_choose(prims + begin, n, cbox, dim);
            const float leaf_cost = (float)n;
            const float split_cost = 1.f / 2.f + ch.cost / box.area();  // bvh.cpp:251
            if ((int64_t)n > max_leaf || split_cost < leaf_cost) {
                const int sb = ch.bucket;
                BuildPrim<D> *m = std::partition(prims + begin, prims + end,
                                                 [&cbox, dim, sb](const BuildPrim<D> &p) {
                                                     return bucket_of(cbox, p.box.centroid(), dim) <= sb;
                                                 });
                mid = (size_t)(m - prims);
            } else {
                make_leaf();
                return;
            }
        }
        // The reference recurses on an empty half forever (stack overflow) if a split
        // leaves one side empty; that needs a centroid extent below FLT_EPSILON.  Such
        // nodes become leaves here.
        if (mid == begin || mid == end) {
            make_leaf();
            return;
        }

        out[me].axis = dim;
        out[me].n_prims = 0;
        if (depth < par_depth && n > 65536) {
            std::vector<FlatNode<D>> left, right;
            int dl = 0;
            std::thread th([&]() {
                BvhBuilder<D> sub{prims, max_leaf, par_depth, 0};
                sub.build(begin, mid, left, depth + 1);
                dl = sub.max_depth;
            });
            build(mid, end, right, depth + 1);
            th.join();
            if (dl > max_depth) max_depth = dl;
            out.insert(out.end(), left.begin(), left.end());
            out.insert(out.end(), right.begin(), right.end());
            out[me].second_child = (int32_t)(1 + left.size());
        } else {
            build(begin, mid, out, depth + 1);
            out[me].second_child = (int32_t)(out.size() - me);
            build(mid, end, out, depth + 1);
        }
        // init_interior (include/shapes/bvh.h:457-465): empty box grown by both children.
        Box<D> ib;
        ib.grow_box(out[me + 1].box);
        ib.grow_box(out[me + out[me].second_child].box);
        out[me].box = ib;
    }
};

}  // namespace

template <int D>
BvhTree<D> build_bvh(const PrimSource<D> &src, int max_prims_in_node, int n_threads) {
    std::vector<BuildPrim<D>> prims((size_t)src.np);
    for (int64_t i = 0; i < src.np; ++i) {
        Box<D> b;  // LineSegment/Triangle::bounding_box: empty box grown by each vertex
        for (int k = 0; k < D; ++k) b.grow_point(vert(src, src.index[i * D + k]));
        prims[(size_t)i] = BuildPrim<D>{(uint32_t)i, b};
    }
    int par_depth = 0;
    while ((1 << par_depth) < n_threads && par_depth < 6) ++par_depth;
    BvhBuilder<D> b{prims.data(), max_prims_in_node, par_depth, 0};
    BvhTree<D> t;
    t.nodes.reserve((size_t)(2 * src.np));
    b.build(0, prims.size(), t.nodes, 0);
    t.max_depth = b.max_depth;
    t.order.resize(prims.size());
    for (size_t i = 0; i < prims.size(); ++i) t.order[i] = (int32_t)prims[i].index;
    return t;
}

// ---------------------------------------------------------------------------
// Silhouettes and normal cones (src/shapes/snch.cpp, silhouette_edge.cpp)
// ---------------------------------------------------------------------------

std::vector<SilVertex> build_polyline_silhouettes(const PrimSource<2> &src) {
    const int64_t nv = src.nv;
    std::vector<int64_t> prev((size_t)nv, -1), next((size_t)nv, -1), order;
    std::vector<uint8_t> seen((size_t)nv, 0);
    auto visit = [&](int64_t v) {
        if (!seen[(size_t)v]) {
            seen[(size_t)v] = 1;
            order.push_back(v);
        }
    };
    for (int64_t e = 0; e < src.np; ++e) {  // polyline.py:60-73
        const int64_t a = src.index[2 * e], b = src.index[2 * e + 1];
        visit(a);
        visit(b);
        next[(size_t)a] = b;
        prev[(size_t)b] = a;
    }
    std::vector<SilVertex> out;
    for (size_t i = 0; i < order.size(); ++i) {  // polyline.py:82-97
        const int64_t cur = order[i], p = prev[(size_t)cur], n = next[(size_t)cur];
        if (p == -1 || n == -1) continue;
        SilVertex s;
        s.v[0] = vert2(src, p);
        s.v[1] = vert2(src, cur);
        s.v[2] = vert2(src, n);
        s.idx[0] = (uint64_t)p;
        s.idx[1] = (uint64_t)cur;
        s.idx[2] = (uint64_t)n;
        s.prim = (uint64_t)i;
        // polyline.py:111-118: drop nearly collinear vertices (normalize = v / |v| in FP32)
        const float e1x = s.v[1].v[0] - s.v[0].v[0], e1y = s.v[1].v[1] - s.v[0].v[1];
        const float e2x = s.v[2].v[0] - s.v[1].v[0], e2y = s.v[2].v[1] - s.v[1].v[1];
        const float i1 = gq_rsqrt(gq_dot2(e1x, e1y, e1x, e1y)), i2 = gq_rsqrt(gq_dot2(e2x, e2y, e2x, e2y));
        const float col = std::fabs(gq_dot2(e1x * i1, e1y * i1, e2x * i2, e2y * i2));
        if (col < 0.99999f) out.push_back(s);
    }
    return out;
}

std::vector<SilEdge> build_silhouette_edges(const PrimSource<3> &src,
                                            std::vector<uint32_t> *face_edge_out) {
    // Edge ids follow the order in which an undirected edge is first met while
    // scanning faces f = 0.. and their edges k = 0..2 (silhouette_edge.cpp:5-19).
    // Half-edges are bucketed by their smaller vertex (a counting sort, each bucket in
    // half-edge order); within a bucket the half-edges with the same larger vertex form
    // one edge, whose first member is its first appearance.  A bucket holds about a
    // vertex's degree; a large one (a fan around one vertex) is sorted instead of
    // scanned, which keeps the pass O(n log n) for any mesh.
    const size_t nh = (size_t)src.np * 3;
    std::vector<uint32_t> lo_of(nh), hi_of(nh);
    uint32_t top = 0;
    for (size_t h = 0; h < nh; ++h) {
        const size_t f = h / 3, k = h % 3;
        uint32_t i0 = (uint32_t)src.index[f * 3 + k];
        uint32_t i1 = (uint32_t)src.index[f * 3 + (k + 1) % 3];
        if (i0 > i1) std::swap(i0, i1);
        lo_of[h] = i0;
        hi_of[h] = i1;
        top = std::max(top, i0);
    }
    std::vector<uint32_t> start(nh ? (size_t)top + 2 : 1, 0);
    for (size_t h = 0; h < nh; ++h) ++start[(size_t)lo_of[h] + 1];
    for (size_t b = 1; b < start.size(); ++b) start[b] += start[b - 1];
    std::vector<uint32_t> slot(nh), fill(start.begin(), start.end() - 1);
    for (size_t h = 0; h < nh; ++h) slot[fill[lo_of[h]]++] = (uint32_t)h;
    std::vector<uint32_t> rep(nh);  // the first half-edge of the same edge
    std::vector<std::pair<uint32_t, uint32_t>> big;
    for (size_t b = 0; b + 1 < start.size(); ++b) {
        const uint32_t j0 = start[b], j1 = start[b + 1];
        if (j1 - j0 <= 32) {
            for (uint32_t j = j0; j < j1; ++j) {
                const uint32_t h = slot[j];
                rep[h] = h;
                for (uint32_t i = j0; i < j; ++i)
                    if (hi_of[slot[i]] == hi_of[h]) {
                        rep[h] = slot[i];
                        break;
                    }
            }
        } else {
            big.clear();
            for (uint32_t j = j0; j < j1; ++j) big.push_back({hi_of[slot[j]], slot[j]});
            std::sort(big.begin(), big.end());
            for (size_t i = 0; i < big.size(); ++i)
                rep[big[i].second] = (i > 0 && big[i].first == big[i - 1].first) ? rep[big[i - 1].second] : big[i].second;
        }
    }
    // edge ids in order of first appearance
    std::vector<uint32_t> face_edge(nh);
    uint32_t n_edges = 0;
    for (size_t h = 0; h < nh; ++h) face_edge[h] = rep[h] == h ? n_edges++ : face_edge[rep[h]];

    std::vector<SilEdge> sil(n_edges);
    for (int64_t f = 0; f < src.np; ++f) {  // silhouette_edge.cpp:28-53
        for (int k = 0; k < 3; ++k) {
            uint64_t i0 = (uint32_t)src.index[f * 3 + k];
            uint64_t i1 = (uint32_t)src.index[f * 3 + (k + 1) % 3];
            uint64_t i2 = (uint32_t)src.index[f * 3 + (k + 2) % 3];
            Vec3 v0 = vert3(src, (int64_t)i0), v1 = vert3(src, (int64_t)i1), v2 = vert3(src, (int64_t)i2);
            bool swapped = false;
            if (i0 > i1) {
                std::swap(i0, i1);
                swapped = true;
            }
            uint32_t e = face_edge[(size_t)f * 3 + k];
            SilEdge &s = sil[e];
            s.v[1] = v0;
            s.v[2] = v1;
            s.v[swapped ? 3 : 0] = v2;
            s.idx[1] = i0;
            s.idx[2] = i1;
            s.idx[swapped ? 3 : 0] = i2;
            s.face[swapped ? 1 : 0] = (uint64_t)f;
            s.orient = swapped ? -1 : 1;
            s.prim = e;
        }
    }
    if (face_edge_out) *face_edge_out = std::move(face_edge);
    return sil;
}

namespace {

// Silhouette geometry used by the cone construction.
inline Vec2 sil_centroid(const SilVertex &s) { return s.v[1]; }
inline Vec3 sil_centroid(const SilEdge &s) { return (s.v[1] + s.v[2]) * 0.5f; }

inline Vec2 sil_n0(const SilVertex &s, bool unit) {  // silhouette_vertex.h:19-25
    Vec2 d = s.v[1] - s.v[0];
    Vec2 n;
    n.v[0] = d.v[1];
    n.v[1] = -d.v[0];
    return unit ? normalized(n) : n;
}
inline Vec2 sil_n1(const SilVertex &s, bool unit) {  // silhouette_vertex.h:28-34
    Vec2 d = s.v[2] - s.v[1];
    Vec2 n;
    n.v[0] = d.v[1];
    n.v[1] = -d.v[0];
    return unit ? normalized(n) : n;
}
// silhouette_edge.h:19-37.  Both use the face through v[0] (the reference's
// normal_1 reads v[2], v[0], v[1]), so the two are the same face normal up to rounding.
inline Vec3 sil_n0(const SilEdge &s, bool unit) {
    Vec3 n = cross(s.v[2] - s.v[1], s.v[0] - s.v[1]);
    return unit ? normalized(n) : n;
}
inline Vec3 sil_n1(const SilEdge &s, bool unit) {
    Vec3 n = cross(s.v[0] - s.v[2], s.v[1] - s.v[2]);
    return unit ? normalized(n) : n;
}
// Both "has face" tests compare a size_t against -1; nothing ever stores -1, so they
// always hold (silhouette_vertex.h:15-16, silhouette_edge.h:13-14).
template <typename S>
inline bool sil_closed(const S &) { return true; }

template <typename S>
inline auto sil_normal(const S &s) {  // normal(): zero + n0 + n1, normalised
    auto n = sil_n0(s, false);
    for (auto &c : n.v) c = 0.f;
    n = n + sil_n0(s, false);
    n = n + sil_n1(s, false);
    return normalized(n);
}

}  // namespace

template <int D>
SnchTree<D> build_snch(const PrimSource<D> &src, const BvhTree<D> &bvh, int n_threads) {
    SnchTree<D> out;
    std::vector<uint32_t> face_edge;
    if constexpr (D == 2) {
        out.raw.assign((size_t)src.nv, SilVertex{});  // snch.cpp:157-184
        for (int64_t e = 0; e < src.np; ++e) {
            uint64_t i0 = (uint32_t)src.index[2 * e], i1 = (uint32_t)src.index[2 * e + 1];
            Vec2 v0 = vert2(src, (int64_t)i0), v1 = vert2(src, (int64_t)i1);
            SilVertex &s0 = out.raw[i0];
            s0.v[1] = v0;
            s0.v[2] = v1;
            s0.idx[1] = i0;
            s0.idx[2] = i1;
            s0.prim = i0;
            SilVertex &s1 = out.raw[i1];
            s1.v[0] = v0;
            s1.v[1] = v1;
            s1.idx[0] = i0;
            s1.idx[1] = i1;
            s1.prim = i1;
        }
    } else {
        out.raw = build_silhouette_edges(src, &face_edge);  // snch.cpp:187-241
    }

    // Per-leaf silhouette lists, duplicates removed only within a leaf (snch.cpp:47-93).
    const size_t nn = bvh.nodes.size();
    out.nodes.assign(nn, SnchNode<D>{});
    std::vector<uint32_t> seen;
    std::unordered_set<uint32_t> seen_big;
    for (size_t i = 0; i < nn; ++i) {
        const FlatNode<D> &bn = bvh.nodes[i];
        SnchNode<D> &sn = out.nodes[i];
        if (bn.n_prims == 0) continue;
        const size_t start = out.ordered.size();
        const bool big = bn.n_prims > 16;
        seen.clear();
        seen_big.clear();
        for (int32_t j = 0; j < bn.n_prims; ++j) {
            const int64_t p = bvh.order[(size_t)(bn.prim_offset + j)];
            for (int k = 0; k < D; ++k) {
                uint32_t sid;
                if constexpr (D == 2)
                    sid = (uint32_t)src.index[2 * p + k];
                else
                    sid = face_edge[(size_t)p * 3 + k];
                bool fresh;
                if (big) {
                    fresh = seen_big.insert(sid).second;
                } else {
                    fresh = std::find(seen.begin(), seen.end(), sid) == seen.end();
                    if (fresh) seen.push_back(sid);
                }
                if (fresh) out.ordered.push_back(sid);
            }
        }
        sn.sil_offset = (int32_t)start;
        sn.n_sil = (int32_t)(out.ordered.size() - start);
    }

    // The node range each cone is computed over, [i, end[i]) in preorder, as the
    // reference's recursion passes it (snch.cpp:151-152): the root gets [0, n); an
    // interior node's right child inherits the node's end, but its left child gets the
    // node's RELATIVE second-child offset as its end.  That end is short of the left
    // subtree's true end by the node's own index, so deeper left subtrees see a
    // truncated range, or an empty one (end <= start): no silhouette is found there and
    // the cone stays invalid (half angle -pi, which the traversal treats as "no cone
    // test").  Kept as the reference builds it, so that node_data() and the traversal's
    // pruning are the reference's.
    std::vector<uint32_t> end(nn);
    {
        std::vector<std::pair<uint32_t, uint32_t>> st;  // (node, end)
        st.push_back({0u, (uint32_t)nn});
        while (!st.empty()) {
            auto [i, e] = st.back();
            st.pop_back();
            end[i] = e;
            const FlatNode<D> &bn = bvh.nodes[i];
            if (bn.n_prims == 0) {
                const uint32_t off = (uint32_t)bn.second_child;
                st.push_back({i + 1, off});
                st.push_back({i + off, e});
            }
        }
    }

    // What the cones read of each listed silhouette, in list order: a node's cone reads
    // every silhouette of its range twice, and the raw silhouettes lie in another order.
    struct ConeIn {
        Vec<D> normal, centroid, n0, n1;  // normal(), centroid, unit face normals
        bool closed;
    };
    const int nt = std::max(1, n_threads);
    std::vector<ConeIn> cin(out.ordered.size());
    auto fill = [&](size_t j0, size_t j1) {
        for (size_t j = j0; j < j1; ++j) {
            const SilOf<D> &s = out.raw[out.ordered[j]];
            cin[j] = ConeIn{sil_normal(s), sil_centroid(s), sil_n0(s, true), sil_n1(s, true), sil_closed(s)};
        }
    };
    if (nt == 1 || cin.size() < 65536) {
        fill(0, cin.size());
    } else {
        std::vector<std::thread> pool;
        const size_t per = (cin.size() + (size_t)nt - 1) / (size_t)nt;
        for (int t = 0; t < nt; ++t)
            pool.emplace_back(fill, std::min(cin.size(), (size_t)t * per), std::min(cin.size(), (size_t)(t + 1) * per));
        for (auto &th : pool) th.join();
    }

    // Cone of every node from all silhouettes below it (snch.cpp:103-154).
    auto cone_of = [&](size_t i) {
        Cone<D> &cone = out.nodes[i].cone;
        const Vec<D> c = bvh.nodes[i].box.centroid();
        bool any = false, all_closed = true;
        for (size_t k = i; k < end[i]; ++k) {
            const SnchNode<D> &sn = out.nodes[k];
            for (int32_t j = 0; j < sn.n_sil; ++j) {
                const ConeIn &s = cin[(size_t)(sn.sil_offset + j)];
                cone.axis = cone.axis + s.normal;
                cone.radius = std::max(cone.radius, norm(s.centroid - c));
                all_closed = all_closed && s.closed;
                any = true;
            }
        }
        if (!any) {
            cone.half_angle = -kPiF;
        } else if (!all_closed) {
            cone.half_angle = kPiF;
        } else {
            float an = norm(cone.axis);
            if (an > kEps) {
                cone.axis = cone.axis / an;
                cone.half_angle = 0.f;
                for (size_t k = i; k < end[i]; ++k) {
                    const SnchNode<D> &sn = out.nodes[k];
                    for (int32_t j = 0; j < sn.n_sil; ++j) {
                        const ConeIn &s = cin[(size_t)(sn.sil_offset + j)];
                        float a0 = std::acos(std::clamp(dot(cone.axis, s.n0), -1.f, 1.f));
                        float a1 = std::acos(std::clamp(dot(cone.axis, s.n1), -1.f, 1.f));
                        cone.half_angle = std::max(cone.half_angle, std::max(a0, a1));
                    }
                }
            }
        }
    };
    if (nt == 1 || nn < 4096) {
        for (size_t i = 0; i < nn; ++i) cone_of(i);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t)
            pool.emplace_back([&, t]() {
                for (size_t i = (size_t)t; i < nn; i += (size_t)nt) cone_of(i);
            });
        for (auto &th : pool) th.join();
    }
    return out;
}

// ---------------------------------------------------------------------------
// Reference float layouts (bvh.h:420-424, snch.h:334-340, line_segment.h:104-108,
// triangle.h:143-147, silhouette_vertex.h:48-54, silhouette_edge.h:106-112)
// ---------------------------------------------------------------------------

template <int D>
std::vector<float> ref_node_data(const BvhTree<D> &t) {
    std::vector<float> r;
    r.reserve(t.nodes.size() * (2 * D + 3));
    for (const auto &n : t.nodes) {
        for (int k = 0; k < D; ++k) r.push_back(n.box.lo.v[k]);
        for (int k = 0; k < D; ++k) r.push_back(n.box.hi.v[k]);
        r.push_back((float)n.prim_offset);
        r.push_back((float)n.second_child);
        r.push_back((float)n.n_prims);
    }
    return r;
}

template <int D>
std::vector<float> ref_prim_data(const PrimSource<D> &src, const BvhTree<D> &t) {
    std::vector<float> r;
    r.reserve(t.order.size() * (D * D + 1));
    for (int32_t p : t.order) {
        for (int k = 0; k < D; ++k) {
            Vec<D> v = vert(src, src.index[(int64_t)p * D + k]);
            for (int c = 0; c < D; ++c) r.push_back(v.v[c]);
        }
        r.push_back((float)p);
    }
    return r;
}

template <int D>
std::vector<float> ref_snch_node_data(const BvhTree<D> &t, const SnchTree<D> &s) {
    std::vector<float> r;
    r.reserve(t.nodes.size() * (3 * D + 7));
    for (size_t i = 0; i < t.nodes.size(); ++i) {
        const auto &n = t.nodes[i];
        const auto &sn = s.nodes[i];
        for (int k = 0; k < D; ++k) r.push_back(n.box.lo.v[k]);
        for (int k = 0; k < D; ++k) r.push_back(n.box.hi.v[k]);
        for (int k = 0; k < D; ++k) r.push_back(sn.cone.axis.v[k]);
        r.push_back(sn.cone.half_angle);
        r.push_back(sn.cone.radius);
        r.push_back((float)n.prim_offset);
        r.push_back((float)n.second_child);
        r.push_back((float)n.n_prims);
        r.push_back((float)sn.sil_offset);
        r.push_back((float)sn.n_sil);
    }
    return r;
}

static void push_sil(std::vector<float> &r, const SilVertex &s) {
    for (int k = 0; k < 3; ++k) {
        r.push_back(s.v[k].v[0]);
        r.push_back(s.v[k].v[1]);
    }
    for (int k = 0; k < 3; ++k) r.push_back((float)s.idx[k]);
    r.push_back((float)s.prim);
}
static void push_sil(std::vector<float> &r, const SilEdge &s) {
    for (int k = 0; k < 4; ++k)
        for (int c = 0; c < 3; ++c) r.push_back(s.v[k].v[c]);
    for (int k = 0; k < 4; ++k) r.push_back((float)s.idx[k]);
    r.push_back((float)s.face[0]);
    r.push_back((float)s.face[1]);
    r.push_back((float)s.prim);
}

template <int D>
std::vector<float> ref_silhouette_data(const SnchTree<D> &s, bool ordered) {
    std::vector<float> r;
    if (ordered) {
        for (uint32_t k : s.ordered) push_sil(r, s.raw[k]);
    } else {
        for (const auto &x : s.raw) push_sil(r, x);
    }
    return r;
}

template std::string validate_source<2>(const PrimSource<2> &);
template std::string validate_source<3>(const PrimSource<3> &);
template BvhTree<2> build_bvh<2>(const PrimSource<2> &, int, int);
template BvhTree<3> build_bvh<3>(const PrimSource<3> &, int, int);
template SnchTree<2> build_snch<2>(const PrimSource<2> &, const BvhTree<2> &, int);
template SnchTree<3> build_snch<3>(const PrimSource<3> &, const BvhTree<3> &, int);
template std::vector<float> ref_node_data<2>(const BvhTree<2> &);
template std::vector<float> ref_node_data<3>(const BvhTree<3> &);
template std::vector<float> ref_prim_data<2>(const PrimSource<2> &, const BvhTree<2> &);
template std::vector<float> ref_prim_data<3>(const PrimSource<3> &, const BvhTree<3> &);
template std::vector<float> ref_snch_node_data<2>(const BvhTree<2> &, const SnchTree<2> &);
template std::vector<float> ref_snch_node_data<3>(const BvhTree<3> &, const SnchTree<3> &);
template std::vector<float> ref_silhouette_data<2>(const SnchTree<2> &, bool);
template std::vector<float> ref_silhouette_data<3>(const SnchTree<3> &, bool);

}  // namespace gqb
