// CPU scene builders: binned-SAH BVH and the SNCH (spatialized normal cone
// hierarchy) on top of it, for 2D line segments and 3D triangles.
//
// Restates gQuery's builder algorithm (src/shapes/bvh.cpp:29-327,
// src/shapes/snch.cpp:12-241, src/shapes/silhouette_edge.cpp:5-60) without Eigen.
// The output is bit-identical to the reference's tree as it comes out of a
// single-threaded build: the reference only reaches its thread pool for nodes
// above 131,072 primitives, where it throws because the pool is never
// initialised; here those subtrees are built by the same recursion, optionally
// on worker threads, and placed exactly where a serial left-first build puts them.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "geom.hpp"

namespace gqb {

// One node of the depth-first flattened binary BVH (include/shapes/bvh.h:408-424).
// Preorder: the left child of an interior node i is i+1, the right child is
// i + second_child.  Leaves own ordered primitives [prim_offset, prim_offset+n_prims).
template <int D>
struct FlatNode {
    Box<D> box;
    int32_t prim_offset = 0;   // leaves only (0 on interior nodes, as value-initialised in the reference)
    int32_t second_child = 0;  // interior only (0 on leaves)
    int32_t n_prims = 0;       // 0 marks an interior node
    int32_t axis = 0;
};

template <int D>
struct BvhTree {
    std::vector<FlatNode<D>> nodes;
    std::vector<int32_t> order;  // ordered primitive slot -> original primitive index
    int max_depth = 0;
};

// Silhouette vertex of a polyline (include/shapes/silhouette_vertex.h:6-55).
// v[1] is the vertex, v[0]/v[2] its predecessor/successor.  Unset fields stay
// zero, exactly like the value-initialised records of the reference.
struct SilVertex {
    Vec2 v[3] = {};
    uint64_t idx[3] = {0, 0, 0};
    uint64_t prim = 0;
};

// Silhouette edge of a mesh (include/shapes/silhouette_edge.h:6-57).
// v[1], v[2] are the edge end points; v[0] / v[3] the opposite vertices of the
// face on either side (v[3] stays (0,0,0) on a boundary edge).
struct SilEdge {
    Vec3 v[4] = {};
    uint64_t idx[4] = {0, 0, 0, 0};
    uint64_t face[2] = {0, 0};
    uint64_t prim = 0;
    // +1 when the stored end points v[1] -> v[2] follow the winding of the face that
    // wrote them last with its index pair in ascending order, -1 otherwise: on a
    // consistently wound mesh the face normals of the record point outward exactly
    // when this is +1 (used only to orient the node bounds of the flattening pass)
    int8_t orient = 1;
};

template <int D>
struct Cone {
    Vec<D> axis = Vec<D>::splat(0.f);
    float half_angle = kPiF;  // bounding_cone.h:15  default half angle pi
    float radius = 0.f;
};

template <int D>
struct SnchNode {
    Cone<D> cone;
    int32_t sil_offset = 0;
    int32_t n_sil = 0;
};

template <int D>
using SilOf = std::conditional_t<D == 2, SilVertex, SilEdge>;

template <int D>
struct SnchTree {
    std::vector<SnchNode<D>> nodes;          // parallel to BvhTree::nodes
    std::vector<SilOf<D>> raw;               // one per vertex (2D) / unique edge (3D)
    std::vector<uint32_t> ordered;           // per-leaf silhouette list -> index into raw
};

struct BuildError {
    std::string what;
};

// Primitive records as the builder sees them.
template <int D>
struct PrimSource {
    const float *verts;    // [nv][D]
    int64_t nv;
    const int32_t *index;  // [np][D]
    int64_t np;
};

// Validates the inputs (index range, counts, finite coordinates); returns an empty string when fine.
template <int D>
std::string validate_source(const PrimSource<D> &src);

template <int D>
BvhTree<D> build_bvh(const PrimSource<D> &src, int max_prims_in_node, int n_threads);

template <int D>
SnchTree<D> build_snch(const PrimSource<D> &src, const BvhTree<D> &bvh, int n_threads);

// The silhouette list of a Polyline (Polyline.configure_silhouette, polyline.py:44-122):
// vertices in order of first appearance in the edge list that have both a predecessor
// and a successor, without those whose two edges are nearly collinear
// (|normalize(b - a) . normalize(c - b)| >= 1 - 1e-5 in FP32); prim = position in the
// first-appearance order.  closest_silhouette_baseline scans this list.
std::vector<SilVertex> build_polyline_silhouettes(const PrimSource<2> &src);

// Raw silhouette edges in first-appearance edge order (silhouette_edge.cpp:5-60).
// face_edge[3*f + k] receives the edge index of face f's k-th edge (k -> k+1).
std::vector<SilEdge> build_silhouette_edges(const PrimSource<3> &src,
                                            std::vector<uint32_t> *face_edge);

// Reference float layouts (the arrays gquery_ext hands to the traversal).
template <int D>
std::vector<float> ref_node_data(const BvhTree<D> &t);                    // stride 2D+3
template <int D>
std::vector<float> ref_prim_data(const PrimSource<D> &src, const BvhTree<D> &t);  // stride 5 / 10
template <int D>
std::vector<float> ref_snch_node_data(const BvhTree<D> &t, const SnchTree<D> &s);  // stride 13 / 16
template <int D>
std::vector<float> ref_silhouette_data(const SnchTree<D> &s, bool ordered);  // stride 10 / 19

Vec2 vert2(const PrimSource<2> &src, int64_t i);
Vec3 vert3(const PrimSource<3> &src, int64_t i);

}  // namespace gqb
