// Device-side scene layout produced by the flattening pass (host) and read by the
// traversal kernels.  All records are 16-byte aligned and read with 128-bit loads.
//
// Binary layout ("exact" kernels: same visit order as gQuery's traversal)
// -----------------------------------------------------------------------
// gQuery pops a node, then reads both children's boxes (bvh.py:159-167).  Here the
// two child boxes of every interior node sit together in one "pair" record, so a
// pop costs one record read.  A child reference is
//     ref >= 0 : interior child, index of its own pair record
//     ref <  0 : leaf child, ~ref = first ordered primitive (or silhouette); the
//                leaf's items run until a record whose `last` flag is set.
// Pair records are numbered in preorder of the interior nodes.
//
// Wide layout ("wide" kernels: quantised 8-wide nodes)
// ----------------------------------------------------
// The binary tree is collapsed into nodes of up to 8 children (leaves unchanged).
// Child boxes are stored as 8-bit offsets on a per-axis grid
//     lo = origin + qlo * 2^e,  hi = origin + qhi * 2^e
// rounded outward on the host so that the decoded box contains the exact child box
// in fp32 arithmetic: a query visits a superset of the nodes it would visit with
// exact boxes and finds the same nearest primitive.
#pragma once

#include <stdint.h>

#define GQ_STACK_EXACT 64   // gQuery's traversal stack size (bvh.py:132)
#define GQ_STACK_WIDE 96
#define GQ_WIDTH 8

#ifdef __cplusplus
extern "C" {
#endif

// Leaf item flags (the .w / last word of primitive and silhouette records).
#define GQ_ITEM_LAST 1u      // last item of its leaf
#define GQ_ITEM_VALID 2u     // silhouette vertex: both neighbour indices present

// 2D segment: (a.x, a.y, b.x, b.y) | (orig_index, flags, 0, 0)          32 B
typedef struct {
    float ax, ay, bx, by;
    int32_t index, flags, pad0, pad1;
} gq_seg_t;

// 3D triangle: (a.xyz, b.x) | (b.yz, c.xy) | (c.z, orig_index, flags, 0)  48 B
typedef struct {
    float ax, ay, az, bx;
    float by, bz, cx, cy;
    float cz;
    int32_t index, flags, pad;
} gq_tri_t;

// Bounding sphere of an ordered triangle, parallel to the triangle records: centre
// and radius, the radius rounded up so the sphere contains the triangle in exact
// arithmetic; its sign bit repeats the triangle's end-of-leaf flag.            16 B
typedef struct {
    float cx, cy, cz, r;
} gq_tsph_t;

// 2D silhouette vertex: (a.xy, b.xy) | (c.xy, prim_id, flags)            32 B
typedef struct {
    float ax, ay, bx, by;
    float cx, cy;
    int32_t prim, flags;
} gq_silv_t;

// 3D silhouette edge: end points a, b and the unit normals of its two faces,
// n0 of (a, b, c) and n1 of (a, d, b), computed once on the host with the
// FP32 operations the reference applies per test (silhouette_edge.py:28-34), and
// span0 = n0 . (b - a), span1 = n1 . (b - a) for the pre-test of sil_filter.h
// (valid when flags has GQ_SIL_FILTER).                                       64 B
typedef struct {
    float ax, ay, az, bx;
    float by, bz, n0x, n0y;
    float n0z, n1x, n1y, n1z;
    int32_t prim, flags;
    float span0, span1;
} gq_sile_t;

// Binary BVH pair records.  sub_l / sub_r: a child whose subtree holds at most
// GQ_COLLAPSE_MAX primitives (in one run of the ordered primitives, as every subtree's
// are) is described again as first | count << 24 (first < 2^24), and the warp-coherent
// closest-point walk tests that run as one leaf instead of walking the subtree; 0 for
// larger subtrees (and in device-built trees).  The exact walks keep the references.
#define GQ_COLLAPSE_MAX 6
typedef struct {  // 2D, 48 B: left box, right box, refs
    float l_lox, l_loy, l_hix, l_hiy;
    float r_lox, r_loy, r_hix, r_hiy;
    int32_t ref_l, ref_r, sub_l, sub_r;
} gq_pair2_t;

typedef struct {  // 3D, 64 B
    float l_lox, l_loy, l_loz, l_hix;
    float l_hiy, l_hiz, r_lox, r_loy;
    float r_loz, r_hix, r_hiy, r_hiz;
    int32_t ref_l, ref_r, sub_l, sub_r;
} gq_pair3_t;

// Binary SNCH pair records: child box + cone (axis, half angle, radius).
typedef struct {  // 2D, 80 B
    float l_lox, l_loy, l_hix, l_hiy;
    float l_ax, l_ay, l_half, l_rad;
    float r_lox, r_loy, r_hix, r_hiy;
    float r_ax, r_ay, r_half, r_rad;
    int32_t ref_l, ref_r, pad0, pad1;
} gq_spair2_t;

// 3D, 160 B (five 32-byte sectors): the reference's boxes and cones of both children
// (96 B), then per child the node bound of sil_filter.h (axis, delta, cos and sin of the
// normal cone's half-angle, lo, hi; the centre is the child box's) that proves a child
// free of silhouettes for a query point.
typedef struct {
    float l_lox, l_loy, l_loz, l_hix;
    float l_hiy, l_hiz, l_ax, l_ay;
    float l_az, l_half, l_rad, r_lox;
    float r_loy, r_loz, r_hix, r_hiy;
    float r_hiz, r_ax, r_ay, r_az;
    float r_half, r_rad;
    int32_t ref_l, ref_r;
    float l_b[8], r_b[8];
} gq_spair3_t;
#ifdef __cplusplus
static_assert(sizeof(gq_spair3_t) == 160, "gq_spair3_t is five 32-byte sectors");
#endif

// Quantised 8-wide node, 3D: 96 B (three 32-byte sectors).
//   origin.xyz, meta = exp_x | exp_y << 8 | exp_z << 16 | nchild << 24 (exps biased by 127)
//   ref[8]      child references (same encoding as pair refs), or a run child: a binary
//               subtree of at most GQ_COLLAPSE_MAX primitives as 0x80000000 | first |
//               count << 24 (bit 30 clear, where ~first has it set), tested as one leaf
//   q[6][8]     qlo_x, qlo_y, qlo_z, qhi_x, qhi_y, qhi_z (8 bits each)
typedef struct {
    float ox, oy, oz;
    uint32_t meta;
    int32_t ref[8];
    uint8_t q[6][8];
} gq_wnode3_t;

// Quantised 8-wide node, 2D: 80 B.
//   origin.xy, meta = exp_x | exp_y << 8 | nchild << 24
typedef struct {
    float ox, oy;
    uint32_t meta, pad;
    int32_t ref[8];
    uint8_t q[4][8];  // qlo_x, qlo_y, qhi_x, qhi_y
} gq_wnode2_t;

// 16-bit child bounds of the 8-wide node with the same index (same children, same
// references, which stay in the 8-bit node): an origin and exponents of its own for the
// finer grid, and the bounds as 16-bit steps (decoded as fma(2^23 + q, 2^e, origin)).
// 3D: 112 B (seven 16-byte words); 2D: 80 B.
typedef struct {
    float ox, oy, oz;
    uint32_t meta;       // exp_x | exp_y << 8 | exp_z << 16 | nchild << 24 (exps biased by 127)
    uint16_t q[6][8];    // qlo_x, qlo_y, qlo_z, qhi_x, qhi_y, qhi_z
} gq_wq16_3_t;
typedef struct {
    float ox, oy;
    uint32_t meta, pad;  // exp_x | exp_y << 8 | nchild << 24
    uint16_t q[4][8];    // qlo_x, qlo_y, qhi_x, qhi_y
} gq_wq16_2_t;

#ifdef __cplusplus
}
#endif
