// Flattening pass: turns the CPU-built binary BVH / SNCH into the device records of
// layout.h (pair records, leaf item records, quantised 8-wide nodes).
#pragma once

#include <vector>

#include "../layout.h"
#include "scene_build.hpp"

namespace gqb {

template <int D>
struct DeviceImage {
    using Pair = std::conditional_t<D == 2, gq_pair2_t, gq_pair3_t>;
    using Prim = std::conditional_t<D == 2, gq_seg_t, gq_tri_t>;
    using SPair = std::conditional_t<D == 2, gq_spair2_t, gq_spair3_t>;
    using Sil = std::conditional_t<D == 2, gq_silv_t, gq_sile_t>;
    using WNode = std::conditional_t<D == 2, gq_wnode2_t, gq_wnode3_t>;
    using WQ16 = std::conditional_t<D == 2, gq_wq16_2_t, gq_wq16_3_t>;

    // binary BVH
    std::vector<Pair> pairs;
    std::vector<Prim> prims;
    std::vector<gq_tsph_t> spheres;  // 3D only: per ordered triangle
    int32_t root_ref = 0;
    float root_lo[D] = {}, root_hi[D] = {};
    int exact_stack = 0;  // entries the binary traversal needs (max leaf depth + 1)

    // quantised 8-wide BVH, and optionally the same nodes' 16-bit child bounds
    std::vector<WNode> wnodes;
    std::vector<WQ16> wq16;
    int32_t wroot_ref = 0;
    int wide_stack = 0;

    // binary SNCH
    std::vector<SPair> spairs;
    std::vector<Sil> sils;
    int32_t sroot_ref = 0;
};

// Reference encoding of an empty SNCH leaf (never produced by valid inputs).
constexpr int32_t kEmptyLeaf = INT32_MIN;

template <int D>
void flatten_bvh(const PrimSource<D> &src, const BvhTree<D> &t, DeviceImage<D> &img);

// with16: also the 16-bit child bounds of every wide node (img.wq16).
template <int D>
void flatten_wide(const BvhTree<D> &t, DeviceImage<D> &img, bool with16 = false);

// flatten_wide over a binary tree given as pair records (pair i: both child boxes of
// interior node i and their references, leaf = ~primitive record), e.g. one built on
// the device; root box and reference given; deep subtrees on n_threads threads (the
// nodes are the same for any thread count, their numbering not).
template <int D>
void flatten_wide_from_pairs(const std::vector<typename DeviceImage<D>::Pair> &pairs, int32_t root_ref,
                             const float *root_lo, const float *root_hi, DeviceImage<D> &img, int n_threads = 1);

// One silhouette in the device layout (also used for the brute-force silhouette list).
void device_silhouette(const SilVertex &x, gq_silv_t &r);
void device_silhouette(const SilEdge &x, gq_sile_t &r);

template <int D>
void flatten_snch(const BvhTree<D> &t, const SnchTree<D> &s, DeviceImage<D> &img, int n_threads = 1);

// Smallest power-of-two exponent e with qmax * 2^e >= hi - lo (clamped to normal floats).
int quant_exponent(float lo, float hi, int qmax = 255);
// Outward-rounded 8-bit bounds of [clo, chi] on the grid origin + q * 2^e.
void quantise_bounds(float origin, int e, float clo, float chi, uint8_t *qlo, uint8_t *qhi);
// The same with 16-bit steps.
void quantise_bounds16(float origin, int e, float clo, float chi, uint16_t *qlo, uint16_t *qhi);
// Origin (biased for the kernels' decode) and exponent of the grid over the parent box
// [lo, hi] with qmax steps: decode(0) <= lo and decode(qmax) >= hi hold in fp32.
void quant_axis(float lo, float hi, int qmax, float *biased, int *e_out);
// Decoding used by the kernels: origin + q * 2^e in fp32.
float dequant(float origin, int e, int q);

}  // namespace gqb
