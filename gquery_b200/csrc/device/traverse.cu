// Closest-point and ray traversals over the binary BVH ("exact": gQuery's visit
// order, bvh.py:127-276 / bvh3d.py:108-239) and over the quantised 8-wide BVH
// ("wide"), run by one per-lane state machine and one launch driver.
//
// Exact variant.  Every decision of the reference is reproduced bit for bit.  The
// nearer child continues in registers instead of being pushed and popped at once
// (the pop-time test `dist <= r_max` is kept).  Optional, outcome-preserving cuts
// (CFG bits): skip a box's square roots when the squared distance already decides
// the test (sqrt is monotone and correctly rounded; 2^-20 margin), and skip a
// triangle whose bounding sphere proves it cannot beat r_max.
//
// Wide variant.  Child boxes are decoded from 8-bit offsets with one byte-permute
// and one fma each; box tests run on squared distances with a 2^-18 slack so no box
// that can hold a strictly closer primitive is skipped; the nearest child continues
// in registers and the other hits are pushed farthest first.
//
// Scheduling.  "while-while" (CFG bit 2): a lane keeps descending interior nodes
// until it reaches a leaf, then all lanes of the warp test their leaves together.
// Persistent launch: warps stay resident and a lane that finished its query takes the
// next unclaimed one (warp-aggregated atomic on a per-call counter).
#include <algorithm>
#include <cstdlib>

#include "prim.cuh"
#include "queries.cuh"
#include "records.cuh"

#include "traverse.cuh"

namespace gqd {

namespace {

using namespace trav;
constexpr int kMaxBlock = 256;


// One query per thread.
template <int D, bool RAY, bool WIDE, int CFG>
__global__ void __launch_bounds__(kMaxBlock) k_trav(DevScene s, gq_vecs a, gq_vecs b, const float *rmax_in, int64_t n,
                                                 const int32_t *perm, gq_cp_out oc, gq_ray_out orr) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t qi = perm ? (int64_t)__ldg(perm + i) : i;
    Stack<WIDE> stk;
    Lane<D, RAY, WIDE> L;
    lane_init(s, L, a, b, rmax_in, qi);
    while (!lane_run<D, RAY, WIDE, CFG>(s, L, stk, 1 << 30)) {
    }
    lane_write(s, L, qi, n, oc, orr);
}

// Persistent warps with lane refill.
template <int D, bool RAY, bool WIDE, int CFG>
__global__ void __launch_bounds__(kMaxBlock) k_trav_persist(DevScene s, gq_vecs a, gq_vecs b, const float *rmax_in,
                                                         int64_t n, const int32_t *perm, gq_cp_out oc,
                                                         gq_ray_out orr, unsigned long long *counter, int budget) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    Stack<WIDE> stk;
    Lane<D, RAY, WIDE> L;
    int64_t qi = -1;
    bool live = false, drained = false;
    for (;;) {
        if (!drained) {
            const unsigned need = __ballot_sync(0xffffffffu, !live);
            if (need) {
                const int leader = __ffs(need) - 1;
                unsigned long long base = 0;
                if ((int)lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(need));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (base + __popc(need) >= (unsigned long long)n) drained = true;
                if (!live) {
                    const unsigned long long mine = base + __popc(need & below);
                    if (mine < (unsigned long long)n) {
                        qi = perm ? (int64_t)__ldg(perm + mine) : (int64_t)mine;
                        lane_init(s, L, a, b, rmax_in, qi);
                        live = true;
                    }
                }
            }
        }
        if (!__any_sync(0xffffffffu, live)) break;
        if (live && lane_run<D, RAY, WIDE, CFG>(s, L, stk, budget)) {
            lane_write(s, L, qi, n, oc, orr);
            live = false;
        }
    }
}

template <int D, bool RAY, bool WIDE, int CFG>
cudaError_t launch_cfg(const DevScene &s, const Tune &t, gq_vecs a, gq_vecs b, const float *rmax, int64_t n,
                       const int32_t *perm, const gq_cp_out &oc, const gq_ray_out &orr, unsigned long long *counter,
                       cudaStream_t st) {
    int slot = block_slot(t.block), block = t.block;
    if (slot < 0) slot = 1, block = 128;
    if (t.persist && counter && n > 4096) {
        static int blocks_per_sm[3] = {0, 0, 0}, n_sm = 0;
        if (!blocks_per_sm[slot]) {
            int dev = 0, b = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_trav_persist<D, RAY, WIDE, CFG>, block, 0);
            blocks_per_sm[slot] = b < 1 ? 1 : b;
        }
        const int64_t want = std::min<int64_t>((int64_t)blocks_per_sm[slot] * n_sm, (n + block - 1) / block);
        cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
        if (e != cudaSuccess) return e;
        k_trav_persist<D, RAY, WIDE, CFG><<<dim3((unsigned)want), block, 0, st>>>(
            s, a, b, rmax, n, perm, oc, orr, counter, std::max(1, t.budget));
    } else {
        k_trav<D, RAY, WIDE, CFG>
            <<<dim3((unsigned)((n + block - 1) / block)), block, 0, st>>>(s, a, b, rmax, n, perm, oc, orr);
    }
    return cudaGetLastError();
}

// Per-lane traversal configuration.  Rays over the 8-wide nodes may take the nearest hit
// child first with the other hits pushed in child order (tuning sorted = 0) instead of
// sorting all hits by entry distance, and while-while scheduling (packet = 2).
template <int D, bool RAY, bool WIDE>
cudaError_t launch_kind(const DevScene &s, const Tune &t, gq_vecs a, gq_vecs b, const float *rmax, int64_t n,
                        const int32_t *perm, const gq_cp_out &oc, const gq_ray_out &orr, unsigned long long *counter,
                        cudaStream_t st, bool q16 = false) {
    if constexpr (WIDE) {  // 16-bit child bounds
        if (q16) return launch_cfg<D, RAY, WIDE, CFG_Q16>(s, t, a, b, rmax, n, perm, oc, orr, counter, st);
    }
    if constexpr (RAY && WIDE) {
        const bool minfirst = !t.sorted, ww = t.packet == 2;
        if (minfirst && ww)
            return launch_cfg<D, RAY, WIDE, CFG_MINFIRST | CFG_WW>(s, t, a, b, rmax, n, perm, oc, orr, counter, st);
        if (minfirst) return launch_cfg<D, RAY, WIDE, CFG_MINFIRST>(s, t, a, b, rmax, n, perm, oc, orr, counter, st);
        if (ww) return launch_cfg<D, RAY, WIDE, CFG_WW>(s, t, a, b, rmax, n, perm, oc, orr, counter, st);
    }
    return launch_cfg<D, RAY, WIDE, 0>(s, t, a, b, rmax, n, perm, oc, orr, counter, st);
}

}  // namespace

cudaError_t launch_cp(const DevScene &s, int variant, const Tune &t, gq_vecs q, int64_t n, const int32_t *perm,
                      const gq_cp_out &o, unsigned long long *counter, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const gq_ray_out none{};
    const bool q16 = variant == GQ_VARIANT_WIDE16;
    const bool wide = variant == GQ_VARIANT_WIDE8 || q16;
    if (counter && n >= 32) {
        if (variant == GQ_VARIANT_COHERENT) return launch_cp_packet(s, 0, t, q, n, perm, o, counter, st);
        if (variant == GQ_VARIANT_WIDE8 && t.packet && s.dim == 3)
            return launch_cp_packet(s, t.sorted ? 1 : 2, t, q, n, perm, o, counter, st);
    }
    if (s.dim == 3)
        return wide ? launch_kind<3, false, true>(s, t, q, q, nullptr, n, perm, o, none, counter, st, q16)
                    : launch_kind<3, false, false>(s, t, q, q, nullptr, n, perm, o, none, counter, st);
    return wide ? launch_kind<2, false, true>(s, t, q, q, nullptr, n, perm, o, none, counter, st, q16)
                : launch_kind<2, false, false>(s, t, q, q, nullptr, n, perm, o, none, counter, st);
}

cudaError_t launch_ray(const DevScene &s, int variant, const Tune &t, gq_vecs x, gq_vecs v, const float *r_max,
                       int64_t n, const int32_t *perm, const gq_ray_out &o, unsigned long long *counter,
                       cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const gq_cp_out none{};
    const bool q16 = variant == GQ_VARIANT_WIDE16;
    const bool wide = variant == GQ_VARIANT_WIDE8 || q16;
    if (variant == GQ_VARIANT_WIDE8 && t.packet == 1 && counter && n >= 32)  // one ray per group of 8 lanes
        return launch_ray_group(s, x, v, r_max, n, perm, o, counter, st);
    if (s.dim == 3)
        return wide ? launch_kind<3, true, true>(s, t, x, v, r_max, n, perm, none, o, counter, st, q16)
                    : launch_kind<3, true, false>(s, t, x, v, r_max, n, perm, none, o, counter, st);
    return wide ? launch_kind<2, true, true>(s, t, x, v, r_max, n, perm, none, o, counter, st, q16)
                : launch_kind<2, true, false>(s, t, x, v, r_max, n, perm, none, o, counter, st);
}

}  // namespace gqd
