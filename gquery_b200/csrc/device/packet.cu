// Single-scene warp-coherent closest point (see packet.cuh): persistent warps take 32
// consecutive queries of the Morton order at a time.
#include <algorithm>

#include "packet.cuh"
#include "records.cuh"

namespace gqd {

namespace {

constexpr int kBlock = 128;

__device__ __forceinline__ float qget(const gq_vecs &v, int64_t i, int k) {
    return v.ptr[(int64_t)k * v.comp_stride + i * v.elem_stride];
}

template <int D, int LAYOUT, bool MINFIRST>
__global__ void __launch_bounds__(kBlock) k_cp_packet(DevScene s, gq_vecs q, int64_t n, const int32_t *perm,
                                                      gq_cp_out o, unsigned long long *counter) {
    const unsigned lane = threadIdx.x & 31u;
    int2 stk[pkt::kPStack];  // (ref, this lane's key); refs are the same in every lane
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(counter, 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= (unsigned long long)n) break;
        const int64_t i = (int64_t)base + lane;
        const bool alive = i < n;
        const int64_t qi = alive ? (perm ? (int64_t)__ldg(perm + i) : i) : 0;
        float p[D];
#pragma unroll
        for (int k = 0; k < D; ++k) p[k] = alive ? qget(q, qi, k) : 0.f;
        float r = kInf;
        int idx = -1;
        bool ovf = false;
        pkt::closest_point<D, LAYOUT, MINFIRST>(s, __ballot_sync(0xffffffffu, alive), p, r, idx, ovf, stk);
        if (ovf && lane == 0 && s.err) atomicOr(s.err, GQ_DEVERR_STACK);
        if (alive) {
            if (D == 3)
                cp3_record(s.prims, idx, (idx >= 0) && !ovf, p[0], p[1], p[D - 1], o, n, qi);
            else
                cp2_record(s.prims, idx, (idx >= 0) && !ovf, p[0], p[D - 1], o, n, qi);
        }
    }
}

template <int D, int LAYOUT, bool MINFIRST>
cudaError_t launch(const DevScene &s, gq_vecs q, int64_t n, const int32_t *perm, const gq_cp_out &o,
                   unsigned long long *counter, cudaStream_t st) {
    static int bps = 0, n_sm = 0;
    if (!bps) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_cp_packet<D, LAYOUT, MINFIRST>, kBlock, 0);
        if (bps < 1) bps = 1;
    }
    const int64_t warps = (n + 31) / 32;
    const int64_t want = std::min<int64_t>((int64_t)bps * n_sm, (warps * 32 + kBlock - 1) / kBlock);
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    k_cp_packet<D, LAYOUT, MINFIRST><<<dim3((unsigned)want), kBlock, 0, st>>>(s, q, n, perm, o, counter);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_cp_packet(const DevScene &s, int layout, gq_vecs q, int64_t n, const int32_t *perm,
                             const gq_cp_out &o, unsigned long long *counter, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    // layout: 0 binary pairs, 1 quantised 8-wide (children sorted), 2 quantised 8-wide (nearest first)
    if (s.dim == 2) return launch<2, 0, false>(s, q, n, perm, o, counter, st);
    if (layout == 2) return launch<3, 1, true>(s, q, n, perm, o, counter, st);
    if (layout == 1) return launch<3, 1, false>(s, q, n, perm, o, counter, st);
    return launch<3, 0, false>(s, q, n, perm, o, counter, st);
}

}  // namespace gqd
