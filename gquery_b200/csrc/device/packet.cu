// Single-scene warp-coherent closest point (see packet.cuh): persistent warps take 32
// consecutive queries of the Morton order at a time.
#include <algorithm>

#include "packet.cuh"
#include "records.cuh"

namespace gqd {

namespace {

constexpr int kMaxBlock = 256;

__device__ __forceinline__ float qget(const gq_vecs &v, int64_t i, int k) {
    return v.ptr[(int64_t)k * v.comp_stride + i * v.elem_stride];
}

template <int D, int LAYOUT, bool MINFIRST, int STK, bool COMPACT = false>
__global__ void __launch_bounds__(kMaxBlock) k_cp_packet(DevScene s, gq_vecs q, int64_t n, const int32_t *perm,
                                                         gq_cp_out o, unsigned long long *counter) {
    const unsigned lane = threadIdx.x & 31u;
    // (ref, this lane's key) per entry; refs are the same in every lane
    int2 plain[COMPACT ? 1 : STK];
    __shared__ int refs[COMPACT ? kMaxBlock / 32 : 1][COMPACT ? STK : 1];
    __half keys[COMPACT ? STK : 1];
    pkt::PStack<COMPACT> stk = [&]() {
        if constexpr (COMPACT)
            return pkt::PStack<true>{refs[threadIdx.x >> 5], keys};
        else
            return pkt::PStack<false>(plain);
    }();
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
        pkt::closest_point<D, LAYOUT, MINFIRST, STK, COMPACT>(s, __ballot_sync(0xffffffffu, alive), p, r, idx, ovf,
                                                                     stk);
        if (ovf && lane == 0 && s.err) atomicOr(s.err, GQ_DEVERR_STACK);
        if (alive) {
            if (D == 3)
                cp3_record(s.prims, idx, (idx >= 0) && !ovf, p[0], p[1], p[D - 1], o, n, qi);
            else
                cp2_record(s.prims, idx, (idx >= 0) && !ovf, p[0], p[D - 1], o, n, qi);
        }
    }
}

template <int D, int LAYOUT, bool MINFIRST, int STK, bool COMPACT = false>
cudaError_t launch(const DevScene &s, int block, gq_vecs q, int64_t n, const int32_t *perm, const gq_cp_out &o,
                   unsigned long long *counter, cudaStream_t st) {
    static int bps[3] = {0, 0, 0}, n_sm = 0;
    int slot = block_slot(block);
    if (slot < 0) slot = 1, block = 128;
    if (!bps[slot]) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_cp_packet<D, LAYOUT, MINFIRST, STK, COMPACT>, block, 0);
        bps[slot] = b < 1 ? 1 : b;
    }
    const int64_t warps = (n + 31) / 32;
    const int64_t want = std::min<int64_t>((int64_t)bps[slot] * n_sm, (warps * 32 + block - 1) / block);
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    k_cp_packet<D, LAYOUT, MINFIRST, STK, COMPACT><<<dim3((unsigned)want), block, 0, st>>>(s, q, n, perm, o,
                                                                                                counter);
    return cudaGetLastError();
}

template <int D, int LAYOUT, bool MINFIRST>
cudaError_t launch_stk(const DevScene &s, const Tune &t, gq_vecs q, int64_t n, const int32_t *perm,
                       const gq_cp_out &o, unsigned long long *counter, cudaStream_t st) {
    if (t.packet == 2) {  // the compact stack (FP16 keys, one node word per warp)
        if (t.stack == 32) return launch<D, LAYOUT, MINFIRST, 32, true>(s, t.block, q, n, perm, o, counter, st);
        return launch<D, LAYOUT, MINFIRST, pkt::kPStack, true>(s, t.block, q, n, perm, o, counter, st);
    }
    if (t.stack == 32) return launch<D, LAYOUT, MINFIRST, 32>(s, t.block, q, n, perm, o, counter, st);
    return launch<D, LAYOUT, MINFIRST, pkt::kPStack>(s, t.block, q, n, perm, o, counter, st);
}

}  // namespace

cudaError_t launch_cp_packet(const DevScene &s, int layout, const Tune &t, gq_vecs q, int64_t n,
                             const int32_t *perm, const gq_cp_out &o, unsigned long long *counter, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    // layout: 0 binary pairs, 1 quantised 8-wide (children sorted), 2 quantised 8-wide (nearest first)
    if (s.dim == 2) return launch_stk<2, 0, false>(s, t, q, n, perm, o, counter, st);
    if (layout == 2) return launch_stk<3, 1, true>(s, t, q, n, perm, o, counter, st);
    if (layout == 1) return launch_stk<3, 1, false>(s, t, q, n, perm, o, counter, st);
    return launch_stk<3, 0, false>(s, t, q, n, perm, o, counter, st);
}

}  // namespace gqd
