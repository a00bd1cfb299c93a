// Closest-point queries that allocate no device memory.
//
// Some callers cannot allocate device memory while they query: plugins whose host
// application owns every device allocation and passes in only input and output
// buffers, or real-time loops that must not touch an allocator at all (cudaMalloc can
// synchronise the device and take unbounded time).  For
// them the per-call scratch of a closest-point query (the work counter of the
// warp-coherent / persistent kernels and the Morton-sort workspace) lives in a
// file-scope device array of fixed size, so at most kNoAllocMaxQueries queries fit
// in one call.
//
// The array exists once per device that loads the library and stays allocated until
// the process exits.  Every call on a device shares it: calls whose kernels overlap on
// the GPU (different streams without ordering between them) race on it.  Each call
// rewrites everything it reads (the counter is cleared on the stream, the permutation
// and sort buffers are fully written), so stale contents of an earlier call never leak.
#include <mutex>

#include "queries.cuh"

namespace gqd {

namespace {

constexpr int64_t kNoAllocMaxQueries = 65536;
constexpr size_t kCounterBytes = 256;
constexpr size_t kPermBytes = kNoAllocMaxQueries * 4;
constexpr size_t kSortBytes = 3 * kNoAllocMaxQueries * 4 + (1u << 20);  // key/value buffers + radix-sort temp
constexpr size_t kNoAllocBytes = kCounterBytes + kPermBytes + kSortBytes;

// The scratch itself.  Host code only sees a host-side stand-in under this name; the
// device address comes from cudaGetSymbolAddress (see device_scratch()).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_addr[kMaxDevices] = {};

// Device address of the scratch on the current device, looked up once per device with
// that device current.  The first call on a device does this lookup, so it should not
// happen while a stream is being captured.  The address belongs to the device's primary
// context: after cudaDeviceReset, or from another context, it is not valid (the header
// says so to callers).
cudaError_t device_scratch(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return cudaSuccess;
}

}  // namespace

int64_t noalloc_max_queries() { return kNoAllocMaxQueries; }

cudaError_t noalloc_closest_point(const DevScene &s, int variant, const Tune &t, gq_vecs q, int64_t n, int sort,
                                  const gq_cp_out &o, cudaStream_t st) {
    if (n < 0 || n > kNoAllocMaxQueries) return cudaErrorInvalidValue;
    if (n == 0) return cudaSuccess;
    void *base = nullptr;
    cudaError_t e = device_scratch(&base);
    if (e != cudaSuccess) return e;
    unsigned long long *counter = reinterpret_cast<unsigned long long *>(base);
    int32_t *perm = reinterpret_cast<int32_t *>(static_cast<unsigned char *>(base) + kCounterBytes);
    void *sort_ws = static_cast<unsigned char *>(base) + kCounterBytes + kPermBytes;
    const int32_t *order = nullptr;
    if (sort && n >= 2) {
        if (morton_scratch_bytes(n) > kSortBytes) return cudaErrorInvalidValue;
        e = morton_order(s, q, n, perm, sort_ws, kSortBytes, st);
        if (e != cudaSuccess) return e;
        order = perm;
    }
    return launch_cp(s, variant, t, q, n, order, o, counter, st);
}

}  // namespace gqd
