// Internal declarations shared by the C-ABI translation units (capi.cpp, server.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gq.h"
#include "device/queries.cuh"
#include "host/flatten.hpp"
#include "host/scene_build.hpp"

namespace gqi {

// Records `msg` as the calling thread's last error and returns `s`.
gq_status fail(gq_status s, const std::string &msg);
gq_status fail_cuda(cudaError_t e, const char *what);

// Selects `dev` for the lifetime of the guard and restores the previous device.
struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace gqi

struct gq_scene {
    int dim = 0;
    int device = 0;
    std::vector<float> verts;
    std::vector<int32_t> index;
    int64_t nv = 0, np = 0;
    gqb::BvhTree<2> t2;
    gqb::BvhTree<3> t3;
    gqb::SnchTree<2> s2;
    gqb::SnchTree<3> s3;
    bool has_snch = false, has_wide = false, has_wide16 = false;
    int exact_stack = 0, wide_stack = 0;
    int64_t n_wide = 0, n_sil = 0;
    std::vector<float> wide_words;  // host copy of the wide nodes (host-only scenes)
    std::vector<float> wide16_words;  // and of their 16-bit bounds records
    std::vector<float> spair_words, sil_words;  // host copies of the SNCH pairs and silhouette records (idem)
    std::vector<void *> allocs;
    int64_t device_bytes = 0;
    gqd::DevScene dev{};
    gq_tuning tune[3] = {};
    // what a saved scene needs besides the device arrays
    size_t image_bytes[6] = {};  // pairs, prims, spheres, wide nodes, SNCH pairs, silhouettes
    int max_prims_in_node = 10;
    int64_t n_nodes = 0;
    int max_depth = 0;
    // host trees (reference arrays): absent in a loaded scene until first asked for
    bool trees_ready = true;
    bool gpu_built = false;  // tree built on the device: no host SAH trees to describe it
    std::mutex tree_mu;
    // closest_silhouette_baseline's list (Mesh / Polyline .silhouettes), uploaded on first use
    const void *base_sils = nullptr;
    int64_t n_base_sils = -1;
    std::mutex base_mu;
    // the SNCH's raw silhouette list as float positions for the FP64 scan, uploaded on first use
    const void *f64_sils = nullptr;
    int64_t n_f64_sils = -1;

    ~gq_scene() {
        if (device < 0 || allocs.empty()) return;
        gqi::DeviceGuard g(device);
        for (void *p : allocs) cudaFree(p);
    }

    template <typename T>
    gq_status upload(const std::vector<T> &v, const void **dst) {
        *dst = nullptr;
        if (v.empty()) return GQ_OK;
        void *p = nullptr;
        const size_t bytes = v.size() * sizeof(T);
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) return gqi::fail(GQ_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        allocs.push_back(p);
        device_bytes += (int64_t)bytes;
        e = cudaMemcpy(p, v.data(), bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return gqi::fail_cuda(e, "cudaMemcpy");
        *dst = p;
        return GQ_OK;
    }
};
