// Serving runtime (declared in include/gq.h): one worker thread per server admits
// requests into per-kind device rings, launches steps on a few stream slots and hands
// results back to the requests' host buffers.
//
// Ring.  Each query kind has a ring of `cap` query slots: device arrays for the inputs
// (AoS points / directions, r_max, scene index) and the result fields, and pinned host
// mirrors of all of them.  A request takes `n` contiguous slots (the tail of the ring
// is skipped when it does not fit there) and gives them back when it completes; space
// is reclaimed in allocation order, so it is first-in first-out like the admission.
// The rings' device bytes are the admission budget.
//
// Step.  A step takes, for each kind it serves, the run of admitted requests that are
// contiguous in the ring (at most step_queries queries) and answers them with one
// batch launch; closest-point and ray requests go to the general slots, silhouette
// requests to slots of their own whose launches hold part of the GPU only;
// inside the step a field with C components is stored component-major with stride m
// (the step's query count) from ring offset off * C, which is where the kernel writes
// it and what one device-to-host copy per field brings back.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "device/batch.cuh"
#include "internal.hpp"

using gqi::DeviceGuard;
using gqi::fail;
using gqi::fail_cuda;

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// Component counts of the fields of one query kind in dimension D.
struct Fields {
    int a = 0, b = 0, r = 0;                 // inputs: floats per query
    int p = 0, n = 0, t = 0, d = 0, id = 0;  // outputs: floats / ints per query
    bool onb = false;
    int64_t bytes_per_query() const {
        return 4 * (a + b + r + 1) + 4 * (p + n + t + d + id) + 1 + (onb ? 1 : 0);
    }
};

Fields fields_of(int kind, int D) {
    Fields f;
    f.a = D;
    if (kind == GQ_KIND_CLOSEST_POINT) {
        f.p = D, f.n = D, f.t = D - 1, f.d = 1, f.id = 1;
    } else if (kind == GQ_KIND_INTERSECT) {
        f.b = D, f.r = 1, f.p = D, f.n = D, f.t = D - 1, f.d = 1, f.id = 1, f.onb = true;
    } else {
        f.r = 1, f.p = D, f.d = 1, f.id = 1;
    }
    return f;
}

struct Req {
    gq_request q;
    double t_submit = 0, t_admit = 0, t_launch = 0;
    int64_t phys = 0;  // first ring slot
    size_t alloc = 0;  // allocation sequence number in its ring
    int step = -1;
};

struct Ring {
    Fields f;
    int64_t cap = 0;
    // device arrays and their pinned host mirrors
    float *a = nullptr, *b = nullptr, *r = nullptr, *p = nullptr, *nrm = nullptr, *t = nullptr, *d = nullptr;
    int32_t *sid = nullptr, *id = nullptr;
    uint8_t *valid = nullptr, *onb = nullptr;
    float *ha = nullptr, *hb = nullptr, *hr = nullptr, *hp = nullptr, *hn = nullptr, *ht = nullptr, *hd = nullptr;
    int32_t *hsid = nullptr, *hid = nullptr;
    uint8_t *hvalid = nullptr, *honb = nullptr;
    // FIFO allocation: live slots are [head, tail) in a monotone counter space
    struct Live {
        int64_t end;
        bool released;
    };
    int64_t head = 0, tail = 0;
    size_t first_seq = 0;  // sequence number of live.front()
    std::deque<Live> live;

    bool alloc(int64_t n, int64_t *phys, size_t *seq) {
        if (live.empty()) head = tail = (tail + cap - 1) / cap * cap;  // an empty ring starts over at slot 0
        const int64_t at = tail % cap;
        const int64_t pad = at + n > cap ? cap - at : 0;
        if ((tail - head) + pad + n > cap) return false;
        const int64_t start = tail + pad;
        tail = start + n;
        *phys = start % cap;
        *seq = first_seq + live.size();
        live.push_back({tail, false});
        return true;
    }
    void release(size_t seq) {
        live[seq - first_seq].released = true;
        while (!live.empty() && live.front().released) {
            head = live.front().end;
            live.pop_front();
            ++first_seq;
        }
    }
};

struct Slot {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    int32_t *err = nullptr;
    bool busy = false;
    bool sil_only = false;  // batch mode: this slot answers silhouette requests only
    int step = -1;
    gq_status status = GQ_OK;
    std::vector<Req *> reqs;
    int64_t off[3] = {0, 0, 0}, m[3] = {0, 0, 0};
};

}  // namespace

struct gq_server {
    int dim = 0, device = 0, flags = 0;
    int64_t step_queries = 0, ring_bytes = 0, sil_step_queries = 0;
    float sil_share = 0.8f;  // per silhouette slot
    std::vector<gq_scene *> scenes;
    gqd::DevScene *dev_scenes = nullptr;
    Ring ring[3];
    std::vector<Slot> slots;
    cudaStream_t copy_st = nullptr;
    cudaEvent_t copy_evt = nullptr;
    std::vector<void *> dev_allocs, host_allocs;

    std::thread worker;
    std::mutex mu;  // guards `submitted` and `completed`
    std::condition_variable cv;
    std::deque<Req *> submitted;
    std::vector<gq_completion> completed;
    std::atomic<bool> stop{false};
    std::atomic<int64_t> outstanding{0};

    // worker-only state
    std::deque<Req *> pending[3], admitted[3];
    int next_step = 0;
    int64_t admitted_bytes = 0;
    std::atomic<int64_t> admitted_peak{0}, requests_done{0}, queries_done{0}, steps{0};
    std::atomic<int32_t> launch_error{0};

    ~gq_server() {
        stop = true;
        cv.notify_all();
        if (worker.joinable()) worker.join();
        DeviceGuard g(device);
        for (Slot &s : slots) {
            if (s.st) cudaStreamSynchronize(s.st);
            if (s.done) cudaEventDestroy(s.done);
            if (s.st) cudaStreamDestroy(s.st);
        }
        if (copy_st) cudaStreamSynchronize(copy_st);
        if (copy_evt) cudaEventDestroy(copy_evt);
        if (copy_st) cudaStreamDestroy(copy_st);
        for (void *p : dev_allocs) cudaFree(p);
        for (void *p : host_allocs) cudaFreeHost(p);
        for (int k = 0; k < 3; ++k) {
            for (Req *r : pending[k]) delete r;
            for (Req *r : admitted[k]) delete r;
        }
        for (Slot &s : slots)
            for (Req *r : s.reqs) delete r;
        for (Req *r : submitted) delete r;
    }

    template <typename T>
    cudaError_t dalloc(T **p, int64_t count) {
        *p = nullptr;
        if (count <= 0) return cudaSuccess;
        void *v = nullptr;
        cudaError_t e = cudaMalloc(&v, (size_t)count * sizeof(T));
        if (e == cudaSuccess) dev_allocs.push_back(v), *p = static_cast<T *>(v);
        return e;
    }
    template <typename T>
    cudaError_t halloc(T **p, int64_t count) {
        *p = nullptr;
        if (count <= 0) return cudaSuccess;
        void *v = nullptr;
        cudaError_t e = cudaMallocHost(&v, (size_t)count * sizeof(T));
        if (e == cudaSuccess) host_allocs.push_back(v), *p = static_cast<T *>(v);
        return e;
    }

    cudaError_t make_ring(Ring &R) {
        const Fields &f = R.f;
        const int64_t c = R.cap;
        cudaError_t e = cudaSuccess;
        auto both = [&](auto **dv, auto **hv, int comps) {
            if (e == cudaSuccess) e = dalloc(dv, c * comps);
            if (e == cudaSuccess) e = halloc(hv, c * comps);
        };
        both(&R.a, &R.ha, f.a);
        both(&R.b, &R.hb, f.b);
        both(&R.r, &R.hr, f.r);
        both(&R.p, &R.hp, f.p);
        both(&R.nrm, &R.hn, f.n);
        both(&R.t, &R.ht, f.t);
        both(&R.d, &R.hd, f.d);
        both(&R.sid, &R.hsid, 1);
        both(&R.id, &R.hid, f.id);
        both(&R.valid, &R.hvalid, 1);
        if (f.onb) both(&R.onb, &R.honb, 1);
        return e;
    }

    void finish(Req *r, double t_done, gq_status st) {
        gq_completion c{};
        c.tag = r->q.tag;
        c.t_submit = r->t_submit;
        c.t_admit = r->t_admit;
        c.t_launch = r->t_launch;
        c.t_done = t_done;
        c.n = r->q.n;
        c.kind = r->q.kind;
        c.step = r->step;
        c.status = st;
        {
            std::lock_guard<std::mutex> lk(mu);
            completed.push_back(c);
        }
        ++requests_done;
        queries_done += r->q.n;
        delete r;
        --outstanding;
    }

    // ---- worker stages ----
    bool intake() {
        std::lock_guard<std::mutex> lk(mu);
        if (submitted.empty()) return false;
        for (Req *r : submitted) pending[r->q.kind].push_back(r);
        submitted.clear();
        return true;
    }

    // Admits pending requests while their ring has room and copies their inputs up.
    bool admit() {
        bool any = false;
        const int D = dim;
        for (int k = 0; k < 3; ++k) {
            Ring &R = ring[k];
            int64_t run_lo = -1, run_hi = -1;  // contiguous run of new slots to copy up
            auto flush = [&]() {
                if (run_lo < 0) return;
                const int64_t lo = run_lo, cnt = run_hi - run_lo;
                cudaMemcpyAsync(R.a + lo * D, R.ha + lo * D, (size_t)cnt * D * 4, cudaMemcpyHostToDevice, copy_st);
                if (R.f.b)
                    cudaMemcpyAsync(R.b + lo * D, R.hb + lo * D, (size_t)cnt * D * 4, cudaMemcpyHostToDevice,
                                    copy_st);
                if (R.f.r) cudaMemcpyAsync(R.r + lo, R.hr + lo, (size_t)cnt * 4, cudaMemcpyHostToDevice, copy_st);
                cudaMemcpyAsync(R.sid + lo, R.hsid + lo, (size_t)cnt * 4, cudaMemcpyHostToDevice, copy_st);
                run_lo = run_hi = -1;
            };
            while (!pending[k].empty()) {
                Req *r = pending[k].front();
                int64_t phys;
                size_t seq;
                if (!R.alloc(r->q.n, &phys, &seq)) break;
                pending[k].pop_front();
                r->phys = phys;
                r->alloc = seq;
                r->t_admit = now_s();
                const int64_t n = r->q.n;
                std::memcpy(R.ha + phys * D, r->q.a, (size_t)n * D * 4);
                if (R.f.b) std::memcpy(R.hb + phys * D, r->q.b, (size_t)n * D * 4);
                if (R.f.r) {
                    if (r->q.r_max)
                        std::memcpy(R.hr + phys, r->q.r_max, (size_t)n * 4);
                    else
                        std::fill(R.hr + phys, R.hr + phys + n, __builtin_inff());
                }
                std::fill(R.hsid + phys, R.hsid + phys + n, r->q.scene);
                if (run_lo >= 0 && phys == run_hi) {
                    run_hi += n;
                } else {
                    flush();
                    run_lo = phys;
                    run_hi = phys + n;
                }
                admitted_bytes += n * R.f.bytes_per_query();
                if (admitted_bytes > admitted_peak) admitted_peak = admitted_bytes;
                admitted[k].push_back(r);
                any = true;
            }
            flush();
        }
        if (any) cudaEventRecord(copy_evt, copy_st);
        return any;
    }

    // Device output record of one kind for a step range; fields component-major with stride m.
    static void step_outputs(Ring &R, int64_t off, gq_cp_out *co, gq_ray_out *ro, gq_sil_out *so) {
        const Fields &f = R.f;
        if (co) *co = gq_cp_out{R.valid + off, R.p + off * f.p, R.nrm + off * f.n, R.t + off * f.t, R.d + off, R.id + off};
        if (ro)
            *ro = gq_ray_out{R.valid + off, R.p + off * f.p, R.nrm + off * f.n, R.t + off * f.t,
                             R.d + off,     R.id + off,      R.onb + off};
        if (so) *so = gq_sil_out{R.valid + off, R.p + off * f.p, R.d + off, R.id + off};
    }

    static void copy_down(Ring &R, int64_t off, int64_t m, cudaStream_t st) {
        const Fields &f = R.f;
        auto cp = [&](void *h, const void *d, size_t bytes) { cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, st); };
        cp(R.hvalid + off, R.valid + off, (size_t)m);
        if (f.p) cp(R.hp + off * f.p, R.p + off * f.p, (size_t)m * f.p * 4);
        if (f.n) cp(R.hn + off * f.n, R.nrm + off * f.n, (size_t)m * f.n * 4);
        if (f.t) cp(R.ht + off * f.t, R.t + off * f.t, (size_t)m * f.t * 4);
        cp(R.hd + off, R.d + off, (size_t)m * 4);
        cp(R.hid + off, R.id + off, (size_t)m * 4);
        if (f.onb) cp(R.honb + off, R.onb + off, (size_t)m);
    }

    bool launch() {
        bool any = false;
        for (Slot &S : slots) {
            if (S.busy) continue;
            bool have = false;
            for (int k = 0; k < 3; ++k)
                if (!(flags & GQ_SERVER_PER_REQUEST) && (k == GQ_KIND_SILHOUETTE) != S.sil_only) continue;
                else have |= !admitted[k].empty();
            if (!have) continue;
            S.reqs.clear();
            for (int k = 0; k < 3; ++k) S.off[k] = 0, S.m[k] = 0;
            if (flags & GQ_SERVER_PER_REQUEST) {
                int kb = -1;  // oldest admitted request of any kind
                for (int k = 0; k < 3; ++k)
                    if (!admitted[k].empty() &&
                        (kb < 0 || admitted[k].front()->t_admit < admitted[kb].front()->t_admit))
                        kb = k;
                Req *r = admitted[kb].front();
                admitted[kb].pop_front();
                S.off[kb] = r->phys;
                S.m[kb] = r->q.n;
                S.reqs.push_back(r);
            } else {
                for (int k = 0; k < 3; ++k) {
                    if ((k == GQ_KIND_SILHOUETTE) != S.sil_only) continue;
                    const int64_t cap = S.sil_only ? sil_step_queries : step_queries;
                    while (!admitted[k].empty()) {
                        Req *r = admitted[k].front();
                        if (S.m[k] == 0)
                            S.off[k] = r->phys;
                        else if (r->phys != S.off[k] + S.m[k] || S.m[k] + r->q.n > cap)
                            break;
                        S.m[k] += r->q.n;
                        S.reqs.push_back(r);
                        admitted[k].pop_front();
                    }
                }
            }
            const double t = now_s();
            S.step = next_step++;
            for (Req *r : S.reqs) r->t_launch = t, r->step = S.step;
            cudaStreamWaitEvent(S.st, copy_evt, 0);
            S.status = run_step(S);
            for (int k = 0; k < 3; ++k)
                if (S.m[k]) copy_down(ring[k], S.off[k], S.m[k], S.st);
            cudaEventRecord(S.done, S.st);
            S.busy = true;
            ++steps;
            any = true;
        }
        return any;
    }

    gq_status run_step(Slot &S) {
        const int D = dim;
        if (flags & GQ_SERVER_PER_REQUEST) {
            Req *r = S.reqs.front();
            const int k = r->q.kind;
            Ring &R = ring[k];
            const int64_t off = r->phys, n = r->q.n;
            const gq_scene *sc = scenes[(size_t)r->q.scene];
            gq_query_opts o{GQ_VARIANT_AUTO, 1, nullptr, S.scratch, (int64_t)S.scratch_bytes};
            const gq_vecs a{R.a + off * D, 1, D};
            if (k == GQ_KIND_CLOSEST_POINT) {
                gq_cp_out co;
                step_outputs(R, off, &co, nullptr, nullptr);
                return gq_closest_point(sc, a, n, &co, &o, S.st);
            }
            if (k == GQ_KIND_INTERSECT) {
                gq_ray_out ro;
                step_outputs(R, off, nullptr, &ro, nullptr);
                return gq_intersect(sc, a, gq_vecs{R.b + off * D, 1, D}, R.r + off, n, &ro, &o, S.st);
            }
            gq_sil_out so;
            step_outputs(R, off, nullptr, nullptr, &so);
            return gq_closest_silhouette(sc, a, R.r + off, n, &so, &o, S.st);
        }
        gqd::BatchKind kinds[3];
        gq_cp_out co{};
        gq_ray_out ro{};
        gq_sil_out so{};
        for (int k = 0; k < 3; ++k) {
            if (!S.m[k]) continue;
            Ring &R = ring[k];
            const int64_t off = S.off[k];
            kinds[k].a = gq_vecs{R.a + off * D, 1, D};
            if (R.f.b) kinds[k].b = gq_vecs{R.b + off * D, 1, D};
            kinds[k].r_max = R.f.r ? R.r + off : nullptr;
            kinds[k].scene = R.sid + off;
            kinds[k].n = S.m[k];
        }
        if (S.m[0]) step_outputs(ring[0], S.off[0], &co, nullptr, nullptr);
        if (S.m[1]) step_outputs(ring[1], S.off[1], nullptr, &ro, nullptr);
        if (S.m[2]) step_outputs(ring[2], S.off[2], nullptr, nullptr, &so);
        bool all_wide = true;
        for (const gq_scene *sc : scenes) all_wide &= sc->has_wide;
        cudaError_t e = gqd::batch_run(dev_scenes, (int)scenes.size(), D, kinds, co, ro, so,
                                       (flags & GQ_BATCH_RAY_EXACT) || !all_wide ? 0 : 1,
                                       gqd::cp_mode_of(flags), gqd::sil_mode_of(flags),
                                       S.sil_only ? sil_share : 1.f, S.scratch, step_queries, S.err, S.st);
        return e == cudaSuccess ? GQ_OK : fail_cuda(e, "server step");
    }

    // Copies one request's results from the pinned ring to its host buffers.
    void scatter(const Slot &S, const Req *r) {
        const int k = r->q.kind;
        const Ring &R = ring[k];
        const Fields &f = R.f;
        const int64_t off = S.off[k], m = S.m[k], n = r->q.n, i0 = r->phys - off;
        auto vec = [&](float *dst, const float *h, int comps) {
            if (!dst) return;
            for (int c = 0; c < comps; ++c)
                std::memcpy(dst + (int64_t)c * n, h + off * comps + (int64_t)c * m + i0, (size_t)n * 4);
        };
        auto one = [&](void *dst, const void *h, size_t es) {
            if (dst) std::memcpy(dst, static_cast<const char *>(h) + (size_t)(off + i0) * es, (size_t)n * es);
        };
        if (k == GQ_KIND_CLOSEST_POINT) {
            const gq_cp_out &o = r->q.cp_out;
            one(o.valid, R.hvalid, 1);
            vec(o.p, R.hp, f.p);
            vec(o.n, R.hn, f.n);
            vec(o.t, R.ht, f.t);
            one(o.d, R.hd, 4);
            one(o.prim_id, R.hid, 4);
        } else if (k == GQ_KIND_INTERSECT) {
            const gq_ray_out &o = r->q.ray_out;
            one(o.valid, R.hvalid, 1);
            vec(o.p, R.hp, f.p);
            vec(o.n, R.hn, f.n);
            vec(o.t, R.ht, f.t);
            one(o.d, R.hd, 4);
            one(o.prim_id, R.hid, 4);
            one(o.on_boundary, R.honb, 1);
        } else {
            const gq_sil_out &o = r->q.sil_out;
            one(o.valid, R.hvalid, 1);
            vec(o.p, R.hp, f.p);
            one(o.d, R.hd, 4);
            one(o.prim_id, R.hid, 4);
        }
    }

    bool complete() {
        bool any = false;
        for (Slot &S : slots) {
            if (!S.busy) continue;
            const cudaError_t q = cudaEventQuery(S.done);
            if (q == cudaErrorNotReady) continue;
            gq_status st = S.status;
            if (q != cudaSuccess) st = fail_cuda(q, "server step");
            if (st != GQ_OK) launch_error = st;
            const double t = now_s();
            for (Req *r : S.reqs) {
                if (st == GQ_OK) scatter(S, r);
                admitted_bytes -= r->q.n * ring[r->q.kind].f.bytes_per_query();
                ring[r->q.kind].release(r->alloc);
                finish(r, t, st);
            }
            S.reqs.clear();
            S.busy = false;
            any = true;
        }
        return any;
    }

    void run() {
        DeviceGuard g(device);
        while (!stop) {
            bool did = intake();
            did |= complete();
            did |= admit();
            did |= launch();
            if (did) continue;
            bool busy = false;
            for (const Slot &S : slots) busy |= S.busy;
            for (int k = 0; k < 3; ++k) busy |= !pending[k].empty() || !admitted[k].empty();
            if (busy) {
                std::this_thread::yield();
            } else {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait_for(lk, std::chrono::milliseconds(2), [&] { return stop.load() || !submitted.empty(); });
            }
        }
        // the steps in flight finish before their buffers can be freed
        for (Slot &S : slots)
            if (S.busy) cudaEventSynchronize(S.done);
    }

    gq_status submit(const gq_request &q, double t_submit) {
        if (q.kind < 0 || q.kind > 2) return fail(GQ_ERR_INVALID, "unknown query kind");
        if (q.scene < 0 || q.scene >= (int32_t)scenes.size()) return fail(GQ_ERR_INVALID, "scene index out of range");
        if (q.n < 1 || q.n > step_queries || q.n > ring[q.kind].cap)
            return fail(GQ_ERR_INVALID, "request size must be in [1, step_queries] and fit its ring (" +
                                            std::to_string(q.n) + " queries)");
        if (!q.a || (q.kind == GQ_KIND_INTERSECT && !q.b)) return fail(GQ_ERR_INVALID, "null query array");
        if (q.kind == GQ_KIND_SILHOUETTE && !scenes[(size_t)q.scene]->has_snch)
            return fail(GQ_ERR_UNSUPPORTED, "silhouette request on a scene built without SNCH");
        Req *r = new (std::nothrow) Req();
        if (!r) return fail(GQ_ERR_NOMEM, "host allocation");
        r->q = q;
        r->t_submit = t_submit;
        ++outstanding;
        {
            std::lock_guard<std::mutex> lk(mu);
            submitted.push_back(r);
        }
        cv.notify_one();
        return GQ_OK;
    }
};

extern "C" {

double gq_server_clock(void) { return now_s(); }

gq_status gq_server_create(gq_scene *const *scenes, int32_t n_scenes, const gq_server_opts *opts, gq_server **out) {
    if (!out) return fail(GQ_ERR_INVALID, "null output");
    *out = nullptr;
    if (!scenes || n_scenes <= 0) return fail(GQ_ERR_INVALID, "a server needs at least one scene");
    gq_server_opts o{};
    if (opts) o = *opts;
    std::unique_ptr<gq_server> s(new (std::nothrow) gq_server());
    if (!s) return fail(GQ_ERR_NOMEM, "host allocation");
    s->flags = o.flags;
    s->step_queries = o.step_queries > 0 ? o.step_queries : (1 << 19);
    const int inflight = o.max_inflight > 0 ? o.max_inflight : 3;
    s->sil_share = o.sil_share > 0.f ? o.sil_share : 1.5f;  // above 1: the slots may oversubscribe
    std::vector<gqd::DevScene> views((size_t)n_scenes);
    for (int32_t i = 0; i < n_scenes; ++i) {
        gq_scene *sc = scenes[i];
        if (!sc) return fail(GQ_ERR_INVALID, "null scene");
        if (sc->device < 0) return fail(GQ_ERR_UNSUPPORTED, "scene was built without a device copy");
        if (i == 0) {
            s->dim = sc->dim;
            s->device = sc->device;
        } else if (sc->dim != s->dim || sc->device != s->device) {
            return fail(GQ_ERR_INVALID, "server scenes must share dimension and device");
        }
        views[(size_t)i] = sc->dev;
        s->scenes.push_back(sc);
    }
    int64_t ring_bytes = 0;
    for (int k = 0; k < 3; ++k) {
        Ring &R = s->ring[k];
        R.f = fields_of(k, s->dim);
        R.cap = o.ring_queries[k] > 0 ? o.ring_queries[k] : (1 << 22);
        ring_bytes += R.cap * R.f.bytes_per_query();
    }
    s->ring_bytes = ring_bytes;
    if (o.budget_bytes > 0 && ring_bytes > o.budget_bytes)
        return fail(GQ_ERR_INVALID, "request rings (" + std::to_string(ring_bytes) + " bytes) exceed budget_bytes");
    DeviceGuard g(s->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scenes' device");
    cudaError_t e = s->dalloc(&s->dev_scenes, n_scenes);
    if (e == cudaSuccess)
        e = cudaMemcpy(s->dev_scenes, views.data(), views.size() * sizeof(gqd::DevScene), cudaMemcpyHostToDevice);
    for (int k = 0; k < 3 && e == cudaSuccess; ++k) e = s->make_ring(s->ring[k]);
    // closest-point / ray steps and the copies on the highest stream priority, silhouette
    // steps (long, persistent launches) on the lowest: when both wait for SMs, the short
    // kinds' blocks are scheduled first
    int prio_low = 0, prio_high = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&s->copy_st, cudaStreamNonBlocking, prio_high);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->copy_evt, cudaEventDisableTiming);
    const bool per_request = (s->flags & GQ_SERVER_PER_REQUEST) != 0;
    const int sil_slots = per_request ? 0 : (o.sil_slots > 0 ? o.sil_slots : 3);
    s->sil_share = std::min(1.f, s->sil_share / (float)std::max(sil_slots, 1));
    s->sil_step_queries = std::min<int64_t>(s->step_queries, o.sil_step_queries > 0 ? o.sil_step_queries : (1 << 15));
    s->slots.resize((size_t)(inflight + sil_slots));
    for (int i = 0; i < sil_slots; ++i) s->slots[(size_t)(inflight + i)].sil_only = true;
    for (Slot &S : s->slots) {
        if (e == cudaSuccess)
            e = cudaStreamCreateWithPriority(&S.st, cudaStreamNonBlocking, S.sil_only ? prio_low : prio_high);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S.done, cudaEventDisableTiming);
        S.scratch_bytes = (s->flags & GQ_SERVER_PER_REQUEST) ? (size_t)gq_query_scratch_bytes(s->step_queries)
                                                             : gqd::batch_scratch_bytes(s->step_queries);
        char *sp = nullptr;
        if (e == cudaSuccess) e = s->dalloc(&sp, (int64_t)S.scratch_bytes);
        S.scratch = sp;
        if (e == cudaSuccess) e = s->dalloc(&S.err, 64);
        if (e == cudaSuccess) e = cudaMemset(S.err, 0, 64 * sizeof(int32_t));
    }
    if (e != cudaSuccess) return fail(GQ_ERR_NOMEM, std::string("server allocation: ") + cudaGetErrorString(e));
    gq_server *raw = s.get();
    try {
        s->worker = std::thread([raw] { raw->run(); });
    } catch (...) {
        return fail(GQ_ERR_NOMEM, "cannot start the worker thread");
    }
    *out = s.release();
    return GQ_OK;
}

gq_status gq_server_free(gq_server *s) {
    delete s;
    return GQ_OK;
}

gq_status gq_server_submit(gq_server *s, const gq_request *q) {
    if (!s || !q) return fail(GQ_ERR_INVALID, "null argument");
    return s->submit(*q, now_s());
}

gq_status gq_server_poll(gq_server *s, gq_completion *out, int64_t cap, int64_t *count) {
    if (!s || !count || (cap > 0 && !out)) return fail(GQ_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    const int64_t k = std::min<int64_t>(std::max<int64_t>(cap, 0), (int64_t)s->completed.size());
    if (k > 0) {
        std::copy(s->completed.begin(), s->completed.begin() + k, out);
        s->completed.erase(s->completed.begin(), s->completed.begin() + k);
    }
    *count = k;
    return GQ_OK;
}

gq_status gq_server_wait_idle(gq_server *s, double timeout_s) {
    if (!s) return fail(GQ_ERR_INVALID, "null server");
    const double end = now_s() + timeout_s;
    while (s->outstanding.load() > 0) {
        if (now_s() > end) return fail(GQ_ERR_DEVICE, "timed out waiting for the server to drain");
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    return s->launch_error.load() ? fail(s->launch_error.load(), "a server step failed") : GQ_OK;
}

gq_status gq_server_get_stats(gq_server *s, gq_server_stats *st) {
    if (!s || !st) return fail(GQ_ERR_INVALID, "null argument");
    *st = gq_server_stats{};
    st->requests_done = s->requests_done.load();
    st->queries_done = s->queries_done.load();
    st->steps = s->steps.load();
    st->admitted_bytes_peak = s->admitted_peak.load();
    st->device_bytes = s->ring_bytes;
    if (s->outstanding.load() == 0) {  // error words are read only while nothing runs
        DeviceGuard g(s->device);
        if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the server's CUDA device");
        int32_t all = 0;
        for (Slot &S : s->slots) {
            int32_t v = 0;
            cudaError_t e = cudaMemcpy(&v, S.err, sizeof v, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) return fail_cuda(e, "server error read");
            all |= v << 8;
        }
        for (gq_scene *sc : s->scenes) {
            int32_t f = 0;
            gq_status r = gq_scene_device_error(sc, nullptr, &f);
            if (r != GQ_OK) return r;
            all |= f;
        }
        st->device_error = all;
    }
    return GQ_OK;
}

gq_status gq_server_run_trace(gq_server *s, const gq_request *reqs, const double *t_arrival, int64_t n,
                              gq_completion *out, double timeout_s) {
    if (!s || (n > 0 && (!reqs || !t_arrival || !out))) return fail(GQ_ERR_INVALID, "null argument");
    const double t0 = now_s();
    for (int64_t i = 0; i < n; ++i) {
        const double target = t0 + t_arrival[i];
        for (;;) {
            const double left = target - now_s();
            if (left <= 0) break;
            if (left > 3e-4)
                std::this_thread::sleep_for(std::chrono::microseconds(100));
            else
                std::this_thread::yield();
        }
        gq_request q = reqs[i];
        q.tag = (uint64_t)i;
        gq_status st = s->submit(q, target);
        if (st != GQ_OK) return st;
    }
    gq_status st = gq_server_wait_idle(s, timeout_s);
    std::vector<gq_completion> done;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        done.swap(s->completed);
    }
    for (const gq_completion &c : done) {
        if (c.tag < (uint64_t)n) {
            out[c.tag] = c;
            out[c.tag].tag = reqs[c.tag].tag;
        }
    }
    return st;
}

}  // extern "C"
