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
// Size classes.  Requests of at least large_queries queries are "large": they have
// rings, steps and stream slots of their own, on lower stream priorities than the
// small requests' (small closest-point / ray steps first, then small silhouette steps,
// large closest-point / ray steps, large silhouette steps).  A small request therefore
// never shares a step with a large one, and the block scheduler places its blocks
// ahead of the pending blocks of every large step.
//
// Step.  A step takes, for each kind it serves, the run of admitted requests of its
// class that are contiguous in the ring (at most step_queries queries) and answers
// them with one batch launch; closest-point and ray requests go to the general slots,
// silhouette requests to slots of their own whose launches hold part of the GPU only;
// inside the step a field with C components is stored component-major with stride m
// (the step's query count) from ring offset off * C, which is where the kernel writes
// it and what one device-to-host copy per field brings back.
//
// Host copies.  Staging a request's queries into the pinned ring and scattering its
// results into its arrays are plain memory copies of up to ~10 MB a request; they are
// split into chunks over a few helper threads, so that one large request does not hold
// the worker (and every other request's admission and completion) for a millisecond.
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

// Memory copies and 32-bit fills, run by the calling thread and `helpers` threads
// together on chunks of at most kChunk bytes; lists under kInline bytes run inline.
class CopyPool {
  public:
    struct Job {
        void *dst;
        const void *src;  // nullptr: fill bytes / 4 words with `word`
        size_t bytes;
        uint32_t word;
    };

    ~CopyPool() { stop(); }

    void start(int helpers) {
        for (int i = 0; i < helpers; ++i) th_.emplace_back([this] { loop(); });
    }

    void stop() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            quit_ = true;
        }
        cv_.notify_all();
        for (std::thread &t : th_) t.join();
        th_.clear();
    }

    // Returns when every job is done.
    void run(const std::vector<Job> &jobs) {
        size_t total = 0;
        for (const Job &j : jobs) total += j.bytes;
        if (th_.empty() || total < kInline) {
            for (const Job &j : jobs) exec(j);
            return;
        }
        {
            std::unique_lock<std::mutex> lk(mu_);
            idle_cv_.wait(lk, [&] { return active_ == 0; });  // a helper still leaving the previous list
            chunks_.clear();
            for (const Job &j : jobs)
                for (size_t o = 0; o < j.bytes; o += kChunk)
                    chunks_.push_back(Job{static_cast<char *>(j.dst) + o,
                                          j.src ? static_cast<const char *>(j.src) + o : nullptr,
                                          std::min(kChunk, j.bytes - o), j.word});
            next_.store(0, std::memory_order_relaxed);
            done_.store(0, std::memory_order_relaxed);
            ++gen_;
        }
        cv_.notify_all();
        work();
        const size_t n = chunks_.size();
        while (done_.load(std::memory_order_acquire) < n) std::this_thread::yield();
    }

  private:
    static constexpr size_t kChunk = 256 << 10, kInline = 512 << 10;  // kChunk: a multiple of 4 (fills)

    static void exec(const Job &j) {
        if (j.src) {
            std::memcpy(j.dst, j.src, j.bytes);
        } else {
            uint32_t *d = static_cast<uint32_t *>(j.dst);
            std::fill(d, d + j.bytes / 4, j.word);
        }
    }

    // chunks_ does not change while a thread is in here (run() waits for active_ == 0)
    void work() {
        const size_t n = chunks_.size();
        for (;;) {
            const size_t i = next_.fetch_add(1, std::memory_order_relaxed);
            if (i >= n) return;
            exec(chunks_[i]);
            done_.fetch_add(1, std::memory_order_release);
        }
    }

    void loop() {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return quit_ || gen_ != seen; });
                if (quit_) return;
                seen = gen_;
                ++active_;
            }
            work();
            {
                std::lock_guard<std::mutex> lk(mu_);
                --active_;
            }
            idle_cv_.notify_all();
        }
    }

    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_, idle_cv_;
    uint64_t gen_ = 0;
    int active_ = 0;
    bool quit_ = false;
    std::vector<Job> chunks_;
    std::atomic<size_t> next_{0}, done_{0};
};

constexpr int kSmall = 0, kLarge = 1;  // request size classes

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
    int cls = kSmall;  // size class: which of its kind's rings it is in
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
    int cls = kSmall;       // size class of the requests it takes
    int step = -1;
    gq_status status = GQ_OK;
    std::vector<Req *> reqs;
    int64_t off[3] = {0, 0, 0}, m[3] = {0, 0, 0};
};

}  // namespace

struct gq_server {
    int dim = 0, device = 0, flags = 0;
    int64_t step_queries = 0, ring_bytes = 0, sil_step_queries = 0;
    int64_t large_queries = 0;  // requests of at least this many queries are large (0: one class)
    float sil_share = 0.8f;     // per silhouette slot
    float large_share = 1.f;    // share of the GPU a large closest-point / ray step's persistent grid may hold
    std::vector<gq_scene *> scenes;
    gqd::DevScene *dev_scenes = nullptr;
    Ring ring[3][2];  // [kind][size class]
    std::vector<Slot> slots;
    cudaStream_t copy_st = nullptr;
    cudaEvent_t copy_evt = nullptr;
    std::vector<void *> dev_allocs, host_allocs;
    CopyPool pool;

    std::thread worker;
    std::mutex mu;  // guards `submitted` and `completed`
    std::condition_variable cv;
    std::deque<Req *> submitted;
    std::vector<gq_completion> completed;
    std::atomic<bool> stop{false};
    std::atomic<int64_t> outstanding{0};

    // worker-only state
    std::deque<Req *> pending[3][2], admitted[3][2];
    std::vector<CopyPool::Job> jobs;
    int next_step = 0;
    int64_t admitted_bytes = 0;
    std::atomic<int64_t> admitted_peak{0}, requests_done{0}, queries_done{0}, steps{0};
    std::atomic<int32_t> launch_error{0};

    ~gq_server() {
        stop = true;
        cv.notify_all();
        if (worker.joinable()) worker.join();
        pool.stop();
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
        for (int k = 0; k < 3; ++k)
            for (int c = 0; c < 2; ++c) {
                for (Req *r : pending[k][c]) delete r;
                for (Req *r : admitted[k][c]) delete r;
            }
        for (Slot &s : slots)
            for (Req *r : s.reqs) delete r;
        for (Req *r : submitted) delete r;
    }

    int class_of(int64_t n) const { return large_queries > 0 && n >= large_queries ? kLarge : kSmall; }

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
        for (Req *r : submitted) pending[r->q.kind][r->cls].push_back(r);
        submitted.clear();
        return true;
    }

    // Admits pending requests while their ring has room, stages their queries in the
    // pinned mirror and copies them up (one copy per field and contiguous run).
    bool admit() {
        const int D = dim;
        struct Run {
            Ring *R;
            int64_t lo, hi;
        };
        std::vector<Run> runs;
        jobs.clear();
        for (int k = 0; k < 3; ++k)
            for (int c = 0; c < 2; ++c) {
                Ring &R = ring[k][c];
                while (!pending[k][c].empty()) {
                    Req *r = pending[k][c].front();
                    int64_t phys;
                    size_t seq;
                    if (!R.alloc(r->q.n, &phys, &seq)) break;
                    pending[k][c].pop_front();
                    r->phys = phys;
                    r->alloc = seq;
                    r->t_admit = now_s();
                    const int64_t n = r->q.n;
                    jobs.push_back({R.ha + phys * D, r->q.a, (size_t)n * D * 4, 0});
                    if (R.f.b) jobs.push_back({R.hb + phys * D, r->q.b, (size_t)n * D * 4, 0});
                    if (R.f.r) jobs.push_back({R.hr + phys, r->q.r_max, (size_t)n * 4, 0x7f800000u});  // NULL: +inf
                    jobs.push_back({R.hsid + phys, nullptr, (size_t)n * 4, (uint32_t)r->q.scene});
                    if (!runs.empty() && runs.back().R == &R && runs.back().hi == phys)
                        runs.back().hi += n;
                    else
                        runs.push_back({&R, phys, phys + n});
                    admitted_bytes += n * R.f.bytes_per_query();
                    if (admitted_bytes > admitted_peak) admitted_peak = admitted_bytes;
                    admitted[k][c].push_back(r);
                }
            }
        if (runs.empty()) return false;
        pool.run(jobs);
        for (const Run &u : runs) {
            Ring &R = *u.R;
            const int64_t lo = u.lo, cnt = u.hi - u.lo;
            cudaMemcpyAsync(R.a + lo * D, R.ha + lo * D, (size_t)cnt * D * 4, cudaMemcpyHostToDevice, copy_st);
            if (R.f.b)
                cudaMemcpyAsync(R.b + lo * D, R.hb + lo * D, (size_t)cnt * D * 4, cudaMemcpyHostToDevice, copy_st);
            if (R.f.r) cudaMemcpyAsync(R.r + lo, R.hr + lo, (size_t)cnt * 4, cudaMemcpyHostToDevice, copy_st);
            cudaMemcpyAsync(R.sid + lo, R.hsid + lo, (size_t)cnt * 4, cudaMemcpyHostToDevice, copy_st);
        }
        cudaEventRecord(copy_evt, copy_st);
        return true;
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
        const bool per_req = (flags & GQ_SERVER_PER_REQUEST) != 0;
        for (Slot &S : slots) {
            if (S.busy) continue;
            auto serves = [&](int k) { return per_req || (k == GQ_KIND_SILHOUETTE) == S.sil_only; };
            bool have = false;
            for (int k = 0; k < 3; ++k) have |= serves(k) && !admitted[k][S.cls].empty();
            if (!have) continue;
            S.reqs.clear();
            for (int k = 0; k < 3; ++k) S.off[k] = 0, S.m[k] = 0;
            if (per_req) {
                int kb = -1;  // oldest admitted request of any kind
                for (int k = 0; k < 3; ++k)
                    if (!admitted[k][S.cls].empty() &&
                        (kb < 0 || admitted[k][S.cls].front()->t_admit < admitted[kb][S.cls].front()->t_admit))
                        kb = k;
                Req *r = admitted[kb][S.cls].front();
                admitted[kb][S.cls].pop_front();
                S.off[kb] = r->phys;
                S.m[kb] = r->q.n;
                S.reqs.push_back(r);
            } else {
                for (int k = 0; k < 3; ++k) {
                    if (!serves(k)) continue;
                    const int64_t cap = S.sil_only && S.cls == kSmall ? sil_step_queries : step_queries;
                    std::deque<Req *> &q = admitted[k][S.cls];
                    while (!q.empty()) {
                        Req *r = q.front();
                        if (S.m[k] == 0)
                            S.off[k] = r->phys;
                        else if (r->phys != S.off[k] + S.m[k] || S.m[k] + r->q.n > cap)
                            break;
                        S.m[k] += r->q.n;
                        S.reqs.push_back(r);
                        q.pop_front();
                    }
                }
            }
            const double t = now_s();
            S.step = next_step++;
            for (Req *r : S.reqs) r->t_launch = t, r->step = S.step;
            cudaStreamWaitEvent(S.st, copy_evt, 0);
            S.status = run_step(S);
            for (int k = 0; k < 3; ++k)
                if (S.m[k]) copy_down(ring[k][S.cls], S.off[k], S.m[k], S.st);
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
            Ring &R = ring[k][S.cls];
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
            Ring &R = ring[k][S.cls];
            const int64_t off = S.off[k];
            kinds[k].a = gq_vecs{R.a + off * D, 1, D};
            if (R.f.b) kinds[k].b = gq_vecs{R.b + off * D, 1, D};
            kinds[k].r_max = R.f.r ? R.r + off : nullptr;
            kinds[k].scene = R.sid + off;
            kinds[k].n = S.m[k];
        }
        if (S.m[0]) step_outputs(ring[0][S.cls], S.off[0], &co, nullptr, nullptr);
        if (S.m[1]) step_outputs(ring[1][S.cls], S.off[1], nullptr, &ro, nullptr);
        if (S.m[2]) step_outputs(ring[2][S.cls], S.off[2], nullptr, nullptr, &so);
        bool all_wide = true;
        for (const gq_scene *sc : scenes) all_wide &= sc->has_wide;
        const float share = S.sil_only ? sil_share : S.cls == kLarge ? large_share : 1.f;
        // One-warp blocks: the silhouette steps' one-warp blocks end all the time, and a
        // block of this step fits in the room any one of them leaves (a 128-thread block
        // would wait for four to end on the same SM while lower-priority one-warp blocks
        // take each single slot).  Small steps are not sorted: the keys and the radix
        // sort are launches of large blocks that would wait the same way, and a small
        // step's requests are contiguous runs of one scene each already.
        cudaError_t e = gqd::batch_run(dev_scenes, (int)scenes.size(), D, kinds, co, ro, so,
                                       (flags & GQ_BATCH_RAY_EXACT) || !all_wide ? 0 : 1,
                                       gqd::cp_mode_of(flags), gqd::sil_mode_of(flags), share, 32,
                                       S.cls == kLarge || !large_queries, S.scratch, step_queries, S.err, S.st);
        return e == cudaSuccess ? GQ_OK : fail_cuda(e, "server step");
    }

    // Queues the copies of one request's results from the pinned ring to its host buffers.
    void scatter(const Slot &S, const Req *r) {
        const int k = r->q.kind;
        const Ring &R = ring[k][r->cls];
        const Fields &f = R.f;
        const int64_t off = S.off[k], m = S.m[k], n = r->q.n, i0 = r->phys - off;
        auto vec = [&](float *dst, const float *h, int comps) {
            if (!dst) return;
            for (int c = 0; c < comps; ++c)
                jobs.push_back({dst + (int64_t)c * n, h + off * comps + (int64_t)c * m + i0, (size_t)n * 4, 0});
        };
        auto one = [&](void *dst, const void *h, size_t es) {
            if (dst) jobs.push_back({dst, static_cast<const char *>(h) + (size_t)(off + i0) * es, (size_t)n * es, 0});
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
            if (st == GQ_OK) {
                jobs.clear();
                for (Req *r : S.reqs) scatter(S, r);
                pool.run(jobs);
            }
            const double t = now_s();
            for (Req *r : S.reqs) {
                admitted_bytes -= r->q.n * ring[r->q.kind][r->cls].f.bytes_per_query();
                ring[r->q.kind][r->cls].release(r->alloc);
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
            for (int k = 0; k < 3; ++k)
                for (int c = 0; c < 2; ++c) busy |= !pending[k][c].empty() || !admitted[k][c].empty();
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
        const int cls = q.n >= 1 ? class_of(q.n) : kSmall;
        if (q.n < 1 || q.n > step_queries || q.n > ring[q.kind][cls].cap)
            return fail(GQ_ERR_INVALID, "request size must be in [1, step_queries] and fit its ring (" +
                                            std::to_string(q.n) + " queries)");
        if (!q.a || (q.kind == GQ_KIND_INTERSECT && !q.b)) return fail(GQ_ERR_INVALID, "null query array");
        if (q.kind == GQ_KIND_SILHOUETTE && !scenes[(size_t)q.scene]->has_snch)
            return fail(GQ_ERR_UNSUPPORTED, "silhouette request on a scene built without SNCH");
        Req *r = new (std::nothrow) Req();
        if (!r) return fail(GQ_ERR_NOMEM, "host allocation");
        r->q = q;
        r->cls = cls;
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
    const bool per_request = (s->flags & GQ_SERVER_PER_REQUEST) != 0;
    // the large class: on by default; off in the plain per-request mode, when no request
    // can reach it, or when half of a kind's ring could not hold a largest request (the
    // split would refuse requests one ring admits)
    const int64_t lq = o.large_queries != 0 ? o.large_queries : (1 << 15);
    bool halves_fit = true;
    for (int k = 0; k < 3; ++k)
        halves_fit &= (o.ring_queries[k] > 0 ? o.ring_queries[k] : (1 << 22)) / 2 >= s->step_queries;
    s->large_queries = (!per_request && lq > 0 && lq <= s->step_queries && halves_fit) ? lq : 0;
    s->large_share = o.large_share > 0.f ? std::min(1.f, o.large_share) : 1.f;
    int64_t ring_bytes = 0;
    for (int k = 0; k < 3; ++k) {
        const int64_t cap = o.ring_queries[k] > 0 ? o.ring_queries[k] : (1 << 22);
        const int64_t large = s->large_queries ? cap / 2 : 0;
        for (int c = 0; c < 2; ++c) {
            Ring &R = s->ring[k][c];
            R.f = fields_of(k, s->dim);
            R.cap = c == kLarge ? large : cap - large;
            ring_bytes += R.cap * R.f.bytes_per_query();
        }
    }
    s->ring_bytes = ring_bytes;
    if (o.budget_bytes > 0 && ring_bytes > o.budget_bytes)
        return fail(GQ_ERR_INVALID, "request rings (" + std::to_string(ring_bytes) + " bytes) exceed budget_bytes");
    DeviceGuard g(s->device);
    if (!g.ok) return fail(GQ_ERR_CUDA, "cannot select the scenes' device");
    cudaError_t e = s->dalloc(&s->dev_scenes, n_scenes);
    if (e == cudaSuccess)
        e = cudaMemcpy(s->dev_scenes, views.data(), views.size() * sizeof(gqd::DevScene), cudaMemcpyHostToDevice);
    for (int k = 0; k < 3 && e == cudaSuccess; ++k)
        for (int c = 0; c < 2 && e == cudaSuccess; ++c) e = s->make_ring(s->ring[k][c]);
    // Stream priorities, highest first: the copies and small closest-point / ray steps,
    // small silhouette steps, large closest-point / ray steps, large silhouette steps
    // (clamped to the device's range).  When several launches wait for SMs, the blocks
    // of the shorter requests are scheduled first.
    int prio_low = 0, prio_high = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    auto level = [&](int i) { return std::min(prio_low, prio_high + i); };  // prio_high <= prio_low
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&s->copy_st, cudaStreamNonBlocking, prio_high);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->copy_evt, cudaEventDisableTiming);
    const int sil_slots = per_request ? 0 : (o.sil_slots > 0 ? o.sil_slots : 3);
    const int large_slots = s->large_queries ? (o.large_slots > 0 ? o.large_slots : 2) : 0;
    s->sil_share = std::min(1.f, s->sil_share / (float)std::max(sil_slots, 1));
    s->sil_step_queries = std::min<int64_t>(s->step_queries, o.sil_step_queries > 0 ? o.sil_step_queries : (1 << 15));
    struct Group {
        int count;
        bool sil;
        int cls, prio;
    };
    const Group groups[4] = {{inflight, false, kSmall, level(0)},
                             {sil_slots, true, kSmall, level(1)},
                             {large_slots, false, kLarge, level(2)},
                             {large_slots, true, kLarge, prio_low}};
    for (const Group &gr : groups)
        for (int i = 0; i < gr.count && e == cudaSuccess; ++i) {
            s->slots.emplace_back();
            Slot &S = s->slots.back();
            S.sil_only = gr.sil;
            S.cls = gr.cls;
            e = cudaStreamCreateWithPriority(&S.st, cudaStreamNonBlocking, gr.prio);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S.done, cudaEventDisableTiming);
            S.scratch_bytes = per_request ? (size_t)gq_query_scratch_bytes(s->step_queries)
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
        const int hw = (int)std::thread::hardware_concurrency();
        s->pool.start(o.copy_threads > 0 ? o.copy_threads - 1 : std::max(0, std::min(7, hw / 2 - 1)));
        s->worker = std::thread([raw] { raw->run(); });
    } catch (...) {
        return fail(GQ_ERR_NOMEM, "cannot start the worker or copy threads");
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
    st->large_queries = s->large_queries;
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
