// Request loop: continuous batching of single-frame requests across plans.
//
// Requests are admitted while in-flight slots remain (a submit waits, bounded,
// for a slot). Worker threads take the oldest queued request whose plan is
// built, coalesce the queued requests with the same plan key, dtype and
// flags behind it (up to max_coalesce per plan) into one launch, and publish
// results per request; requests of other built plans with the same dtype and
// flags join the batch (up to eight plans, and at most a quarter of the queue,
// so that a backlog spreads over the workers instead of piling into one
// batch), which runs as one work-queue gather
// (dg_multi: row-warp CTAs claiming (plan, row item, frame block) tiles,
// replayed as a CUDA graph, no partial sums). Four workers run batches
// concurrently on their own streams, so one batch's copies overlap another's
// gather; their staging grows stream-ordered and is kept. max_coalesce 1
// serves one request per launch on the plan's own lane mapping, tuned for
// one frame (the plain path). Plans live in an HBM cache bounded by bytes
// and are managed by two builder threads: a request for a plan that is not
// built asks a builder and stays queued while the workers serve other plans;
// the builder builds the plan on the device (for the plain path also tunes
// it once per key and allocates its partial sums), admits it by evicting
// least-recently-used plans that no worker is using, and destroys evicted
// and stale plans, so no worker ever waits for a build or a free. A submit
// copies its frame into a pooled pinned buffer outside the server lock (or
// borrows the caller's); the worker copies the pinned buffers straight to the
// device, and each request's results straight back into a pooled pinned
// buffer that dg_server_poll copies out and returns. Re-registering a key (a
// changed PONI) gives it a new generation: the next request rebuilds the
// plan, and the stale plan is destroyed once no worker uses it. A build that
// fails fails the requests of that generation. Each request's result is
// identical alone and in any mix: the gather's arithmetic depends only on the
// plan, never on which frames or plans share a launch.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <memory>
#include <thread>
#include <unordered_map>

#include "dg_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct PlanSpec {
    dg_geometry geometry{};
    dg_method method{};
    std::vector<uint8_t> mask;
    int32_t dim1 = 0, dim2 = 0, n_radial = 0, n_azimuthal = 0;
    bool has_az_range = false;
    double az_range[2] = {0, 0};
    uint64_t generation = 0;
    int64_t n_bins() const { return n_azimuthal ? int64_t(n_radial) * n_azimuthal : n_radial; }
};

// Pinned host buffers by byte size, reused across requests.
struct PinnedPool {
    std::mutex mu;
    std::unordered_map<size_t, std::vector<void *>> free;
    std::unordered_map<size_t, size_t> made;  // buffers allocated, by size
    void *get(size_t bytes) {
        {
            std::lock_guard<std::mutex> lock(mu);
            auto &v = free[bytes];
            if (!v.empty()) {
                void *p = v.back();
                v.pop_back();
                return p;
            }
            made[bytes]++;
        }
        void *p = nullptr;
        if (cudaMallocHost(&p, bytes) != cudaSuccess) {
            (void)cudaGetLastError();
            std::lock_guard<std::mutex> lock(mu);
            made[bytes]--;
            return nullptr;
        }
        return p;
    }
    // Allocates buffers of `bytes` until `count` of that size exist, the new
    // ones free. A page-locked allocation is slow and keeps copies on other
    // streams from overlapping it, so it belongs before a stream's requests
    // rather than on a worker's path.
    void reserve(size_t bytes, size_t count) {
        for (;;) {
            {
                std::lock_guard<std::mutex> lock(mu);
                if (made[bytes] >= count) return;
                made[bytes]++;
            }
            void *p = nullptr;
            if (cudaMallocHost(&p, bytes) != cudaSuccess) {
                (void)cudaGetLastError();
                std::lock_guard<std::mutex> lock(mu);
                made[bytes]--;
                return;
            }
            put(bytes, p);
        }
    }
    void put(size_t bytes, void *p) {
        if (!p) return;
        std::lock_guard<std::mutex> lock(mu);
        free[bytes].push_back(p);
    }
    ~PinnedPool() {
        for (auto &kv : free)
            for (void *p : kv.second) cudaFreeHost(p);
    }
};

struct Request {
    uint64_t ticket = 0, key = 0;
    int32_t dtype = 0;
    uint32_t flags = 0;
    void *frame = nullptr;  // pinned, frame_bytes long (the caller's with DG_SUBMIT_BORROW)
    size_t frame_bytes = 0;
    bool borrowed = false;
    Clock::time_point submitted;
    double latency_us = 0;
    // Results in a pooled page-locked buffer: nout arrays of n_bins doubles
    // (intensity, then sigma, then spread as requested), copied there from
    // the device and out of it by dg_server_poll.
    double *res = nullptr;
    size_t res_bytes = 0;
    int64_t n_bins = 0;
    dg_status status = DG_OK;
    std::string error;
    bool done = false;
};

struct CacheEntry {
    dg_plan *plan = nullptr;
    int64_t bytes = 0;
    int users = 0;
    uint64_t last_use = 0;
    uint64_t generation = 0;
};

size_t px_size(int32_t dtype) {
    return dtype == DG_U16 ? 2 : dtype == DG_F64 ? 8 : 4;
}

std::string last_error_text() {
    char buf[512];
    dg_last_error(buf, sizeof buf);
    return buf;
}

}  // namespace

struct dg_server {
    dg_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_slot, cv_build;
    std::unordered_map<uint64_t, PlanSpec> specs;
    std::unordered_map<uint64_t, CacheEntry> cache;
    std::deque<Request *> queue;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> requests;
    int64_t inflight = 0;
    int64_t cache_bytes = 0;
    uint64_t next_ticket = 1, use_clock = 0;
    dg_server_stats stats{};
    bool stop = false;
    std::vector<std::thread> workers;
    std::vector<std::thread> builders;
    PinnedPool pinned;
    std::vector<CacheEntry> retired;    // stale plans still in use by a worker
    std::vector<dg_plan *> to_destroy;  // plans no worker uses, for the builder
    uint64_t next_generation = 1;
    // Plans to build, once per key and generation: the first request's dtype
    // and flags tune the new plan.
    std::deque<uint64_t> build_queue;
    std::unordered_map<uint64_t, std::pair<int32_t, uint32_t>> build_pending;
    struct BuildFailure {
        uint64_t generation;
        dg_status status;
        std::string message;
    };
    std::unordered_map<uint64_t, BuildFailure> failed;
    std::unordered_map<uint64_t, int32_t> tuned;  // key -> lane mapping its last plan used

    // A new plan's lane mapping for the plain path's one-request launches,
    // tuned on a zero frame of the request's type (timing does not depend on
    // the values); left at the default if anything fails. Builder thread.
    void tune(dg_plan *plan, int32_t dtype, uint32_t flags) {
        const int64_t nf = 1;
        const size_t bytes = size_t(plan->dim1) * plan->dim2 * px_size(dtype) * size_t(nf);
        void *d = nullptr;
        if (cudaMallocAsync(&d, bytes, plan->stream) != cudaSuccess) {
            (void)cudaGetLastError();
            return;
        }
        cudaMemsetAsync(d, 0, bytes, plan->stream);
        if (dg_plan_autotune(plan, d, dtype, nf, flags & (DG_ERRORS | DG_AZIMUTHAL_STD), nullptr,
                             nullptr, nullptr, 0) != DG_OK)
            (void)last_error_text();
        cudaFreeAsync(d, plan->stream);
        cudaStreamSynchronize(plan->stream);
    }

    // Queues a build of `key` unless one is queued or running (lock held).
    void request_build_locked(uint64_t key, int32_t dtype, uint32_t flags) {
        if (build_pending.count(key)) return;
        build_pending[key] = {dtype, flags};
        build_queue.push_back(key);
        cv_build.notify_one();
    }

    // Moves a stale cache entry out of the cache (lock held): to the builder
    // for destruction now if idle, else when its last user releases it.
    void retire_locked(std::unordered_map<uint64_t, CacheEntry>::iterator it) {
        cache_bytes -= it->second.bytes;
        if (it->second.users == 0) {
            to_destroy.push_back(it->second.plan);
            cv_build.notify_one();
        } else {
            retired.push_back(it->second);
        }
        cache.erase(it);
    }

    void release(uint64_t key, dg_plan *plan) {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end() && it->second.plan == plan) {
            if (it->second.users > 0) it->second.users--;
            return;
        }
        for (size_t i = 0; i < retired.size(); ++i)
            if (retired[i].plan == plan) {
                if (--retired[i].users == 0) {
                    to_destroy.push_back(plan);
                    retired.erase(retired.begin() + long(i));
                    cv_build.notify_one();
                }
                return;
            }
    }

    // Builds, tunes and admits plans, and destroys the ones the cache let go:
    // every device allocation and free of a plan happens on this thread, so
    // the workers' streams never wait for a build or an eviction.
    void builder_main() {
        cudaSetDevice(cfg.device);
        for (;;) {
            std::vector<dg_plan *> dead;
            uint64_t key = 0;
            bool have = false;
            PlanSpec spec;
            std::pair<int32_t, uint32_t> hint{DG_U32, 0};
            {
                std::unique_lock<std::mutex> lock(mu);
                cv_build.wait(lock, [&] {
                    return stop || !build_queue.empty() || !to_destroy.empty();
                });
                dead.swap(to_destroy);
                if (!build_queue.empty() && !stop) {
                    key = build_queue.front();
                    build_queue.pop_front();
                    spec = specs.at(key);
                    hint = build_pending.at(key);
                    have = true;
                }
                if (!have && stop && dead.empty()) break;
            }
            for (dg_plan *p : dead) dg_plan_destroy(p);
            if (!have) continue;
            const auto t_build = Clock::now();
            dg_plan *plan = nullptr;
            dg_status st = dg_plan_create(&spec.geometry, &spec.method,
                                          spec.mask.empty() ? nullptr : spec.mask.data(),
                                          spec.dim1, spec.dim2, spec.n_radial, spec.n_azimuthal,
                                          spec.has_az_range ? spec.az_range : nullptr, &plan);
            if (st != DG_OK) {
                const std::string msg = last_error_text();
                {
                    std::lock_guard<std::mutex> lock(mu);
                    failed[key] = {spec.generation, st, msg};
                    build_pending.erase(key);
                }
                cv_work.notify_all();
                continue;
            }
            // The plain path launches each request on the plan's own lane
            // mapping: a rebuilt key (new PONI, same shape and bins) keeps the
            // mapping its previous plan was tuned to, a new key is tuned once,
            // and partial sums (if the mapping uses any) are allocated now
            // rather than by a worker's first launch. The coalescing path's
            // work-queue gather (row warps) needs neither.
            if (cfg.max_coalesce <= 1) {
                int32_t known = -1;
                {
                    std::lock_guard<std::mutex> lock(mu);
                    auto t = tuned.find(key);
                    if (t != tuned.end()) known = t->second;
                }
                if (known < 0 || dg_plan_variant(plan, known, nullptr, nullptr) != DG_OK) {
                    tune(plan, hint.first, hint.second);
                    int32_t v = 0;
                    dg_plan_variant(plan, -1, &v, nullptr);
                    std::lock_guard<std::mutex> lock(mu);
                    tuned[key] = v;
                }
                std::lock_guard<std::mutex> lock(plan->mu);
                cudaSetDevice(plan->device);
                try {
                    dg::reserve_partials(plan->gather, 1, hint.second, hint.first);
                } catch (const dg::Error &) {
                }
            }
            // Result buffers for the plan's requests, page-locked now: as many
            // as the workers' batches hold at once, at most 1 GiB of them (a
            // rebuilt key with the same bins finds its buffers made already).
            {
                const int nout = 1 + ((hint.second & DG_ERRORS) ? 1 : 0) +
                                 ((hint.second & DG_AZIMUTHAL_STD) ? 1 : 0);
                const size_t bytes = size_t(nout) * size_t(spec.n_bins()) * 8;
                const size_t want = size_t(kWorkers) * size_t(std::max(cfg.max_coalesce, 1)) + 16;
                pinned.reserve(bytes, std::min(want, std::max<size_t>(1, (size_t(1) << 30) / bytes)));
            }
            dg_plan_info info{};
            dg_plan_query(plan, &info);
            std::vector<dg_plan *> evicted;
            {
                std::lock_guard<std::mutex> lock(mu);
                build_pending.erase(key);
                stats.build_us += int64_t(
                    std::chrono::duration<double, std::micro>(Clock::now() - t_build).count());
                if (specs.at(key).generation != spec.generation) {
                    evicted.push_back(plan);  // re-registered while building
                } else {
                    auto old = cache.find(key);
                    if (old != cache.end()) retire_locked(old);
                    stats.plan_builds++;
                    // Admission by memory: evict idle plans, oldest first.
                    while (cache_bytes + info.device_bytes > cfg.cache_bytes) {
                        uint64_t victim = 0, oldest = UINT64_MAX;
                        for (auto &kv : cache)
                            if (kv.second.users == 0 && kv.second.last_use < oldest) {
                                oldest = kv.second.last_use;
                                victim = kv.first;
                            }
                        if (oldest == UINT64_MAX) break;  // everything busy: over budget briefly
                        cache_bytes -= cache[victim].bytes;
                        evicted.push_back(cache[victim].plan);
                        cache.erase(victim);
                        stats.plan_evictions++;
                    }
                    CacheEntry e;
                    e.plan = plan;
                    e.bytes = info.device_bytes;
                    e.last_use = ++use_clock;
                    e.generation = spec.generation;
                    cache[key] = e;
                    cache_bytes += e.bytes;
                }
            }
            cv_work.notify_all();
            for (dg_plan *p : evicted) dg_plan_destroy(p);
        }
    }

    // Finishes a request (lock held; notify after).
    void finish_locked(Request *r, dg_status st, const std::string &err) {
        r->status = st;
        r->error = err;
        r->done = true;
        r->latency_us = std::chrono::duration<double, std::micro>(Clock::now() - r->submitted).count();
        if (st == DG_OK) stats.completed++;
        else stats.failed++;
        if (!r->borrowed) pinned.put(r->frame_bytes, r->frame);
        r->frame = nullptr;
        if (st != DG_OK && r->res) {
            pinned.put(r->res_bytes, r->res);
            r->res = nullptr;
        }
        inflight--;
    }

    // One batch of a worker: up to max_coalesce queued requests of each of up
    // to kPlansPerLaunch built plans, all of one dtype and one set of flags.
    struct Group {
        uint64_t key = 0;
        dg_plan *plan = nullptr;
        std::vector<Request *> reqs;
        size_t in_off = 0, out_off = 0;
    };
    static constexpr int kPlansPerLaunch = 8;
    static constexpr int kWorkers = 4;

    // The cached plan of `key` if it is built for the current generation,
    // with a user reference taken (lock held).
    dg_plan *take_ready_locked(uint64_t key) {
        auto c = cache.find(key);
        if (c == cache.end() || c->second.generation != specs.at(key).generation) return nullptr;
        c->second.users++;
        c->second.last_use = ++use_clock;
        stats.plan_hits++;
        return c->second.plan;
    }

    void worker_main() {
        cudaSetDevice(cfg.device);
        cudaStream_t stream = nullptr;
        cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
        // Coalescing batches run through the work-queue gather: all their
        // plans in one graph launch, every plan summed with the same lane
        // mapping, so a request's result does not depend on its company.
        // max_coalesce 1 is the plain path: one request per launch on the
        // plan's own tuned mapping.
        const bool plain = cfg.max_coalesce <= 1;
        dg_multi *multi = nullptr;
        if (!plain && dg_multi_create(cfg.device, kPlansPerLaunch, &multi) != DG_OK) multi = nullptr;
        unsigned char *d_in = nullptr;
        double *d_out = nullptr;
        size_t in_cap = 0, out_cap = 0;
        for (;;) {
            std::vector<Group> groups;
            bool failed_some = false;
            {
                std::unique_lock<std::mutex> lock(mu);
                cv_work.wait_for(lock, std::chrono::microseconds(std::max(cfg.poll_us, 50)),
                                 [&] { return stop || !queue.empty(); });
                if (stop && queue.empty()) break;
                // The oldest request whose plan is built heads the batch;
                // requests of plans not built yet ask the builder and wait in
                // the queue; requests whose build failed fail.
                auto it = queue.begin();
                while (it != queue.end()) {
                    Request *r = *it;
                    if (dg_plan *p = take_ready_locked(r->key)) {
                        Group g;
                        g.key = r->key;
                        g.plan = p;
                        g.reqs.push_back(r);
                        groups.push_back(std::move(g));
                        it = queue.erase(it);
                        break;
                    }
                    auto f = failed.find(r->key);
                    if (f != failed.end() && f->second.generation == specs.at(r->key).generation) {
                        finish_locked(r, f->second.status, f->second.message);
                        failed_some = true;
                        it = queue.erase(it);
                        continue;
                    }
                    request_build_locked(r->key, r->dtype, r->flags);
                    ++it;
                }
                if (!groups.empty()) {
                    // the requests behind it: its plan's, then other built
                    // plans', at most a share of the queue per worker, so
                    // the other workers' batches overlap this one's copies
                    // and gather rather than wait for the next backlog
                    const Request *head = groups.front().reqs.front();
                    const size_t share = (queue.size() + 1 + kWorkers - 1) / kWorkers;
                    size_t taken = 1;
                    for (it = queue.begin(); it != queue.end() && taken < share;) {
                        Request *r = *it;
                        if (r->dtype != head->dtype || r->flags != head->flags) {
                            ++it;
                            continue;
                        }
                        Group *g = nullptr;
                        for (auto &x : groups)
                            if (x.key == r->key) g = &x;
                        if (!g && !plain && int(groups.size()) < kPlansPerLaunch) {
                            if (dg_plan *p = take_ready_locked(r->key)) {
                                groups.emplace_back();
                                g = &groups.back();
                                g->key = r->key;
                                g->plan = p;
                            }
                        }
                        if (g && int(g->reqs.size()) < cfg.max_coalesce) {
                            g->reqs.push_back(r);
                            it = queue.erase(it);
                            ++taken;
                        } else {
                            ++it;
                        }
                    }
                }
            }
            if (failed_some) {
                cv_done.notify_all();
                cv_slot.notify_all();
            }
            if (groups.empty()) continue;
            const Request *head = groups.front().reqs.front();
            const int nout = 1 + ((head->flags & DG_ERRORS) ? 1 : 0) +
                             ((head->flags & DG_AZIMUTHAL_STD) ? 1 : 0);
            size_t in_need = 0, out_need = 0, n_frames = 0;
            for (auto &g : groups) {
                g.in_off = in_need;
                g.out_off = out_need;
                in_need += g.reqs.size() * g.reqs.front()->frame_bytes;
                out_need += g.reqs.size() * size_t(g.plan->n_bins) * nout;
                n_frames += g.reqs.size();
            }
            std::string err;
            dg_status st = DG_OK;
            // Staging grows by doubling, stream-ordered on this worker's own
            // stream (no device-wide synchronisation), and is kept.
            if (in_cap < in_need) {
                if (d_in) cudaFreeAsync(d_in, stream);
                in_cap = std::max(in_need, 2 * in_cap);
                if (cudaMallocAsync(reinterpret_cast<void **>(&d_in), in_cap, stream) != cudaSuccess) {
                    (void)cudaGetLastError();
                    d_in = nullptr;
                    in_cap = 0;
                }
            }
            if (out_cap < out_need) {
                if (d_out) cudaFreeAsync(d_out, stream);
                out_cap = std::max(out_need, 2 * out_cap);
                if (cudaMallocAsync(reinterpret_cast<void **>(&d_out), out_cap * 8, stream) !=
                    cudaSuccess) {
                    (void)cudaGetLastError();
                    d_out = nullptr;
                    out_cap = 0;
                }
            }
            // each request's results go from the device straight to its own
            // pooled page-locked buffer
            bool res_ok = true;
            for (auto &g : groups)
                for (Request *r : g.reqs) {
                    r->n_bins = g.plan->n_bins;
                    r->res_bytes = size_t(nout) * size_t(r->n_bins) * 8;
                    r->res = static_cast<double *>(pinned.get(r->res_bytes));
                    if (!r->res) res_ok = false;
                }
            const auto t_batch = Clock::now();
            if (!d_in || !d_out || !res_ok || (!plain && !multi)) {
                st = DG_DEVICE;
                err = "request loop staging allocation failed";
            } else {
                std::vector<dg_multi_item> items;
                for (auto &g : groups) {
                    const size_t fb = g.reqs.front()->frame_bytes, nf = g.reqs.size();
                    const size_t nb = size_t(g.plan->n_bins);
                    for (size_t i = 0; i < nf; ++i)
                        cudaMemcpyAsync(d_in + g.in_off + i * fb, g.reqs[i]->frame, fb,
                                        cudaMemcpyHostToDevice, stream);
                    dg_multi_item m{};
                    m.plan = g.plan;
                    m.d_frames = d_in + g.in_off;
                    m.n_frames = int64_t(nf);
                    double *o = d_out + g.out_off;
                    int k = 0;
                    m.d_intensity = o + nf * nb * k++;
                    if (head->flags & DG_ERRORS) m.d_sigma = o + nf * nb * k++;
                    if (head->flags & DG_AZIMUTHAL_STD) m.d_std = o + nf * nb * k++;
                    items.push_back(m);
                }
                if (plain) {
                    const dg_multi_item &m = items.front();
                    st = dg_integrate_device(m.plan, m.d_frames, head->dtype, m.n_frames,
                                             head->flags, m.d_intensity, m.d_sigma, m.d_std,
                                             stream);
                } else {
                    st = dg_multi_integrate(multi, items.data(), int32_t(items.size()),
                                            head->dtype, head->flags, stream);
                }
                if (st != DG_OK) err = last_error_text();
                for (auto &g : groups) {
                    const size_t nf = g.reqs.size(), nb = size_t(g.plan->n_bins);
                    for (size_t i = 0; i < nf; ++i)
                        for (int k = 0; k < nout; ++k)
                            cudaMemcpyAsync(g.reqs[i]->res + k * nb,
                                            d_out + g.out_off + (k * nf + i) * nb, nb * 8,
                                            cudaMemcpyDeviceToHost, stream);
                }
                if (cudaStreamSynchronize(stream) != cudaSuccess && st == DG_OK) {
                    st = DG_DEVICE;
                    err = cudaGetErrorString(cudaGetLastError());
                }
                for (auto &g : groups)
                    if (st == DG_OK && dg::bin_tile_wait_failed(g.plan->gather)) {
                        st = DG_TIMEOUT;
                        err = "bin-tile gather: a chunk-pipeline wait gave up after 1 s";
                    }
            }
            for (auto &g : groups) release(g.key, g.plan);
            {
                std::lock_guard<std::mutex> lock(mu);
                stats.batch_us += int64_t(
                    std::chrono::duration<double, std::micro>(Clock::now() - t_batch).count());
                stats.launches++;
                if (n_frames > 1) stats.coalesced_frames += int64_t(n_frames);
                for (auto &g : groups)
                    for (Request *r : g.reqs) finish_locked(r, st, err);
            }
            cv_done.notify_all();
            cv_slot.notify_all();
        }
        if (d_in) cudaFreeAsync(d_in, stream);
        if (d_out) cudaFreeAsync(d_out, stream);
        if (stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
        if (multi) dg_multi_destroy(multi);
    }
};

namespace {
dg_status server_fail(dg_status st, const std::string &msg) {
    dg::set_last_error(msg);
    return st;
}
}  // namespace

extern "C" {

dg_status dg_server_create(const dg_server_config *config, dg_server **out) {
    if (!config || !out) return server_fail(DG_INVALID_INPUT, "config and out must not be NULL");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || config->device < 0 ||
        config->device >= count) {
        (void)cudaGetLastError();
        return server_fail(DG_UNAVAILABLE, "no such CUDA device");
    }
    if (config->max_inflight_frames <= 0 || config->cache_bytes <= 0 || config->max_coalesce <= 0)
        return server_fail(DG_INVALID_INPUT, "server limits must be positive");
    auto s = std::make_unique<dg_server>();
    s->cfg = *config;
    for (int i = 0; i < dg_server::kWorkers; ++i)
        s->workers.emplace_back([p = s.get()] { p->worker_main(); });
    // two builders: a rebuild of one large plan does not hold up another's
    for (int i = 0; i < 2; ++i) s->builders.emplace_back([p = s.get()] { p->builder_main(); });
    *out = s.release();
    return DG_OK;
}

dg_status dg_server_destroy(dg_server *server) {
    if (!server) return DG_OK;
    {
        std::unique_lock<std::mutex> lock(server->mu);
        server->stop = true;
    }
    server->cv_work.notify_all();
    server->cv_build.notify_all();
    for (auto &t : server->workers) t.join();
    for (auto &t : server->builders) t.join();
    for (dg_plan *p : server->to_destroy) dg_plan_destroy(p);
    for (auto &kv : server->cache) dg_plan_destroy(kv.second.plan);
    for (auto &e : server->retired) dg_plan_destroy(e.plan);
    for (auto &kv : server->requests) {
        if (kv.second->frame && !kv.second->borrowed)
            server->pinned.put(kv.second->frame_bytes, kv.second->frame);
        if (kv.second->res) server->pinned.put(kv.second->res_bytes, kv.second->res);
    }
    delete server;
    return DG_OK;
}

dg_status dg_server_register(dg_server *server, uint64_t key, const dg_geometry *geometry,
                             const dg_method *method, const uint8_t *mask, int32_t dim1,
                             int32_t dim2, int32_t n_radial, int32_t n_azimuthal,
                             const double *azimuthal_range) {
    if (!server || !geometry || !method || dim1 <= 0 || dim2 <= 0 || n_radial <= 0)
        return server_fail(DG_INVALID_INPUT, "invalid plan registration");
    PlanSpec spec;
    spec.geometry = *geometry;
    spec.method = *method;
    spec.method.device = server->cfg.device;
    if (mask) spec.mask.assign(mask, mask + int64_t(dim1) * dim2);
    spec.dim1 = dim1;
    spec.dim2 = dim2;
    spec.n_radial = n_radial;
    spec.n_azimuthal = n_azimuthal;
    if (azimuthal_range) {
        spec.has_az_range = true;
        spec.az_range[0] = azimuthal_range[0];
        spec.az_range[1] = azimuthal_range[1];
    }
    {
        std::unique_lock<std::mutex> lock(server->mu);
        // A re-registered key (a changed PONI) gets a new generation; its
        // cached plan is retired (now, or when its users finish).
        spec.generation = server->next_generation++;
        server->specs[key] = std::move(spec);
        server->failed.erase(key);
        auto it = server->cache.find(key);
        if (it != server->cache.end()) server->retire_locked(it);
    }
    return DG_OK;
}

dg_status dg_server_submit(dg_server *server, uint64_t key, const void *frame, int32_t dtype,
                           uint32_t flags, int32_t wait_ms, uint64_t *ticket) {
    if (!server || !frame || !ticket) return server_fail(DG_INVALID_INPUT, "NULL argument");
    if (dtype < DG_U16 || dtype > DG_F64) return server_fail(DG_INVALID_INPUT, "unknown dtype");
    if (flags & ~(DG_ERRORS | DG_AZIMUTHAL_STD | DG_SUBMIT_BORROW))
        return server_fail(DG_INVALID_INPUT, "unknown flags");
    const bool borrow = (flags & DG_SUBMIT_BORROW) != 0;
    flags &= ~DG_SUBMIT_BORROW;
    std::unique_lock<std::mutex> lock(server->mu);
    auto spec = server->specs.find(key);
    if (spec == server->specs.end()) return server_fail(DG_INVALID_INPUT, "unregistered plan key");
    const size_t bytes = size_t(spec->second.dim1) * spec->second.dim2 * px_size(dtype);
    if (!server->cv_slot.wait_for(lock, std::chrono::milliseconds(std::max(wait_ms, 0)), [&] {
            return server->inflight < server->cfg.max_inflight_frames;
        }))
        return server_fail(DG_TIMEOUT, "no request slot freed in time");
    server->inflight++;  // the slot is taken; the copy happens unlocked
    lock.unlock();
    auto r = std::make_unique<Request>();
    r->key = key;
    r->dtype = dtype;
    r->flags = flags;
    r->submitted = Clock::now();
    r->frame_bytes = bytes;
    r->borrowed = borrow;
    r->frame = borrow ? const_cast<void *>(frame) : server->pinned.get(bytes);
    if (!r->frame) {
        lock.lock();
        server->inflight--;
        lock.unlock();
        server->cv_slot.notify_one();
        return server_fail(DG_DEVICE, "pinned staging allocation failed");
    }
    if (!borrow) std::memcpy(r->frame, frame, bytes);
    lock.lock();
    r->ticket = server->next_ticket++;
    *ticket = r->ticket;
    server->queue.push_back(r.get());
    server->requests[r->ticket] = std::move(r);
    server->stats.submitted++;
    lock.unlock();
    server->cv_work.notify_one();
    return DG_OK;
}

dg_status dg_server_poll(dg_server *server, uint64_t ticket, int32_t wait_ms, double *oi,
                         double *os, double *od, double *latency_us) {
    if (!server) return server_fail(DG_INVALID_INPUT, "server must not be NULL");
    std::unique_lock<std::mutex> lock(server->mu);
    auto it = server->requests.find(ticket);
    if (it == server->requests.end()) return server_fail(DG_INVALID_INPUT, "unknown ticket");
    Request *r = it->second.get();
    if (!server->cv_done.wait_for(lock, std::chrono::milliseconds(std::max(wait_ms, 0)),
                                  [&] { return r->done; }))
        return server_fail(DG_TIMEOUT, "request not finished");
    dg_status st = r->status;
    if (st == DG_OK) {
        const int64_t nb = r->n_bins;
        int k = 0;
        if (oi) std::memcpy(oi, r->res, size_t(nb) * 8);
        ++k;
        if (r->flags & DG_ERRORS) {
            if (os) std::memcpy(os, r->res + k * nb, size_t(nb) * 8);
            ++k;
        }
        if ((r->flags & DG_AZIMUTHAL_STD) && od) std::memcpy(od, r->res + k * nb, size_t(nb) * 8);
        server->pinned.put(r->res_bytes, r->res);
        r->res = nullptr;
    } else {
        server_fail(st, r->error);
    }
    if (latency_us) *latency_us = r->latency_us;
    server->requests.erase(it);
    return st;
}

dg_status dg_server_stats_get(dg_server *server, dg_server_stats *out) {
    if (!server || !out) return server_fail(DG_INVALID_INPUT, "NULL argument");
    std::unique_lock<std::mutex> lock(server->mu);
    *out = server->stats;
    out->cache_bytes = server->cache_bytes;
    return DG_OK;
}

}  // extern "C"
