// Request loop: continuous batching of single-frame requests across plans.
//
// Requests are admitted while in-flight slots remain (a submit waits, bounded,
// for a slot). Worker threads take the oldest queued request, coalesce every
// queued request with the same plan key, dtype and flags behind it (up to
// max_coalesce) into one launch, and publish results per request. Plans live
// in an HBM cache bounded by bytes: a miss builds the plan on the device, and
// least-recently-used plans that no worker is using are evicted until the
// cache fits. Four workers run batches concurrently on their own streams,
// so one batch's copies overlap another's gather. A submit copies its frame
// into a pooled pinned buffer outside the server lock; the worker copies the
// pinned buffers straight to the device. Re-registering a key (a changed
// PONI) gives it a new generation: the next request rebuilds the plan, and
// the stale plan is destroyed once no worker uses it. Each request's result
// is identical alone and in any mix: the gather's arithmetic depends only on
// the plan, never on which frames share a launch.
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
    void *get(size_t bytes) {
        {
            std::lock_guard<std::mutex> lock(mu);
            auto &v = free[bytes];
            if (!v.empty()) {
                void *p = v.back();
                v.pop_back();
                return p;
            }
        }
        void *p = nullptr;
        if (cudaMallocHost(&p, bytes) != cudaSuccess) {
            (void)cudaGetLastError();
            return nullptr;
        }
        return p;
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
    std::vector<double> out_i, out_s, out_d;
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
    std::condition_variable cv_work, cv_done, cv_slot;
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
    PinnedPool pinned;
    std::vector<CacheEntry> retired;  // stale plans still in use
    uint64_t next_generation = 1;
    std::unordered_map<uint64_t, int> building;  // keys a worker is building now
    std::unordered_map<uint64_t, int32_t> tuned;  // key -> lane mapping its last plan used

    // Returns a plan for `key` with a user reference, building it on a miss and
    // evicting idle LRU plans to stay within the byte budget. Called unlocked.
    // A new plan's lane mapping, tuned for the small coalesced launches of the
    // loop on zero frames of the request's type (timing does not depend on
    // the values); left at the default if anything fails.
    void tune(dg_plan *plan, int32_t dtype, uint32_t flags) {
        const int64_t nf = std::max(1, std::min(8, cfg.max_coalesce));
        const size_t bytes = size_t(plan->dim1) * plan->dim2 * px_size(dtype) * size_t(nf);
        void *d = nullptr;
        if (cudaMalloc(&d, bytes) != cudaSuccess) {
            (void)cudaGetLastError();
            return;
        }
        cudaMemsetAsync(d, 0, bytes, plan->stream);
        if (dg_plan_autotune(plan, d, dtype, nf, flags & (DG_ERRORS | DG_AZIMUTHAL_STD), nullptr,
                             nullptr, nullptr, 0) != DG_OK)
            (void)last_error_text();
        cudaFree(d);
    }

    dg_plan *acquire(uint64_t key, int32_t dtype, uint32_t flags, std::string &err,
                     dg_status &st) {
        PlanSpec spec;
        {
            std::unique_lock<std::mutex> lock(mu);
            spec = specs.at(key);
            auto it = cache.find(key);
            if (it != cache.end() && it->second.generation == spec.generation) {
                it->second.users++;
                it->second.last_use = ++use_clock;
                stats.plan_hits++;
                return it->second.plan;
            }
            if (it != cache.end()) retire_locked(it);
            building[key]++;
        }
        struct Built {
            dg_server *s;
            uint64_t key;
            ~Built() {
                std::lock_guard<std::mutex> lock(s->mu);
                if (--s->building[key] == 0) s->building.erase(key);
            }
        } built{this, key};
        const auto t_build = Clock::now();
        dg_plan *plan = nullptr;
        st = dg_plan_create(&spec.geometry, &spec.method, spec.mask.empty() ? nullptr : spec.mask.data(),
                            spec.dim1, spec.dim2, spec.n_radial, spec.n_azimuthal,
                            spec.has_az_range ? spec.az_range : nullptr, &plan);
        if (st != DG_OK) {
            err = last_error_text();
            return nullptr;
        }
        // A rebuilt key (new PONI, same shape and bins) keeps the mapping its
        // previous plan was tuned to; a new key is tuned once.
        int32_t known = -1;
        {
            std::lock_guard<std::mutex> lock(mu);
            auto t = tuned.find(key);
            if (t != tuned.end()) known = t->second;
        }
        if (known < 0 || dg_plan_variant(plan, known, nullptr, nullptr) != DG_OK) {
            tune(plan, dtype, flags);
            int32_t v = 0;
            dg_plan_variant(plan, -1, &v, nullptr);
            std::lock_guard<std::mutex> lock(mu);
            tuned[key] = v;
        }
        {
            std::lock_guard<std::mutex> lock(mu);
            stats.build_us += int64_t(
                std::chrono::duration<double, std::micro>(Clock::now() - t_build).count());
        }
        dg_plan_info info{};
        dg_plan_query(plan, &info);
        std::vector<dg_plan *> evicted;
        dg_plan *result = nullptr;
        {
            std::unique_lock<std::mutex> lock(mu);
            auto it = cache.find(key);
            if (it != cache.end() && it->second.generation != spec.generation) {
                retire_locked(it);
                it = cache.end();
            }
            if (it != cache.end()) {  // another worker built it meanwhile
                evicted.push_back(plan);
                it->second.users++;
                it->second.last_use = ++use_clock;
                result = it->second.plan;
            } else {
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
                e.users = 1;
                e.last_use = ++use_clock;
                e.generation = spec.generation;
                cache[key] = e;
                cache_bytes += e.bytes;
                result = plan;
            }
        }
        for (dg_plan *p : evicted) dg_plan_destroy(p);
        return result;
    }

    // Moves a stale cache entry out of the cache (lock held): destroyed now
    // if idle, else when its last user releases it.
    void retire_locked(std::unordered_map<uint64_t, CacheEntry>::iterator it) {
        cache_bytes -= it->second.bytes;
        if (it->second.users == 0) {
            dg_plan *p = it->second.plan;
            cache.erase(it);
            dg_plan_destroy(p);  // not in use by any worker
            return;
        }
        retired.push_back(it->second);
        cache.erase(it);
    }

    void release(uint64_t key, dg_plan *plan) {
        dg_plan *dead = nullptr;
        {
            std::unique_lock<std::mutex> lock(mu);
            auto it = cache.find(key);
            if (it != cache.end() && it->second.plan == plan) {
                if (it->second.users > 0) it->second.users--;
            } else {
                for (size_t i = 0; i < retired.size(); ++i)
                    if (retired[i].plan == plan) {
                        if (--retired[i].users == 0) {
                            dead = plan;
                            retired.erase(retired.begin() + long(i));
                        }
                        break;
                    }
            }
        }
        if (dead) dg_plan_destroy(dead);
    }

    void worker_main() {
        cudaSetDevice(cfg.device);
        cudaStream_t stream = nullptr;
        cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
        unsigned char *d_in = nullptr;
        double *d_out = nullptr, *h_out = nullptr;
        size_t in_cap = 0, out_cap = 0;
        for (;;) {
            std::vector<Request *> batch;
            {
                std::unique_lock<std::mutex> lock(mu);
                cv_work.wait_for(lock, std::chrono::microseconds(std::max(cfg.poll_us, 50)),
                                 [&] { return stop || !queue.empty(); });
                if (stop && queue.empty()) break;
                if (queue.empty()) continue;
                // the oldest request whose plan no other worker is building
                auto hit = queue.begin();
                while (hit != queue.end() && building.count((*hit)->key)) ++hit;
                if (hit == queue.end()) {
                    lock.unlock();
                    std::this_thread::sleep_for(std::chrono::microseconds(200));
                    continue;
                }
                Request *head = *hit;
                queue.erase(hit);
                batch.push_back(head);
                for (auto it = queue.begin(); it != queue.end() &&
                                              int(batch.size()) < cfg.max_coalesce;) {
                    Request *r = *it;
                    if (r->key == head->key && r->dtype == head->dtype && r->flags == head->flags) {
                        batch.push_back(r);
                        it = queue.erase(it);
                    } else {
                        ++it;
                    }
                }
            }
            Request *head = batch.front();
            std::string err;
            dg_status st = DG_OK;
            dg_plan *plan = acquire(head->key, head->dtype, head->flags, err, st);
            if (plan) {
                const size_t fb = head->frame_bytes;
                const int64_t nb = plan->n_bins;
                const int nout = 1 + ((head->flags & DG_ERRORS) ? 1 : 0) +
                                 ((head->flags & DG_AZIMUTHAL_STD) ? 1 : 0);
                const size_t nf = batch.size();
                if (in_cap < nf * fb) {
                    if (d_in) cudaFree(d_in);
                    in_cap = nf * fb;
                    if (cudaMalloc(&d_in, in_cap) != cudaSuccess) {
                        (void)cudaGetLastError();
                        d_in = nullptr;
                        in_cap = 0;
                    }
                }
                if (out_cap < nf * size_t(nb) * nout) {
                    if (d_out) cudaFree(d_out);
                    if (h_out) cudaFreeHost(h_out);
                    out_cap = nf * size_t(nb) * nout;
                    if (cudaMalloc(&d_out, out_cap * 8) != cudaSuccess ||
                        cudaMallocHost(&h_out, out_cap * 8) != cudaSuccess) {
                        (void)cudaGetLastError();
                        d_out = nullptr;
                        h_out = nullptr;
                        out_cap = 0;
                    }
                }
                const auto t_batch = Clock::now();
                if (!d_in || !d_out) {
                    st = DG_DEVICE;
                    err = "request loop staging allocation failed";
                } else {
                    for (size_t i = 0; i < nf; ++i)
                        cudaMemcpyAsync(d_in + i * fb, batch[i]->frame, fb, cudaMemcpyHostToDevice,
                                        stream);
                    double *di = d_out, *ds = nullptr, *dd = nullptr;
                    int k = 1;
                    if (head->flags & DG_ERRORS) ds = d_out + nf * nb * k++;
                    if (head->flags & DG_AZIMUTHAL_STD) dd = d_out + nf * nb * k++;
                    st = dg_integrate_device(plan, d_in, head->dtype, int64_t(nf), head->flags, di,
                                             ds, dd, stream);
                    if (st != DG_OK) err = last_error_text();
                    cudaMemcpyAsync(h_out, d_out, nf * nb * nout * 8, cudaMemcpyDeviceToHost,
                                    stream);
                    if (cudaStreamSynchronize(stream) != cudaSuccess && st == DG_OK) {
                        st = DG_DEVICE;
                        err = cudaGetErrorString(cudaGetLastError());
                    }
                    if (st == DG_OK && dg::bin_tile_wait_failed(plan->gather)) {
                        st = DG_TIMEOUT;
                        err = "bin-tile gather: a chunk-pipeline wait gave up after 1 s";
                    }
                    if (st == DG_OK) {
                        for (size_t i = 0; i < nf; ++i) {
                            Request *r = batch[i];
                            int kk = 0;
                            r->out_i.assign(h_out + i * nb, h_out + (i + 1) * nb);
                            ++kk;
                            if (ds) {
                                r->out_s.assign(h_out + (kk * nf + i) * nb,
                                                h_out + (kk * nf + i + 1) * nb);
                                ++kk;
                            }
                            if (dd)
                                r->out_d.assign(h_out + (kk * nf + i) * nb,
                                                h_out + (kk * nf + i + 1) * nb);
                        }
                    }
                }
                release(head->key, plan);
                std::lock_guard<std::mutex> lock(mu);
                stats.batch_us += int64_t(
                    std::chrono::duration<double, std::micro>(Clock::now() - t_batch).count());
            }
            {
                std::unique_lock<std::mutex> lock(mu);
                auto now = Clock::now();
                stats.launches++;
                if (batch.size() > 1) stats.coalesced_frames += int64_t(batch.size());
                for (Request *r : batch) {
                    r->status = st;
                    r->error = err;
                    r->done = true;
                    r->latency_us =
                        std::chrono::duration<double, std::micro>(now - r->submitted).count();
                    if (st == DG_OK) stats.completed++;
                    else stats.failed++;
                    if (!r->borrowed) pinned.put(r->frame_bytes, r->frame);
                    r->frame = nullptr;
                    inflight--;
                }
            }
            cv_done.notify_all();
            cv_slot.notify_all();
        }
        if (d_in) cudaFree(d_in);
        if (d_out) cudaFree(d_out);
        if (h_out) cudaFreeHost(h_out);
        if (stream) cudaStreamDestroy(stream);
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
    for (int i = 0; i < 4; ++i) s->workers.emplace_back([p = s.get()] { p->worker_main(); });
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
    for (auto &t : server->workers) t.join();
    for (auto &kv : server->cache) dg_plan_destroy(kv.second.plan);
    for (auto &e : server->retired) dg_plan_destroy(e.plan);
    for (auto &kv : server->requests)
        if (kv.second->frame) server->pinned.put(kv.second->frame_bytes, kv.second->frame);
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
        if (oi) std::copy(r->out_i.begin(), r->out_i.end(), oi);
        if (os && !r->out_s.empty()) std::copy(r->out_s.begin(), r->out_s.end(), os);
        if (od && !r->out_d.empty()) std::copy(r->out_d.begin(), r->out_d.end(), od);
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
