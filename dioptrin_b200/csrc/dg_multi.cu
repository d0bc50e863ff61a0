// Batches of several plans in one launch: the work-queue gather.
//
// A dg_multi holds the device descriptors of one call (a header and one
// QueuePlan per plan batch) and, per pixel type and output set, a CUDA graph
// of the call's device work: the copy of the descriptors from page-locked
// host staging and the work-queue gather (row-warp CTAs that claim (plan,
// row item, block of four frames) tiles from a counter the copy resets and
// write each row's results themselves). The graph is captured on the first
// call of its kind and replayed after that, the descriptors and the gather's
// grid changing between calls while the graph stays the same: one graph
// launch per batch of plans, whatever their number and sizes. The grid is
// one CTA per tile, which the hardware schedules as CTAs retire, beside other
// streams' kernels; a batch of more than 2^24 tiles runs a resident grid (the
// CTAs the SMs hold at once) whose CTAs claim tiles until the queue is empty. No plan scratch is used, so calls on
// different streams that share plans are not ordered against each other. The
// reference's streaming driver (src/batch/bounded.rs:172) and its engine's
// pipelined tiles (src/integration/cuda/device.rs:1417-1584) keep one plan
// per launch.
#include <algorithm>
#include <climits>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <vector>

#include "dg_internal.h"

struct dg_multi {
    std::mutex mu;
    int32_t device = 0;
    int32_t max_plans = 0;
    dg::DeviceArray<unsigned char> dev;  // QueueHeader, then max_plans QueuePlans
    unsigned char *host = nullptr;       // page-locked staging of the same layout
    size_t bytes = 0;
    cudaStream_t capture = nullptr;      // graphs are captured here, launched anywhere
    cudaEvent_t done = nullptr;          // the last call's device work has finished
    bool pending = false;
    bool resident = false;               // test hook: the claiming grid for every call
    // Per (dtype, flags): the captured graph, its instance, and the gather's
    // kernel node, whose grid is set for each call.
    struct Graph {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaGraphNode_t kernel = nullptr;
        cudaKernelNodeParams params{};
    };
    std::map<std::pair<int32_t, uint32_t>, Graph> graphs;
    ~dg_multi() {
        for (auto &g : graphs) {
            if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
            if (g.second.graph) cudaGraphDestroy(g.second.graph);
        }
        if (done) cudaEventDestroy(done);
        if (capture) cudaStreamDestroy(capture);
        if (host) cudaFreeHost(host);
    }
};

namespace {

dg_status multi_guard(const std::function<void()> &f) {
    try {
        f();
        return DG_OK;
    } catch (const dg::Error &e) {
        dg::set_last_error(e.message);
        return e.status;
    } catch (const std::exception &e) {
        dg::set_last_error(e.what());
        return DG_DEVICE;
    } catch (...) {
        dg::set_last_error("unknown failure");
        return DG_DEVICE;
    }
}

size_t px_bytes(int32_t dtype) {
    switch (dtype) {
    case DG_U16: return 2;
    case DG_U32:
    case DG_I32:
    case DG_F32: return 4;
    case DG_F64: return 8;
    default: dg::fail(DG_INVALID_INPUT, "unknown pixel dtype " + std::to_string(dtype));
    }
}

// Makes `device` current for the scope and restores the caller's device.
struct Scope {
    int previous = -1;
    explicit Scope(int device) {
        DG_CUDA(cudaGetDevice(&previous));
        if (previous != device) DG_CUDA(cudaSetDevice(device));
    }
    ~Scope() {
        int now = -1;
        if (cudaGetDevice(&now) == cudaSuccess && now != previous && previous >= 0)
            cudaSetDevice(previous);
    }
};

}  // namespace

extern "C" {

dg_status dg_multi_create(int32_t device, int32_t max_plans, dg_multi **out) {
    return multi_guard([&] {
        if (!out) dg::fail(DG_INVALID_INPUT, "out must not be NULL");
        *out = nullptr;
        if (max_plans <= 0 || max_plans > 4096)
            dg::fail(DG_INVALID_INPUT, "max_plans must be in 1..4096");
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
            (void)cudaGetLastError();
            dg::fail(DG_UNAVAILABLE, "CUDA device " + std::to_string(device) + " does not exist");
        }
        Scope scope(device);
        auto m = std::make_unique<dg_multi>();
        m->device = device;
        m->max_plans = max_plans;
        m->bytes = sizeof(dg::QueueHeader) + size_t(max_plans) * sizeof(dg::QueuePlan);
        m->dev.alloc(m->bytes);
        if (cudaHostAlloc(reinterpret_cast<void **>(&m->host), m->bytes, cudaHostAllocPortable) !=
            cudaSuccess) {
            (void)cudaGetLastError();
            m->host = nullptr;
            dg::fail(DG_DEVICE, "page-locked descriptor staging allocation failed");
        }
        std::memset(m->host, 0, m->bytes);
        DG_CUDA(cudaStreamCreateWithFlags(&m->capture, cudaStreamNonBlocking));
        DG_CUDA(cudaEventCreateWithFlags(&m->done, cudaEventDisableTiming));
        *out = m.release();
    });
}

dg_status dg_multi_destroy(dg_multi *multi) {
    if (!multi) return DG_OK;
    {
        std::lock_guard<std::mutex> lock(multi->mu);
        if (multi->pending) cudaEventSynchronize(multi->done);
    }
    int previous = -1;
    cudaGetDevice(&previous);
    cudaSetDevice(multi->device);
    delete multi;
    if (previous >= 0) cudaSetDevice(previous);
    return DG_OK;
}

dg_status dg_multi_test_resident(dg_multi *multi, int32_t on) {
    if (!multi) {
        dg::set_last_error("multi must not be NULL");
        return DG_INVALID_INPUT;
    }
    std::lock_guard<std::mutex> lock(multi->mu);
    multi->resident = on != 0;
    return DG_OK;
}

dg_status dg_multi_integrate(dg_multi *multi, const dg_multi_item *items, int32_t n_items,
                             int32_t dtype, uint32_t flags, void *stream) {
    return multi_guard([&] {
        using dg::fail;
        if (!multi) fail(DG_INVALID_INPUT, "multi must not be NULL");
        if (n_items < 0 || n_items > multi->max_plans)
            fail(DG_INVALID_INPUT, "n_items must be in 0..max_plans");
        if (n_items > 0 && !items) fail(DG_INVALID_INPUT, "items must not be NULL");
        const size_t es = px_bytes(dtype);
        if (flags & ~(DG_ERRORS | DG_AZIMUTHAL_STD)) fail(DG_INVALID_INPUT, "unknown flags");
        std::vector<dg_plan *> plans;
        for (int32_t i = 0; i < n_items; ++i) {
            const dg_multi_item &it = items[i];
            if (!it.plan) fail(DG_INVALID_INPUT, "item plan must not be NULL");
            if (it.plan->device != multi->device)
                fail(DG_INVALID_INPUT, "every plan must be on the multi's device");
            if (it.n_frames < 0 || it.n_frames > 256)
                fail(DG_UNSUPPORTED, "an item carries 0..256 frames");
            if (it.n_frames == 0) continue;
            if (!it.d_frames || !it.d_intensity)
                fail(DG_INVALID_INPUT, "item frames and intensity must not be NULL");
            if ((flags & DG_ERRORS) && !it.d_sigma)
                fail(DG_INVALID_INPUT, "errors requested without an output");
            if ((flags & DG_AZIMUTHAL_STD) && !it.d_std)
                fail(DG_INVALID_INPUT, "azimuthal_std requested without an output");
            if ((flags & DG_AZIMUTHAL_STD) && it.plan->n_azimuthal != 0)
                fail(DG_UNSUPPORTED, "azimuthal_std is defined for 1D tables only");
            if (reinterpret_cast<uintptr_t>(it.d_frames) % es)
                fail(DG_INVALID_INPUT, "device frames must be aligned to the pixel size");
            for (const void *o : {(const void *)it.d_intensity, (const void *)it.d_sigma,
                                  (const void *)it.d_std})
                if (reinterpret_cast<uintptr_t>(o) % 8)
                    fail(DG_INVALID_INPUT, "device outputs must be 8-byte aligned");
            plans.push_back(it.plan);
        }
        std::vector<dg_plan *> order(plans);
        std::sort(order.begin(), order.end());
        if (std::adjacent_find(order.begin(), order.end()) != order.end())
            fail(DG_INVALID_INPUT, "a plan may appear in one item of a call only");
        std::lock_guard<std::mutex> mlock(multi->mu);
        std::vector<std::unique_lock<std::mutex>> locks;
        for (dg_plan *p : order) locks.emplace_back(p->mu);  // address order: no deadlock
        Scope scope(multi->device);
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : multi->capture;
        // The previous call's graph reads the staging when it runs: wait for
        // it before overwriting the staging.
        if (multi->pending) DG_CUDA(cudaEventSynchronize(multi->done));
        multi->pending = false;
        auto *hdr = reinterpret_cast<dg::QueueHeader *>(multi->host);
        auto *desc = reinterpret_cast<dg::QueuePlan *>(multi->host + sizeof(dg::QueueHeader));
        int32_t items_total = 0, n = 0;
        for (int32_t i = 0; i < n_items; ++i) {
            const dg_multi_item &it = items[i];
            if (it.n_frames == 0) continue;
            const dg::GatherTable &t = it.plan->gather;
            dg::QueuePlan q = dg::queue_plan(
                t, it.d_frames, int64_t(it.plan->dim1) * it.plan->dim2, int(it.n_frames),
                it.d_intensity, (flags & DG_ERRORS) ? it.d_sigma : nullptr,
                (flags & DG_AZIMUTHAL_STD) ? it.d_std : nullptr);
            if (q.n_items <= 0 && t.n_rows > 0)
                fail(DG_UNSUPPORTED, "the work-queue gather needs a table of at most 2^31 entries");
            q.item_first = items_total;
            const int64_t tiles = int64_t(q.n_items) * q.frame_blocks;
            if (items_total + tiles > INT32_MAX / 2)
                fail(DG_UNSUPPORTED, "too many tiles for one launch");
            items_total += int32_t(tiles);
            desc[n++] = q;
        }
        if (n == 0) return;
        hdr->n_plans = n;
        hdr->total_items = items_total;
        hdr->counter = 0;
        const auto key = std::make_pair(dtype, flags);
        auto g = multi->graphs.find(key);
        if (g == multi->graphs.end()) {
            cudaGraph_t graph = nullptr;
            DG_CUDA(cudaStreamBeginCapture(multi->capture, cudaStreamCaptureModeThreadLocal));
            try {
                DG_CUDA(cudaMemcpyAsync(multi->dev.ptr, multi->host, multi->bytes,
                                        cudaMemcpyHostToDevice, multi->capture));
                dg::queue_launch(
                    dtype, flags, reinterpret_cast<dg::QueueHeader *>(multi->dev.ptr),
                    reinterpret_cast<const dg::QueuePlan *>(multi->dev.ptr +
                                                            sizeof(dg::QueueHeader)),
                    multi->capture);
            } catch (...) {
                cudaStreamEndCapture(multi->capture, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            DG_CUDA(cudaStreamEndCapture(multi->capture, &graph));
            dg_multi::Graph entry;
            entry.graph = graph;
            size_t n_nodes = 0;
            cudaError_t e = cudaGraphGetNodes(graph, nullptr, &n_nodes);
            std::vector<cudaGraphNode_t> nodes(n_nodes);
            if (e == cudaSuccess) e = cudaGraphGetNodes(graph, nodes.data(), &n_nodes);
            for (size_t i = 0; e == cudaSuccess && i < n_nodes; ++i) {
                cudaGraphNodeType type;
                e = cudaGraphNodeGetType(nodes[i], &type);
                if (e == cudaSuccess && type == cudaGraphNodeTypeKernel) {
                    entry.kernel = nodes[i];
                    e = cudaGraphKernelNodeGetParams(nodes[i], &entry.params);
                }
            }
            if (e == cudaSuccess && !entry.kernel) e = cudaErrorInvalidValue;
            if (e == cudaSuccess) e = cudaGraphInstantiate(&entry.exec, graph, 0);
            if (e != cudaSuccess) {
                if (entry.exec) cudaGraphExecDestroy(entry.exec);
                cudaGraphDestroy(graph);
                DG_CUDA(e);
            }
            g = multi->graphs.emplace(key, entry).first;
        }
        // this call's grid: one CTA per claim of tiles, up to the resident
        // capacity (the capture used the capacity)
        dg_multi::Graph &gr = g->second;
        gr.params.gridDim =
            dim3(unsigned(dg::queue_grid(dtype, flags, items_total, multi->resident)), 1, 1);
        DG_CUDA(cudaGraphExecKernelNodeSetParams(gr.exec, gr.kernel, &gr.params));
        DG_CUDA(cudaGraphLaunch(gr.exec, s));
        DG_CUDA(cudaEventRecord(multi->done, s));
        multi->pending = true;
        for (int32_t i = 0; i < n_items; ++i)
            if (items[i].n_frames) items[i].plan->gather.launches += 1;
    });
}

}  // extern "C"
