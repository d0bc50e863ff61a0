// C ABI of libdioptrin_b200: plan lifecycle and integration entry points.
//
// Every entry point converts failures into a dg_status and a thread-local
// message (dg_last_error); no C++ exception crosses the boundary. Calls on one
// plan are serialised by the plan's mutex; separate plans run concurrently
// (src/integration/cuda.rs:374-386 gives the reference's same rule).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>

#include "dg_internal.h"

namespace dg {

[[noreturn]] void fail(dg_status status, const std::string &message) {
    throw Error{status, message};
}

void check_cuda(cudaError_t err, const char *what) {
    if (err == cudaSuccess) return;
    (void)cudaGetLastError();
    fail(DG_DEVICE, std::string(what) + ": " + cudaGetErrorString(err));
}

}  // namespace dg

namespace {

thread_local std::string g_last_error;

// Detector rows per gather strip (see dg_gather.cu): small enough that a
// unit's bins cover a few kilobytes of each frame, large enough that a bin's
// ring is cut into few segments. A 2D bin is a compact patch of ~100
// entries, so its plans take taller strips: most of its rows are then one
// segment, with fewer partial sums to write and fold (the Eiger-9M cake's
// 64-frame batch: 1.17 against 1.35 ms, 261 k → 153 k segments).
#ifndef DG_STRIP_ROWS
#define DG_STRIP_ROWS 16
#endif
#ifndef DG_STRIP_ROWS_2D
#define DG_STRIP_ROWS_2D 64
#endif
constexpr int32_t kStripRows = DG_STRIP_ROWS;
constexpr int32_t kStripRows2d = DG_STRIP_ROWS_2D;

}  // namespace

void dg::set_last_error(const std::string &message) { g_last_error = message; }

namespace {

template <class F>
dg_status guarded(F &&f) {
    try {
        f();
        return DG_OK;
    } catch (const dg::Error &e) {
        g_last_error = e.message;
        return e.status;
    } catch (const std::bad_alloc &) {
        g_last_error = "host allocation failed";
        return DG_DEVICE;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return DG_DEVICE;
    } catch (...) {
        g_last_error = "unknown failure";
        return DG_DEVICE;
    }
}

// Makes `device` current for the scope and restores the caller's device.
struct DeviceScope {
    int previous = -1;
    explicit DeviceScope(int device) {
        DG_CUDA(cudaGetDevice(&previous));
        if (previous != device) DG_CUDA(cudaSetDevice(device));
    }
    ~DeviceScope() {
        int now = -1;
        if (cudaGetDevice(&now) == cudaSuccess && now != previous && previous >= 0)
            cudaSetDevice(previous);
    }
};

size_t dtype_size(int32_t dtype) {
    switch (dtype) {
    case DG_U16: return 2;
    case DG_U32:
    case DG_I32:
    case DG_F32: return 4;
    case DG_F64: return 8;
    default: dg::fail(DG_INVALID_INPUT, "unknown pixel dtype " + std::to_string(dtype));
    }
}

// check_configuration (src/integration/cuda.rs:1001-1057), in its order.
void check_config(const dg_geometry *g, const dg_method *m, int32_t dim1, int32_t dim2,
                  int32_t n_radial, int32_t n_azimuthal) {
    using dg::fail;
    if (!g || !m) fail(DG_INVALID_INPUT, "geometry and method must not be NULL");
    if (n_radial <= 0) fail(DG_INVALID_INPUT, "n_points must be between 1 and 2147483647");
    if (n_azimuthal < 0) fail(DG_INVALID_INPUT, "n_azimuthal must not be negative");
    if (m->flags & ~(DG_PLAN_KEEP_TABLES | DG_PLAN_FLIP_VERTICAL))
        fail(DG_INVALID_INPUT, "unknown plan flags");
    if (n_azimuthal > 0 && int64_t(n_radial) * n_azimuthal > INT32_MAX)
        fail(DG_INVALID_INPUT, "2D bin count must be in 1..=2147483647");
    if (dim1 <= 0 || dim2 <= 0)
        fail(DG_INVALID_INPUT, "image shape (" + std::to_string(dim1) + ", " +
                                   std::to_string(dim2) + ") has a zero side");
    if (int64_t(dim1) * dim2 > int64_t(INT32_MAX))
        fail(DG_INVALID_INPUT, "image shape exceeds 2147483647 pixels");
    if (m->max_batch_bytes < 0) fail(DG_INVALID_INPUT, "max_batch_bytes must be positive");
    if (m->kind < DG_METHOD_COUNTING || m->kind > DG_METHOD_SUPERSAMPLED)
        fail(DG_UNSUPPORTED, "unknown integration method");
    if (m->kind == DG_METHOD_SUPERSAMPLED && m->n_ss <= 0)
        fail(DG_INVALID_INPUT, "n_ss must be positive");
    if (m->unit < DG_UNIT_TTH_RAD || m->unit > DG_UNIT_Q_NM)
        fail(DG_INVALID_INPUT, "unknown radial unit");
    if ((m->unit == DG_UNIT_Q_A || m->unit == DG_UNIT_Q_NM) && !(g->wavelength > 0.0))
        fail(DG_INVALID_INPUT, "Wavelength must be positive for q conversion");
    if (m->precision < DG_PRECISION_F32 || m->precision > DG_PRECISION_F64)
        fail(DG_INVALID_INPUT, "unknown precision");
    if (m->has_radial_range &&
        !(std::isfinite(m->radial_min) && std::isfinite(m->radial_max) &&
          m->radial_min < m->radial_max))
        fail(DG_INVALID_INPUT, "radial_range must be finite with min < max");
    if (m->has_polarization &&
        !(m->polarization_factor >= -1.0 && m->polarization_factor <= 1.0))
        fail(DG_INVALID_INPUT, "polarization_factor must lie in [-1, 1]");
}

void check_device(int32_t device) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        dg::fail(DG_UNAVAILABLE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    if (device < 0 || device >= count)
        dg::fail(DG_UNAVAILABLE, "CUDA device " + std::to_string(device) + " does not exist (" +
                                     std::to_string(count) + " visible)");
}

void check_frames(const dg_plan *plan, const void *frames, int32_t dtype, int64_t n_frames,
                  uint32_t flags, const void *oi, const void *os, const void *od) {
    using dg::fail;
    if (!plan) fail(DG_INVALID_INPUT, "plan must not be NULL");
    (void)dtype_size(dtype);
    if (n_frames < 0) fail(DG_INVALID_INPUT, "frame count must not be negative");
    if (flags & ~(DG_ERRORS | DG_AZIMUTHAL_STD)) fail(DG_INVALID_INPUT, "unknown flags");
    if (n_frames == 0) return;
    if (!frames) fail(DG_INVALID_INPUT, "frames must not be NULL");
    if (!oi) fail(DG_INVALID_INPUT, "intensity output must not be NULL");
    if ((flags & DG_ERRORS) && !os) fail(DG_INVALID_INPUT, "errors requested without an output");
    if ((flags & DG_AZIMUTHAL_STD) && !od)
        fail(DG_INVALID_INPUT, "azimuthal_std requested without an output");
    if (flags & DG_AZIMUTHAL_STD) {
        if (plan->n_azimuthal != 0)
            fail(DG_UNSUPPORTED, "azimuthal_std is defined for 1D tables only");
    }
}

// Device arrays must be aligned to their element size (the kernels load
// pixels with naturally aligned loads and asynchronous 4-byte copies).
void check_device_alignment(const void *frames, int32_t dtype, const void *oi, const void *os,
                            const void *od) {
    const uintptr_t es = uintptr_t(dtype_size(dtype));
    if (reinterpret_cast<uintptr_t>(frames) % es)
        dg::fail(DG_INVALID_INPUT, "device frames must be aligned to the pixel size");
    for (const void *o : {oi, os, od})
        if (reinterpret_cast<uintptr_t>(o) % 8)
            dg::fail(DG_INVALID_INPUT, "device outputs must be 8-byte aligned");
}

}  // namespace

int64_t dg_plan::device_bytes() const {
    int64_t b = 0;
    b += full.row_ptr.bytes() + full.col.bytes() + full.w.bytes();
    b += table.row_ptr.bytes() + table.col.bytes() + table.w.bytes();
    b += norm.bytes();
    b += gather.seg.bytes() + gather.unit.bytes() + gather.row_seg.bytes() +
         gather.seg_ids.bytes() + gather.first_valid.bytes() + gather.entry.bytes() +
         gather.entry_std.bytes() + gather.den.bytes() + gather.den_std.bytes() +
         gather.entry_nlo.bytes() + gather.origin.bytes() +
         gather.valid_std.bytes() + gather.partial.bytes() + gather.fl_unit.bytes() +
         gather.fl_px.bytes() + gather.fl_pair_a.bytes() + gather.fl_pair_b.bytes() +
         gather.fl_pair_c.bytes() +
         gather.fl_pair_s.bytes() + gather.fl_seg_org.bytes() + gather.entry_raw.bytes() +
         gather.cnt.bytes() + gather.bt[0].bytes() + gather.bt[1].bytes() +
         gather.rw_row_ptr.bytes() + gather.rw_rows.bytes() + gather.rw_item.bytes() +
         gather.px_norm.bytes();
    b += stage_in.bytes() + stage_out.bytes() + stage_comp.bytes() + stage_desc.bytes() +
         stage_mask.bytes();
    return b;
}

extern "C" {

dg_status dg_plan_create(const dg_geometry *geometry, const dg_method *method,
                         const uint8_t *mask, int32_t dim1, int32_t dim2, int32_t n_radial,
                         int32_t n_azimuthal, const double *azimuthal_range, dg_plan **out) {
    return guarded([&] {
        if (!out) dg::fail(DG_INVALID_INPUT, "out must not be NULL");
        *out = nullptr;
        check_config(geometry, method, dim1, dim2, n_radial, n_azimuthal);
        check_device(method->device);
        DeviceScope scope(method->device);
        auto plan = std::make_unique<dg_plan>();
        plan->device = method->device;
        plan->geometry = *geometry;
        plan->method = *method;
        plan->dim1 = dim1;
        plan->dim2 = dim2;
        plan->n_radial = n_radial;
        plan->n_azimuthal = n_azimuthal;
        plan->n_bins = n_azimuthal ? int64_t(n_radial) * n_azimuthal : n_radial;
        // The plan's own stream runs at the device's greatest priority: its
        // build (and calls that pass no stream) go ahead of other queued work,
        // e.g. a request loop's persistent gathers.
        int least = 0, greatest = 0;
        DG_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        DG_CUDA(cudaStreamCreateWithPriority(&plan->stream, cudaStreamNonBlocking, greatest));
        cudaStream_t s = plan->stream;
        cudaEvent_t e0, e1;
        DG_CUDA(cudaEventCreate(&e0));
        DG_CUDA(cudaEventCreate(&e1));
        DG_CUDA(cudaEventRecord(e0, s));
        dg::BuildResult built;
        try {
            dg::build_table(*geometry, *method, dim1, dim2, n_radial, n_azimuthal,
                            azimuthal_range, s, built);
            const int64_t npix = int64_t(dim1) * dim2;
            dg::DeviceArray<uint8_t> d_mask;
            bool any = false;
            if (mask) any = std::any_of(mask, mask + npix, [](uint8_t v) { return v != 0; });
            if (any) {
                d_mask.alloc(size_t(npix));
                DG_CUDA(cudaMemcpyAsync(d_mask.ptr, mask, size_t(npix), cudaMemcpyHostToDevice, s));
            }
            dg::compact_table(built.full, any ? d_mask.ptr : nullptr, int32_t(npix), s, plan->table);
            dg::make_gather_table(plan->table, built.norm.ptr, dim1, dim2,
                                  n_azimuthal ? kStripRows2d : kStripRows, s, plan->gather);
            if (method->flags & DG_PLAN_FLIP_VERTICAL) dg::flip_gather_rows(plan->gather, dim1, dim2, s);
            DG_CUDA(cudaEventRecord(e1, s));
            DG_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            DG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            plan->build_ms = ms;
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        plan->hist_min = built.hist_min;
        plan->hist_step = built.hist_step;
        plan->guard_corners = built.guard_corners;
        plan->singular_pixels = built.singular_pixels;
        plan->full_entries = built.full.nnz;
        plan->radial = built.radial_centres;
        plan->azimuthal = built.azimuthal_centres;
        plan->norm = std::move(built.norm);
        if (method->flags & DG_PLAN_KEEP_TABLES) plan->full = std::move(built.full);
        // Chunk budget (src/integration/cuda.rs:137-158): min(1 GiB, free/2)
        // unless given; one frame costs pixels * 8 (f64 worst case) plus its
        // outputs.
        size_t free_b = 0, total_b = 0;
        DG_CUDA(cudaMemGetInfo(&free_b, &total_b));
        int64_t budget = method->max_batch_bytes > 0
                             ? method->max_batch_bytes
                             : std::min<int64_t>(int64_t(1) << 30, int64_t(free_b / 2));
        int64_t per_frame = int64_t(dim1) * dim2 * 8 + plan->n_bins * 24;
        plan->max_batch_frames = budget / per_frame;
        if (plan->max_batch_frames < 1) {
            if (method->max_batch_bytes > 0)
                dg::fail(DG_INVALID_INPUT, "max_batch_bytes is smaller than one frame");
            dg::fail(DG_DEVICE, "not enough free device memory for one frame");
        }
        *out = plan.release();
    });
}

dg_status dg_plan_destroy(dg_plan *plan) {
    return guarded([&] {
        if (!plan) return;
        {
            std::lock_guard<std::mutex> lock(plan->mu);
            int prev = -1;
            cudaGetDevice(&prev);
            cudaSetDevice(plan->device);
            if (plan->stream) cudaStreamSynchronize(plan->stream);
            plan->full = dg::DeviceCsr();
            plan->table = dg::DeviceCsr();
            plan->norm.release();
            plan->gather = dg::GatherTable();
            plan->stage_in.release();
            plan->stage_out.release();
            plan->stage_mask.release();
            dg::bslz4_release(plan);
            if (plan->stream) cudaStreamDestroy(plan->stream);
            plan->stream = nullptr;
            if (prev >= 0) cudaSetDevice(prev);
        }
        delete plan;
    });
}

dg_status dg_plan_query(const dg_plan *plan, dg_plan_info *out) {
    return guarded([&] {
        if (!plan || !out) dg::fail(DG_INVALID_INPUT, "plan and out must not be NULL");
        std::memset(out, 0, sizeof *out);
        out->dim1 = plan->dim1;
        out->dim2 = plan->dim2;
        out->n_radial = plan->n_radial;
        out->n_azimuthal = plan->n_azimuthal;
        out->table_entries = plan->table.nnz;
        out->full_entries = plan->full_entries;
        out->max_batch_frames = plan->max_batch_frames;
        out->device = plan->device;
        out->precision = plan->method.precision;
        out->hist_min = plan->hist_min;
        out->hist_step = plan->hist_step;
        out->build_ms = plan->build_ms;
        out->device_bytes = plan->device_bytes();
        out->guard_corners = plan->guard_corners;
        out->singular_pixels = plan->singular_pixels;
    });
}

dg_status dg_plan_radial(const dg_plan *plan, double *out, int64_t n) {
    return guarded([&] {
        if (!plan || !out) dg::fail(DG_INVALID_INPUT, "plan and out must not be NULL");
        if (n != int64_t(plan->radial.size()))
            dg::fail(DG_INVALID_INPUT, "radial axis has " + std::to_string(plan->radial.size()) +
                                           " values");
        std::copy(plan->radial.begin(), plan->radial.end(), out);
    });
}

dg_status dg_plan_azimuthal(const dg_plan *plan, double *out, int64_t n) {
    return guarded([&] {
        if (!plan || !out) dg::fail(DG_INVALID_INPUT, "plan and out must not be NULL");
        if (n != int64_t(plan->azimuthal.size()))
            dg::fail(DG_INVALID_INPUT, "azimuthal axis has " +
                                           std::to_string(plan->azimuthal.size()) + " values");
        std::copy(plan->azimuthal.begin(), plan->azimuthal.end(), out);
    });
}

dg_status dg_plan_export_table(const dg_plan *cplan, int32_t which, int64_t *row_ptr,
                               int32_t *col, double *weight, double *denominator) {
    return guarded([&] {
        if (!cplan) dg::fail(DG_INVALID_INPUT, "plan must not be NULL");
        dg_plan *plan = const_cast<dg_plan *>(cplan);
        std::lock_guard<std::mutex> lock(plan->mu);
        const dg::DeviceCsr *t = nullptr;
        if (which == 0) t = &plan->table;
        else if (which == 1) {
            if (!plan->full.row_ptr.ptr)
                dg::fail(DG_INVALID_INPUT, "the unmasked table needs DG_PLAN_KEEP_TABLES");
            t = &plan->full;
        } else dg::fail(DG_INVALID_INPUT, "which must be 0 or 1");
        DeviceScope scope(plan->device);
        cudaStream_t s = plan->stream;
        if (row_ptr)
            DG_CUDA(cudaMemcpyAsync(row_ptr, t->row_ptr.ptr, size_t(t->n_rows + 1) * 8,
                                    cudaMemcpyDeviceToHost, s));
        if (col && t->nnz)
            DG_CUDA(cudaMemcpyAsync(col, t->col.ptr, size_t(t->nnz) * 4, cudaMemcpyDeviceToHost, s));
        if (weight && t->nnz)
            DG_CUDA(cudaMemcpyAsync(weight, t->w.ptr, size_t(t->nnz) * 8, cudaMemcpyDeviceToHost, s));
        if (denominator) {
            if (which != 0) dg::fail(DG_INVALID_INPUT, "denominators exist for the masked table");
            DG_CUDA(cudaMemcpyAsync(denominator, plan->gather.den.ptr, size_t(t->n_rows) * 8,
                                    cudaMemcpyDeviceToHost, s));
        }
        DG_CUDA(cudaStreamSynchronize(s));
    });
}

dg_status dg_integrate_device(dg_plan *plan, const void *d_frames, int32_t dtype,
                              int64_t n_frames, uint32_t flags, double *d_i, double *d_s,
                              double *d_d, void *stream) {
    return guarded([&] {
        check_frames(plan, d_frames, dtype, n_frames, flags, d_i, d_s, d_d);
        if (n_frames == 0) return;
        check_device_alignment(d_frames, dtype, d_i, d_s, d_d);
        std::lock_guard<std::mutex> lock(plan->mu);
        DeviceScope scope(plan->device);
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : plan->stream;
        dg::run_gather(plan->gather, d_frames, dtype, int64_t(plan->dim1) * plan->dim2, n_frames,
                       flags, plan->method.precision, d_i, (flags & DG_ERRORS) ? d_s : nullptr,
                       (flags & DG_AZIMUTHAL_STD) ? d_d : nullptr, s);
    });
}

// Allocation-free integration: the partial sums go to the library's fixed
// device array (dg::noalloc_scratch) instead of the plan's own, so nothing is
// allocated once the plan exists. Every call on a device shares that array
// and leaves its contents behind; calls that overlap on the GPU race on it.
// Each launch's partial sums are written by its gather before its finalize
// reads them, so nothing needs clearing between calls.
dg_status dg_integrate_device_noalloc(dg_plan *plan, const void *d_frames, int32_t dtype,
                                      int64_t n_frames, uint32_t flags, double *d_i, double *d_s,
                                      double *d_d, void *stream) {
    return guarded([&] {
        check_frames(plan, d_frames, dtype, n_frames, flags, d_i, d_s, d_d);
        if (n_frames == 0) return;
        check_device_alignment(d_frames, dtype, d_i, d_s, d_d);
        std::lock_guard<std::mutex> lock(plan->mu);
        DeviceScope scope(plan->device);
        size_t cap = 0;
        double *scratch = dg::noalloc_scratch(&cap);
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : plan->stream;
        dg::run_gather(plan->gather, d_frames, dtype, int64_t(plan->dim1) * plan->dim2, n_frames,
                       flags, plan->method.precision, d_i, (flags & DG_ERRORS) ? d_s : nullptr,
                       (flags & DG_AZIMUTHAL_STD) ? d_d : nullptr, s, scratch, cap);
    });
}

dg_status dg_integrate_device_plain(dg_plan *plan, const void *d_frames, int32_t dtype,
                                    int64_t n_frames, uint32_t flags, double *d_i, double *d_s,
                                    double *d_d, void *stream) {
    return guarded([&] {
        check_frames(plan, d_frames, dtype, n_frames, flags, d_i, d_s, d_d);
        if (n_frames == 0) return;
        check_device_alignment(d_frames, dtype, d_i, d_s, d_d);
        std::lock_guard<std::mutex> lock(plan->mu);
        DeviceScope scope(plan->device);
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : plan->stream;
        const int64_t npix = int64_t(plan->dim1) * plan->dim2;
        const size_t es = dtype_size(dtype);
        const int64_t nb = plan->n_bins;
        for (int64_t f = 0; f < n_frames; ++f) {
            const void *fp = static_cast<const unsigned char *>(d_frames) + f * npix * es;
            dg::run_gather(plan->gather, fp, dtype, npix, 1, flags, plan->method.precision,
                           d_i + f * nb, (flags & DG_ERRORS) ? d_s + f * nb : nullptr,
                           (flags & DG_AZIMUTHAL_STD) ? d_d + f * nb : nullptr, s);
        }
    });
}

dg_status dg_plan_test_wait_timeout(dg_plan *plan, const void *d_frames, int32_t dtype,
                                    int64_t n_frames, uint32_t flags, double *d_i, double *d_s,
                                    double *d_d) {
    return guarded([&] {
        check_frames(plan, d_frames, dtype, n_frames, flags, d_i, d_s, d_d);
        if (n_frames == 0) dg::fail(DG_INVALID_INPUT, "the check needs at least one frame");
        check_device_alignment(d_frames, dtype, d_i, d_s, d_d);
        std::lock_guard<std::mutex> lock(plan->mu);
        DeviceScope scope(plan->device);
        if (!dg::gather_variant_needs_tiles(plan->gather.variant))
            dg::fail(DG_UNSUPPORTED, "the plan's gather lane mapping has no chunk pipeline "
                                     "(select mapping 7 or 8)");
        cudaStream_t s = plan->stream;
        dg::check_bin_tile_waits(plan->gather);  // report an earlier failure as itself
        plan->gather.withhold_test = 1;
        try {
            dg::run_gather(plan->gather, d_frames, dtype, int64_t(plan->dim1) * plan->dim2,
                           n_frames, flags, plan->method.precision, d_i,
                           (flags & DG_ERRORS) ? d_s : nullptr,
                           (flags & DG_AZIMUTHAL_STD) ? d_d : nullptr, s);
        } catch (...) {
            plan->gather.withhold_test = 0;
            throw;
        }
        plan->gather.withhold_test = 0;
        DG_CUDA(cudaStreamSynchronize(s));
        dg::check_bin_tile_waits(plan->gather);
    });
}

namespace {

// Arguments of the per-frame-mask and raw-sum calls.
void check_masked(const dg_plan *plan, const void *frames, int32_t dtype, int64_t n_frames,
                  const void *masks, int64_t mask_stride, uint32_t flags, bool raw,
                  const void *o0, const void *o1, const void *o2, const void *o3) {
    using dg::fail;
    if (!plan) fail(DG_INVALID_INPUT, "plan must not be NULL");
    (void)dtype_size(dtype);
    if (n_frames < 0) fail(DG_INVALID_INPUT, "frame count must not be negative");
    if (flags & DG_AZIMUTHAL_STD)
        fail(DG_UNSUPPORTED, "azimuthal_std is not available with per-frame masks or raw sums");
    if (flags & ~DG_ERRORS) fail(DG_INVALID_INPUT, "unknown flags");
    if (!raw && !masks) fail(DG_INVALID_INPUT, "per-frame masks must not be NULL");
    const int64_t npix = int64_t(plan->dim1) * plan->dim2;
    if (mask_stride < 0 || (mask_stride != 0 && mask_stride < npix))
        fail(DG_INVALID_INPUT, "mask_stride must be 0 (one mask for every frame) or at least the "
                               "frame's " + std::to_string(npix) + " pixels");
    if (n_frames == 0) return;
    if (!frames) fail(DG_INVALID_INPUT, "frames must not be NULL");
    if (!o0) fail(DG_INVALID_INPUT, raw ? "signal output must not be NULL"
                                        : "intensity output must not be NULL");
    if (raw) {
        if (!o1 || !o3) fail(DG_INVALID_INPUT, "norm and count outputs must not be NULL");
        if ((flags & DG_ERRORS) && !o2) fail(DG_INVALID_INPUT, "variance requested without an output");
    } else if ((flags & DG_ERRORS) && !o1) {
        fail(DG_INVALID_INPUT, "errors requested without an output");
    }
}

// Runs the n_chunks chunks of a host-memory call through two staging slots
// (one when there is a single chunk): copy_in(k, slot, cs) queues chunk k's
// host-to-device copies on the plan's copy stream, gather(k, slot, s) its
// kernels on the plan's stream and results(k, s) the copies of its results
// back. Chunk k + 1's copies are queued before chunk k's gather, and a slot
// is copied into again only once the gather that read it has run, so the
// host link never waits for a gather. On an error nothing of the call stays
// in flight (queued copies read the caller's buffers until they complete).
extern "C++" {  // a template inside the C-ABI block
template <class CopyIn, class Gather, class Results>
void run_two_slots(dg_plan *plan, int64_t n_chunks, CopyIn copy_in, Gather gather,
                   Results results) {
    cudaStream_t s = plan->stream;
    dg::ensure_copy_pipeline(plan);
    cudaStream_t cs = plan->copy_stream;
    cudaEvent_t *copied = plan->bs_copied, *consumed = plan->bs_decoded;
    const int n_slots = n_chunks > 1 ? 2 : 1;
    struct Drain {
        cudaStream_t a, b;
        bool done = false;
        ~Drain() {
            if (!done) {
                cudaStreamSynchronize(a);
                cudaStreamSynchronize(b);
            }
        }
    } drain{cs, s};
    // the copy stream starts after everything already queued on the plan
    DG_CUDA(cudaEventRecord(consumed[0], s));
    DG_CUDA(cudaStreamWaitEvent(cs, consumed[0], 0));
    auto issue = [&](int64_t k) {
        const int slot = int(k % n_slots);
        if (k >= n_slots) DG_CUDA(cudaStreamWaitEvent(cs, consumed[slot], 0));
        copy_in(k, slot, cs);
        DG_CUDA(cudaEventRecord(copied[slot], cs));
    };
    issue(0);
    for (int64_t k = 0; k < n_chunks; ++k) {
        const int slot = int(k % n_slots);
        DG_CUDA(cudaStreamWaitEvent(s, copied[slot], 0));
        if (k + 1 < n_chunks) issue(k + 1);
        gather(k, slot, s);
        DG_CUDA(cudaEventRecord(consumed[slot], s));
        results(k, s);
    }
    DG_CUDA(cudaStreamSynchronize(s));
    drain.done = true;
}
}  // extern "C++"

// Host-memory form of the masked / raw calls: frames, masks and results
// staged through the plan's buffers in chunks, two slots (run_two_slots).
void run_masked_host(dg_plan *plan, const void *frames, int32_t dtype, int64_t n_frames,
                     const uint8_t *masks, int64_t mask_stride, uint32_t flags, bool raw,
                     double *o0, double *o1, double *o2, double *o3) {
    std::lock_guard<std::mutex> lock(plan->mu);
    DeviceScope scope(plan->device);
    cudaStream_t s = plan->stream;
    const int64_t npix = int64_t(plan->dim1) * plan->dim2;
    const size_t es = dtype_size(dtype);
    const int64_t nb = plan->n_bins;
    // Two staging slots of frames (and of per-frame masks), as in
    // dg_integrate: chunk k + 1 is copied on the copy stream while chunk k is
    // gathered. Two slots of max_batch_frames frames fit the chunk budget
    // (8 bytes a pixel) while a frame and its mask take at most 4 bytes a
    // pixel; otherwise each slot holds half as many.
    const size_t per_px = es + ((masks && mask_stride) ? 1 : 0);
    const int64_t per_slot =
        std::max<int64_t>(1, per_px <= 4 ? plan->max_batch_frames : plan->max_batch_frames / 2);
    const int64_t chunk = std::min<int64_t>(per_slot, n_frames);
    const int64_t n_chunks = (n_frames + chunk - 1) / chunk;
    const int n_slots = n_chunks > 1 ? 2 : 1;
    const size_t slot_bytes = (size_t(chunk * npix) * es + 255) / 256 * 256;
    const int nout = raw ? 4 : 2;
    if (plan->stage_in.count < n_slots * slot_bytes) {
        plan->stage_in.release();
        plan->stage_in.alloc(n_slots * slot_bytes);
    }
    if (plan->stage_out.count < size_t(chunk * nb * nout)) {
        plan->stage_out.release();
        plan->stage_out.alloc(size_t(chunk * nb * nout));
    }
    // per-frame masks: a slot of chunk rows each; one plan-wide mask: one row
    const size_t mask_slot = (masks && mask_stride) ? (size_t(chunk * npix) + 255) / 256 * 256 : 0;
    const size_t mask_bytes = masks ? (mask_stride ? n_slots * mask_slot : size_t(npix)) : 0;
    if (plan->stage_mask.count < mask_bytes) {
        plan->stage_mask.release();
        plan->stage_mask.alloc(mask_bytes);
    }
    dg::prepare_raw(plan->gather, plan->table, plan->norm.ptr, s);
    if (masks && !mask_stride)
        DG_CUDA(cudaMemcpyAsync(plan->stage_mask.ptr, masks, size_t(npix), cudaMemcpyHostToDevice, s));
    const bool used[4] = {true, raw || (flags & DG_ERRORS), raw && (flags & DG_ERRORS), raw};
    double *const h[4] = {o0, o1, o2, o3};
    auto frames_of = [&](int64_t k) { return std::min<int64_t>(chunk, n_frames - k * chunk); };
    run_two_slots(
        plan, n_chunks,
        [&](int64_t k, int slot, cudaStream_t cs) {
            const int64_t f0 = k * chunk, nf = frames_of(k);
            DG_CUDA(cudaMemcpyAsync(plan->stage_in.ptr + slot * slot_bytes,
                                    static_cast<const unsigned char *>(frames) + f0 * npix * es,
                                    size_t(nf * npix) * es, cudaMemcpyHostToDevice, cs));
            if (masks && mask_stride)
                DG_CUDA(cudaMemcpy2DAsync(plan->stage_mask.ptr + slot * mask_slot, size_t(npix),
                                          masks + f0 * mask_stride, size_t(mask_stride),
                                          size_t(npix), size_t(nf), cudaMemcpyHostToDevice, cs));
        },
        [&](int64_t k, int slot, cudaStream_t gs) {
            const int64_t nf = frames_of(k);
            double *d[4];
            for (int q = 0; q < 4; ++q) d[q] = plan->stage_out.ptr + q * nf * nb;
            const uint8_t *dm =
                masks ? plan->stage_mask.ptr + (mask_stride ? slot * mask_slot : 0) : nullptr;
            dg::run_gather_raw(plan->gather, plan->stage_in.ptr + slot * slot_bytes, dtype, npix,
                               nf, dm, mask_stride ? npix : 0, flags, raw, d[0],
                               used[1] ? d[1] : nullptr, used[2] ? d[2] : nullptr,
                               used[3] ? d[3] : nullptr, gs);
        },
        [&](int64_t k, cudaStream_t gs) {
            const int64_t f0 = k * chunk, nf = frames_of(k);
            for (int q = 0; q < 4; ++q)
                if (used[q])
                    DG_CUDA(cudaMemcpyAsync(h[q] + f0 * nb, plan->stage_out.ptr + q * nf * nb,
                                            size_t(nf * nb) * 8, cudaMemcpyDeviceToHost, gs));
        });
}

}  // namespace

dg_status dg_integrate_dynamic(dg_plan *plan, const void *frames, int32_t dtype, int64_t n_frames,
                               const uint8_t *masks, int64_t mask_stride, uint32_t flags,
                               double *out_intensity, double *out_sigma) {
    return guarded([&] {
        check_masked(plan, frames, dtype, n_frames, masks, mask_stride, flags, false,
                     out_intensity, out_sigma, nullptr, nullptr);
        if (n_frames == 0) return;
        run_masked_host(plan, frames, dtype, n_frames, masks, mask_stride, flags, false,
                        out_intensity, out_sigma, nullptr, nullptr);
    });
}

dg_status dg_integrate_dynamic_device(dg_plan *plan, const void *d_frames, int32_t dtype,
                                      int64_t n_frames, const uint8_t *d_masks,
                                      int64_t mask_stride, uint32_t flags, double *d_i,
                                      double *d_s, void *stream) {
    return guarded([&] {
        check_masked(plan, d_frames, dtype, n_frames, d_masks, mask_stride, flags, false, d_i,
                     d_s, nullptr, nullptr);
        if (n_frames == 0) return;
        check_device_alignment(d_frames, dtype, d_i, d_s, nullptr);
        std::lock_guard<std::mutex> lock(plan->mu);
        DeviceScope scope(plan->device);
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : plan->stream;
        dg::prepare_raw(plan->gather, plan->table, plan->norm.ptr, s);
        dg::run_gather_raw(plan->gather, d_frames, dtype, int64_t(plan->dim1) * plan->dim2,
                           n_frames, d_masks, mask_stride, flags, false, d_i,
                           (flags & DG_ERRORS) ? d_s : nullptr, nullptr, nullptr, s);
    });
}

dg_status dg_integrate_raw(dg_plan *plan, const void *frames, int32_t dtype, int64_t n_frames,
                           const uint8_t *masks, int64_t mask_stride, uint32_t flags,
                           double *out_signal, double *out_norm, double *out_variance,
                           double *out_count) {
    return guarded([&] {
        check_masked(plan, frames, dtype, n_frames, masks, mask_stride, flags, true, out_signal,
                     out_norm, out_variance, out_count);
        if (n_frames == 0) return;
        run_masked_host(plan, frames, dtype, n_frames, masks, mask_stride, flags, true,
                        out_signal, out_norm, out_variance, out_count);
    });
}

dg_status dg_integrate_raw_device(dg_plan *plan, const void *d_frames, int32_t dtype,
                                  int64_t n_frames, const uint8_t *d_masks, int64_t mask_stride,
                                  uint32_t flags, double *d_signal, double *d_norm,
                                  double *d_variance, double *d_count, void *stream) {
    return guarded([&] {
        check_masked(plan, d_frames, dtype, n_frames, d_masks, mask_stride, flags, true,
                     d_signal, d_norm, d_variance, d_count);
        if (n_frames == 0) return;
        check_device_alignment(d_frames, dtype, d_signal, d_norm, d_count);
        check_device_alignment(d_frames, dtype, d_variance, nullptr, nullptr);
        std::lock_guard<std::mutex> lock(plan->mu);
        DeviceScope scope(plan->device);
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : plan->stream;
        dg::prepare_raw(plan->gather, plan->table, plan->norm.ptr, s);
        dg::run_gather_raw(plan->gather, d_frames, dtype, int64_t(plan->dim1) * plan->dim2,
                           n_frames, d_masks, mask_stride, flags, true, d_signal, d_norm,
                           (flags & DG_ERRORS) ? d_variance : nullptr, d_count, s);
    });
}

dg_status dg_host_alloc(int32_t device, int64_t bytes, void **out) {
    return guarded([&] {
        if (!out) dg::fail(DG_INVALID_INPUT, "out must not be NULL");
        *out = nullptr;
        if (bytes <= 0) dg::fail(DG_INVALID_INPUT, "pinned allocation size must be positive");
        check_device(device);
        DeviceScope scope(device);
        void *p = nullptr;
        const cudaError_t e = cudaHostAlloc(&p, size_t(bytes), cudaHostAllocPortable);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            dg::fail(DG_DEVICE, "pinned host allocation of " + std::to_string(bytes) +
                                    " bytes failed: " + cudaGetErrorString(e));
        }
        *out = p;
    });
}

dg_status dg_host_free(void *ptr) {
    return guarded([&] {
        if (ptr) DG_CUDA(cudaFreeHost(ptr));
    });
}

int32_t dg_host_is_pinned(const void *ptr) {
    if (!ptr) return 0;
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, ptr);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    return a.type == cudaMemoryTypeHost ? 1 : 0;
}

dg_status dg_integrate(dg_plan *plan, const void *frames, int32_t dtype, int64_t n_frames,
                       uint32_t flags, double *oi, double *os, double *od) {
    return guarded([&] {
        check_frames(plan, frames, dtype, n_frames, flags, oi, os, od);
        if (n_frames == 0) return;
        std::lock_guard<std::mutex> lock(plan->mu);
        DeviceScope scope(plan->device);
        const int64_t npix = int64_t(plan->dim1) * plan->dim2;
        const size_t es = dtype_size(dtype);
        const int64_t nb = plan->n_bins;
        // Two staging slots: chunk k + 1's frames cross the host link on the
        // copy stream while the plan's stream gathers chunk k and returns its
        // results, so the link never waits for a gather. The chunk budget
        // counts 8 bytes a pixel, so two slots of max_batch_frames frames of
        // at most 4-byte pixels fit it; 8-byte pixels take half as many.
        const int64_t per_slot =
            std::max<int64_t>(1, es <= 4 ? plan->max_batch_frames : plan->max_batch_frames / 2);
        const int64_t chunk = std::min<int64_t>(per_slot, n_frames);
        const int64_t n_chunks = (n_frames + chunk - 1) / chunk;
        const int n_slots = n_chunks > 1 ? 2 : 1;
        const size_t slot_bytes = (size_t(chunk * npix) * es + 255) / 256 * 256;
        const int nout = 1 + ((flags & DG_ERRORS) ? 1 : 0) + ((flags & DG_AZIMUTHAL_STD) ? 1 : 0);
        if (plan->stage_in.count < n_slots * slot_bytes) {
            plan->stage_in.release();
            plan->stage_in.alloc(n_slots * slot_bytes);
        }
        if (plan->stage_out.count < size_t(chunk * nb * nout)) {
            plan->stage_out.release();
            plan->stage_out.alloc(size_t(chunk * nb * nout));
        }
        auto frames_of = [&](int64_t k) { return std::min<int64_t>(chunk, n_frames - k * chunk); };
        auto outs = [&](int64_t k, double **d) {
            const int64_t nf = frames_of(k);
            d[0] = plan->stage_out.ptr;
            d[1] = (flags & DG_ERRORS) ? d[0] + nf * nb : nullptr;
            d[2] = (flags & DG_AZIMUTHAL_STD) ? d[0] + nf * nb * (d[1] ? 2 : 1) : nullptr;
        };
        run_two_slots(
            plan, n_chunks,
            [&](int64_t k, int slot, cudaStream_t cs) {
                DG_CUDA(cudaMemcpyAsync(plan->stage_in.ptr + slot * slot_bytes,
                                        static_cast<const unsigned char *>(frames) +
                                            k * chunk * npix * es,
                                        size_t(frames_of(k) * npix) * es, cudaMemcpyHostToDevice,
                                        cs));
            },
            [&](int64_t k, int slot, cudaStream_t gs) {
                double *d[3];
                outs(k, d);
                dg::run_gather(plan->gather, plan->stage_in.ptr + slot * slot_bytes, dtype, npix,
                               frames_of(k), flags, plan->method.precision, d[0], d[1], d[2], gs);
            },
            [&](int64_t k, cudaStream_t gs) {
                double *d[3];
                outs(k, d);
                double *const h[3] = {oi, os, od};
                const int64_t f0 = k * chunk, nf = frames_of(k);
                for (int q = 0; q < 3; ++q)
                    if (d[q])
                        DG_CUDA(cudaMemcpyAsync(h[q] + f0 * nb, d[q], size_t(nf * nb) * 8,
                                                cudaMemcpyDeviceToHost, gs));
            });
        dg::check_bin_tile_waits(plan->gather);
    });
}

dg_status dg_plan_profile(dg_plan *plan, int32_t enable) {
    return guarded([&] {
        if (!plan) dg::fail(DG_INVALID_INPUT, "plan must not be NULL");
        std::lock_guard<std::mutex> lock(plan->mu);
        plan->gather.profile = enable != 0;
    });
}

dg_status dg_plan_kernel_time(dg_plan *plan, int32_t reset, double *gather_ms,
                              int64_t *gather_launches, int64_t *launches) {
    return guarded([&] {
        if (!plan) dg::fail(DG_INVALID_INPUT, "plan must not be NULL");
        std::lock_guard<std::mutex> lock(plan->mu);
        DeviceScope scope(plan->device);
        dg::gather_kernel_time(plan->gather, reset != 0, gather_ms, gather_launches, launches);
    });
}

dg_status dg_plan_autotune(dg_plan *plan, const void *d_frames, int32_t dtype, int64_t n_frames,
                           uint32_t flags, void *stream, int32_t *variant, double *ms,
                           int32_t n_ms) {
    return guarded([&] {
        if (!plan) dg::fail(DG_INVALID_INPUT, "plan must not be NULL");
        if (flags & ~uint32_t(DG_ERRORS | DG_AZIMUTHAL_STD)) dg::fail(DG_INVALID_INPUT, "unknown flags");
        if (n_frames <= 0 || !d_frames)
            dg::fail(DG_INVALID_INPUT, "autotuning needs device frames (n_frames >= 1)");
        if ((flags & DG_AZIMUTHAL_STD) && plan->n_azimuthal != 0)
            dg::fail(DG_UNSUPPORTED, "azimuthal_std is defined for 1D tables only");
        check_device_alignment(d_frames, dtype, nullptr, nullptr, nullptr);
        std::lock_guard<std::mutex> lock(plan->mu);
        DeviceScope scope(plan->device);
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : plan->stream;
        // bin tiles pay off only when a launch fills the GPU
        for (int v : {7, 8})
            if (dg::bin_tiles_fill_gpu(plan->gather, v, n_frames))
                dg::ensure_bin_tiles(plan->gather, plan->table, v, s);
        std::vector<double> each;
        const int v = dg::autotune_gather(plan->gather, d_frames, dtype,
                                          int64_t(plan->dim1) * plan->dim2, n_frames, flags, s,
                                          &each);
        if (variant) *variant = v;
        for (int32_t i = 0; ms && i < n_ms && size_t(i) < each.size(); ++i) ms[i] = each[size_t(i)];
    });
}

dg_status dg_plan_variant(dg_plan *plan, int32_t set, int32_t *current, int32_t *count) {
    return guarded([&] {
        if (!plan) dg::fail(DG_INVALID_INPUT, "plan must not be NULL");
        std::lock_guard<std::mutex> lock(plan->mu);
        if (set >= dg::gather_variant_count())
            dg::fail(DG_INVALID_INPUT, "gather mapping " + std::to_string(set) + " does not exist");
        if (set >= 0 && dg::gather_variant_needs_tiles(set)) {
            DeviceScope scope(plan->device);
            dg::ensure_bin_tiles(plan->gather, plan->table, set, plan->stream);
        }
        if (set >= 0 && !dg::gather_variant_available(plan->gather, set))
            dg::fail(DG_UNSUPPORTED, "gather mapping " + std::to_string(set) +
                                         " is not available for this plan");
        if (set >= 0) plan->gather.variant = set;
        if (current) *current = plan->gather.variant;
        if (count) *count = dg::gather_variant_count();
    });
}

dg_status dg_eval_math(int32_t which, const double *d_a, const double *d_b, int64_t n,
                       double *d_out) {
    return guarded([&] {
        if (n < 0) dg::fail(DG_INVALID_INPUT, "n must not be negative");
        if (n > 0 && (!d_a || !d_out || ((which == 0 || which == 2) && !d_b)))
            dg::fail(DG_INVALID_INPUT, "arrays must not be NULL");
        cudaStream_t s = nullptr;
        DG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            dg::eval_math(which, d_a, d_b, n, d_out, s);
            DG_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        cudaStreamDestroy(s);
    });
}

dg_status dg_device_info_get(int32_t device, dg_device_info *out) {
    return guarded([&] {
        if (!out) dg::fail(DG_INVALID_INPUT, "out must not be NULL");
        std::memset(out, 0, sizeof *out);
        out->device = device;
        check_device(device);
        cudaDeviceProp p{};
        DG_CUDA(cudaGetDeviceProperties(&p, device));
        out->available = 1;
        out->cc_major = p.major;
        out->cc_minor = p.minor;
        out->sm_count = p.multiProcessorCount;
        out->total_memory_bytes = int64_t(p.totalGlobalMem);
        int v = 0;
        cudaDriverGetVersion(&v);
        out->driver_version = v;
        std::strncpy(out->name, p.name, sizeof(out->name) - 1);
    });
}

int32_t dg_last_error(char *buf, size_t len) {
    const std::string &m = g_last_error;
    if (buf && len) {
        size_t n = std::min(len - 1, m.size());
        std::memcpy(buf, m.data(), n);
        buf[n] = 0;
    }
    return int32_t(m.size());
}

}  // extern "C"
