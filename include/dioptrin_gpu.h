/*
 * dioptrin_gpu.h — C ABI of the B200 lookup-table integration library.
 *
 * Plain pointers and sizes only. A plan is the device-resident snapshot of
 * one integrator configuration (geometry, method, unit, radial range,
 * polarisation, mask) for one image shape and bin count: its CSR table is
 * built on the GPU and kept in HBM until the plan is destroyed.
 *
 * Each entry point names the reference interface it replaces
 * (paths are inside the reference crate, CPrescher/Dioptrin v0.20.1).
 */
#ifndef DIOPTRIN_GPU_H
#define DIOPTRIN_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DG_EXPORT __attribute__((visibility("default")))
#else
#define DG_EXPORT
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: the five CudaError variants (src/integration/cuda.rs:218-237)
 * plus a timeout for the request loop's bounded waits. */
typedef enum dg_status {
    DG_OK = 0,
    DG_NOT_COMPILED = 1, /* CudaError::NotCompiled */
    DG_UNAVAILABLE = 2,  /* CudaError::Unavailable: no device / no such ordinal */
    DG_UNSUPPORTED = 3,  /* CudaError::Unsupported: method, mask mode, table size */
    DG_INVALID_INPUT = 4,/* CudaError::InvalidInput: shapes, sizes, budgets */
    DG_DEVICE = 5,       /* CudaError::Device: driver error, out of memory */
    DG_TIMEOUT = 6       /* a bounded wait expired (request loop, device spin) */
} dg_status;

/* IntegrationMethod (src/integration.rs:222-236). */
enum {
    DG_METHOD_COUNTING = 0,
    DG_METHOD_PIXEL_SPLIT = 1,
    DG_METHOD_PYFAI_FULL = 2,
    DG_METHOD_SUPERSAMPLED = 3
};

/* RadialUnit (src/integration.rs:115-128). */
enum { DG_UNIT_TTH_RAD = 0, DG_UNIT_TTH_DEG = 1, DG_UNIT_Q_A = 2, DG_UNIT_Q_NM = 3 };

/* Pixel types a plan accepts (CudaPixel, src/integration/cuda.rs:354-367). */
enum { DG_U16 = 0, DG_U32 = 1, DG_I32 = 2, DG_F32 = 3, DG_F64 = 4 };

/* CudaPrecision (src/integration/cuda.rs:64-73). Weights are stored in FP32
 * in every mode; F32_COMPENSATED accumulates with double-word FP32 sums, F64
 * accumulates in FP64. */
enum { DG_PRECISION_F32 = 0, DG_PRECISION_F32_COMPENSATED = 1, DG_PRECISION_F64 = 2 };

/* Integration flags. */
#define DG_ERRORS 1u        /* propagated Poisson sigma (integrate1d_with_errors) */
#define DG_AZIMUTHAL_STD 2u /* weighted population spread (integrate1d_with_azimuthal_std) */
/* dg_server_submit only: the frame is not copied at submission; it must stay
 * valid and unchanged until the request completes (dg_server_poll), and is
 * copied to the device straight from the caller's memory (page-locked memory
 * from dg_host_alloc gives an asynchronous DMA). */
#define DG_SUBMIT_BORROW 256u

/* Plan-creation flags. */
#define DG_PLAN_KEEP_TABLES 1u /* keep the unmasked f64 CSR for dg_plan_export_table */
/* InputOrder::FlipVertical (src/integration/fixed.rs:18-23, applied to the
 * uploaded columns as in src/integration/cuda/device.rs:506-528): frames
 * arrive bottom row first (top-to-bottom raw HDF5 frames); the plan's pixel
 * indices are remapped once at creation, so results equal those of the
 * row-flipped frames in detector order, bit for bit. Per-frame masks follow
 * the frames' order; the plan mask, exported tables and radial axes stay in
 * detector order. */
#define DG_PLAN_FLIP_VERTICAL 2u

/* Poni (src/poni.rs:13-24); SI units, angles in radians. */
typedef struct dg_geometry {
    double pixel1, pixel2, distance, poni1, poni2, rot1, rot2, rot3, wavelength;
} dg_geometry;

/* Integrator configuration captured by a plan (src/integration.rs:278-297,
 * Cuda1dOptions src/integration/cuda.rs:118-211). */
typedef struct dg_method {
    int32_t kind;              /* DG_METHOD_* */
    int32_t n_ss;              /* subpixels per side for DG_METHOD_SUPERSAMPLED */
    int32_t unit;              /* DG_UNIT_* */
    int32_t has_polarization;  /* with_polarization_factor was called */
    double polarization_factor;
    int32_t has_radial_range;  /* with_radial_range */
    double radial_min, radial_max;
    int32_t precision;         /* DG_PRECISION_* */
    int32_t device;            /* CUDA ordinal */
    int64_t max_batch_bytes;   /* chunk budget for host-memory calls; 0 = automatic */
    uint32_t flags;            /* DG_PLAN_* */
} dg_method;

typedef struct dg_plan dg_plan;

/* Replaces Integrator::prepare_cuda1d (src/integration/cuda.rs:1089-1103) and
 * prepare_cuda2d (:1111-1157). n_azimuthal == 0 selects 1D. azimuthal_range is
 * NULL or two doubles (radians). mask is NULL or dim1*dim2 bytes, nonzero =
 * masked (src/mask.rs:4-9). Checks run in the reference's order
 * (src/integration/cuda.rs:1071-1088): configuration, shape, device, build. */
DG_EXPORT dg_status dg_plan_create(const dg_geometry *geometry, const dg_method *method,
                         const uint8_t *mask, int32_t dim1, int32_t dim2, int32_t n_radial,
                         int32_t n_azimuthal, const double *azimuthal_range, dg_plan **out);

/* Replaces Drop for Cuda1dPlan (src/integration/cuda.rs:374-386). NULL is a no-op. */
DG_EXPORT dg_status dg_plan_destroy(dg_plan *plan);

typedef struct dg_plan_info {
    int32_t dim1, dim2, n_radial, n_azimuthal;
    int64_t table_entries;   /* Cuda1dPlan::table_entries (masked table) */
    int64_t full_entries;    /* entries before mask compaction */
    int64_t max_batch_frames;/* Cuda1dPlan::max_batch_frames */
    int32_t device, precision;
    double hist_min, hist_step;
    double build_ms;         /* device CSR build, event-timed */
    int64_t device_bytes;    /* HBM held by the plan */
    int64_t guard_corners;   /* corners within the FP64 guard band of a bin edge */
    int64_t singular_pixels; /* pixels integrated by detector-plane sampling */
} dg_plan_info;

/* Replaces Cuda1dPlan::{shape, n_points, table_entries, max_batch_frames,
 * device} (src/integration/cuda.rs:420-470). */
DG_EXPORT dg_status dg_plan_query(const dg_plan *plan, dg_plan_info *out);

/* Radial (and for 2D azimuthal) bin centres; Cuda1dPlan::radial
 * (src/integration/cuda.rs:455-460). n must equal the bin count. */
DG_EXPORT dg_status dg_plan_radial(const dg_plan *plan, double *out, int64_t n);
DG_EXPORT dg_status dg_plan_azimuthal(const dg_plan *plan, double *out, int64_t n);

/* Copies a table to host memory for parity checks. which = 0: the masked
 * table the gather uses (fixed_csr_parts, src/lut/prepared.rs:194-202), with
 * its f64 denominators; which = 1: the unmasked table (needs
 * DG_PLAN_KEEP_TABLES). row_ptr has n_bins+1 entries, col/weight
 * *_entries; any pointer may be NULL to skip it. weight is the f64 weight the
 * builder produced (1.0 for counting tables). */
DG_EXPORT dg_status dg_plan_export_table(const dg_plan *plan, int32_t which, int64_t *row_ptr,
                               int32_t *col, double *weight, double *denominator);

/* Replaces Cuda1dPlan::integrate_frames / integrate_stack
 * (src/integration/cuda.rs:499-564) and Cuda2dPlan::integrate_*_into
 * (:770-863): n_frames row-major frames stacked in HOST memory, results to
 * HOST arrays of n_frames * n_bins doubles (out_sigma needs DG_ERRORS,
 * out_std DG_AZIMUTHAL_STD; pass NULL otherwise). Frames are copied to the
 * device in chunks of at most max_batch_frames. Results do not depend on how
 * frames are chunked or batched. */
DG_EXPORT dg_status dg_integrate(dg_plan *plan, const void *frames, int32_t dtype, int64_t n_frames,
                       uint32_t flags, double *out_intensity, double *out_sigma,
                       double *out_std);

/* Same with frames and results already in DEVICE memory of the plan's GPU,
 * enqueued on `stream` (a cudaStream_t; NULL = the plan's own stream). No
 * synchronisation: the caller owns completion. */
DG_EXPORT dg_status dg_integrate_device(dg_plan *plan, const void *d_frames, int32_t dtype,
                              int64_t n_frames, uint32_t flags, double *d_intensity,
                              double *d_sigma, double *d_std, void *stream);

/* Allocation-free form of dg_integrate_device; it has no counterpart in the
 * reference. For callers that may not allocate device memory while they
 * integrate (a real-time acquisition loop with a fixed memory budget, a thread
 * that must not enter the CUDA allocator): dg_integrate_device allocates its
 * partial sums on first use, this call keeps them in one fixed 32 MiB array
 * that every GPU loading the library holds until the process exits. It calls
 * no cudaMalloc or cudaFree; the plan (from dg_plan_create, which does
 * allocate) and the frames and results are the caller's. A plan whose partial
 * sums for a single frame exceed the array is rejected with
 * DG_UNSUPPORTED. The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress); make it before any stream capture. All
 * calls on a device share the array, so calls that overlap on the GPU race:
 * serialise them. Results equal dg_integrate_device's. */
DG_EXPORT dg_status dg_integrate_device_noalloc(dg_plan *plan, const void *d_frames,
                                                int32_t dtype, int64_t n_frames, uint32_t flags,
                                                double *d_intensity, double *d_sigma,
                                                double *d_std, void *stream);

/* One-frame-per-launch form of dg_integrate_device: one gather launch per
 * frame, the table re-read for every frame. The plain GPU path the batched
 * kernel is measured against. */
DG_EXPORT dg_status dg_integrate_device_plain(dg_plan *plan, const void *d_frames, int32_t dtype,
                                    int64_t n_frames, uint32_t flags, double *d_intensity,
                                    double *d_sigma, double *d_std, void *stream);

/* Failure-detection check of the bin-tile gathers (lane mappings 7 and 8);
 * it has no counterpart in the reference. Their warps pass chunks through
 * shared-memory barriers whose every wait gives up after 1 s; the kernel then
 * marks a flag in mapped host memory, and the plan's next call (host-memory
 * calls: the same call) returns DG_TIMEOUT. This call runs one gather of the
 * device frames with one warp of one CTA never reporting a chunk summed, so
 * the other warps' waits run out. It waits for the GPU and returns DG_TIMEOUT
 * when the kernel reported the expired wait (DG_OK when the tile had too few
 * chunks to stall); the results are undefined, and the plan integrates
 * normally afterwards. DG_UNSUPPORTED unless the plan uses mapping 7 or 8. */
DG_EXPORT dg_status dg_plan_test_wait_timeout(dg_plan *plan, const void *d_frames, int32_t dtype,
                                              int64_t n_frames, uint32_t flags,
                                              double *d_intensity, double *d_sigma,
                                              double *d_std);

/* Kernel timing for roofline reports; the reference times its CUDA phases
 * with events in src/integration/cuda/bench.rs:139-196. With enable != 0,
 * every gather-kernel launch of the plan is bracketed by CUDA events on the
 * stream it runs on. dg_plan_kernel_time waits for the last recorded event and
 * returns the summed gather-kernel time, the number of gather launches and the
 * number of all kernel launches since the last reset. */
DG_EXPORT dg_status dg_plan_profile(dg_plan *plan, int32_t enable);
DG_EXPORT dg_status dg_plan_kernel_time(dg_plan *plan, int32_t reset, double *gather_ms,
                                        int64_t *gather_launches, int64_t *launches);

/* Per-plan autotuner of the gather's launch shape; it has no counterpart in
 * the reference, whose gather kernels run one fixed shape
 * (src/integration/cuda/device.rs). The gather has several lane mappings
 * (entry slices per frame group, frames per lane, entries in flight per
 * lane). dg_plan_autotune times each on up to 256 of the given DEVICE frames
 * (dtype, flags as dg_integrate_device) on `stream` (NULL: the plan's own),
 * keeps the fastest for every later call of the plan and returns it in
 * *variant (may be NULL); ms (may be NULL) receives the launch time of each
 * mapping in mapping order, n_ms entries at most.
 * Synchronous. The mappings round differently within the stated tolerance;
 * one plan's results are reproducible between calls made with the same
 * mapping; mappings a table cannot use are skipped (their time is -1).
 * dg_plan_variant reads the plan's mapping into *current and the number of
 * mappings into *count (either may be NULL) and, when set >= 0, selects
 * mapping `set` first (DG_UNSUPPORTED if the table cannot use it). */
DG_EXPORT dg_status dg_plan_autotune(dg_plan *plan, const void *d_frames, int32_t dtype,
                                     int64_t n_frames, uint32_t flags, void *stream,
                                     int32_t *variant, double *ms, int32_t n_ms);
DG_EXPORT dg_status dg_plan_variant(dg_plan *plan, int32_t set, int32_t *current,
                                    int32_t *count);

/* Page-locked host buffers for frames. Replaces Cuda1dPlan's pinned staging
 * (alloc_pinned_batch, src/python/cuda.rs:808-870; is_pinned_host,
 * src/integration/cuda/device.rs:1055-1078): a reader decodes straight into
 * the buffer and the host-memory calls copy from it by DMA, asynchronously.
 * dg_host_alloc makes `bytes` of pinned memory usable from every device
 * (allocated while `device` is current); dg_host_free releases it;
 * dg_host_is_pinned is 1 for page-locked host memory, else 0 (any pointer). */
DG_EXPORT dg_status dg_host_alloc(int32_t device, int64_t bytes, void **out);
DG_EXPORT dg_status dg_host_free(void *ptr);
DG_EXPORT int32_t dg_host_is_pinned(const void *ptr);

/* Per-frame masks (MaskMode::Dynamic). Replaces Dynamic1dPlan::integrate
 * (src/integration/dynamic.rs:159-196; the per-row sums with a mask check,
 * src/lut/prepared.rs:1011-1118), which the reference's GPU plans reject
 * (src/integration/cuda.rs:1036-1040). masks holds n_frames uint8 masks of
 * dim1 * dim2 bytes, mask_stride bytes apart (0: one mask for every frame);
 * a nonzero byte masks its pixel. Each bin sums w*s, w^2*max(s,0) and
 * w*norm over the entries whose pixel is unmasked in that frame, so
 * denominators follow the frame's mask: I = 0 where the denominator is 0,
 * else S/N; sigma likewise (normalize_bin, prepared.rs:985-996). A plan made
 * for per-frame masks is created without a mask (the reference's
 * prepare_dynamic1d excludes the stored mask); a plan mask, if given, is
 * applied as well. DG_ERRORS only: azimuthal_std is DG_UNSUPPORTED here.
 * Frames, masks and results in HOST memory; the _device form takes DEVICE
 * memory and enqueues on `stream` (NULL: the plan's own) without
 * synchronising. */
DG_EXPORT dg_status dg_integrate_dynamic(dg_plan *plan, const void *frames, int32_t dtype,
                                         int64_t n_frames, const uint8_t *masks,
                                         int64_t mask_stride, uint32_t flags,
                                         double *out_intensity, double *out_sigma);
DG_EXPORT dg_status dg_integrate_dynamic_device(dg_plan *plan, const void *d_frames,
                                                int32_t dtype, int64_t n_frames,
                                                const uint8_t *d_masks, int64_t mask_stride,
                                                uint32_t flags, double *d_intensity,
                                                double *d_sigma, void *stream);

/* Raw sums before division, for merging several detectors. Replaces
 * Integrator::integrate1d_raw / integrate1d_raw_with_variance
 * (src/integration/methods.rs:299-360), whose IntermediateResult1d
 * (src/lut/integrate.rs:372-379) holds per bin sum_signal = sum w*s,
 * sum_norm = sum w*norm, sum_variance = sum w^2*max(s,0) (with DG_ERRORS)
 * and count = sum w. masks NULL: the plan's own mask, with sum_norm and
 * count the plan's FP64 sums; otherwise per-frame masks as in
 * dg_integrate_dynamic. Outputs are n_frames * n_bins doubles each
 * (out_variance may be NULL without DG_ERRORS). */
DG_EXPORT dg_status dg_integrate_raw(dg_plan *plan, const void *frames, int32_t dtype,
                                     int64_t n_frames, const uint8_t *masks, int64_t mask_stride,
                                     uint32_t flags, double *out_signal, double *out_norm,
                                     double *out_variance, double *out_count);
DG_EXPORT dg_status dg_integrate_raw_device(dg_plan *plan, const void *d_frames, int32_t dtype,
                                            int64_t n_frames, const uint8_t *d_masks,
                                            int64_t mask_stride, uint32_t flags,
                                            double *d_signal, double *d_norm,
                                            double *d_variance, double *d_count, void *stream);

/* Bitshuffle/LZ4 frames. Replaces Cuda1dPlan::integrate_bslz4 and
 * Cuda2dPlan::integrate_bslz4 / integrate_bslz4_into
 * (src/integration/cuda.rs:554-564, :758-767, :843-863), whose chunks are
 * `&[&[u8]]`: chunks[f] points to chunk_bytes[f] bytes of frame f's raw HDF5
 * Bitshuffle/LZ4 chunk in HOST memory (a big-endian u64 of the frame's bytes,
 * a big-endian u32 block size with 0 meaning 8192, then per block a
 * big-endian u32 length and an LZ4 block of bitshuffled elements, the last
 * n mod 8 elements verbatim). dtype is DG_U16, DG_U32 or DG_I32 (Bslz4Dtype,
 * cuda.rs:338-342). Only the compressed bytes cross PCIe; the frames are
 * decoded on the device and integrated as by dg_integrate, with identical
 * results. Block sizes up to 48 KiB, multiples of 8 elements. A chunk whose
 * header does not match the plan's frame size, whose blocks are truncated or
 * exceed the LZ4 bound is rejected with DG_INVALID_INPUT before any device
 * work (device.rs:2056-2178); malformed LZ4 data found while decoding returns
 * DG_INVALID_INPUT ("corrupt or truncated Bitshuffle/LZ4 compressed block").
 * Chunks may be pageable or pinned; pinned chunks copy asynchronously while
 * the previous batch is decoded and integrated. Synchronous. */
DG_EXPORT dg_status dg_integrate_bslz4(dg_plan *plan, const void *const *chunks,
                                       const int64_t *chunk_bytes, int64_t n_frames,
                                       int32_t dtype, uint32_t flags, double *out_intensity,
                                       double *out_sigma, double *out_std);

/* Host encoder of the same chunk format (bitshuffle, then LZ4 with greedy
 * matching); it has no counterpart in the reference, whose chunks come from
 * the detector's HDF5 files. Writes the chunk of n_elems elements of
 * elem_bytes (2 or 4) bytes to out (capacity bytes; dg_bslz4_bound gives a
 * sufficient capacity, or -1 for invalid arguments) and its size to
 * *out_bytes. block_bytes 0 writes the default 8192-byte blocks. */
DG_EXPORT int64_t dg_bslz4_bound(int64_t n_elems, int32_t elem_bytes, int32_t block_bytes);
DG_EXPORT dg_status dg_bslz4_compress(const void *frame, int64_t n_elems, int32_t elem_bytes,
                                      int32_t block_bytes, void *out, int64_t capacity,
                                      int64_t *out_bytes);

/* Decode-kernel time of dg_integrate_bslz4 calls made while dg_plan_profile is
 * enabled: the summed CUDA-event time of the decode launches and their number
 * since the last reset (waits for the last one). */
DG_EXPORT dg_status dg_plan_decode_time(dg_plan *plan, int32_t reset, double *ms,
                                        int64_t *launches);

/* Evaluates one FP64 primitive of the device table builders on n values in
 * DEVICE memory of the current device, for parity checks against the C
 * library the reference calls (f64::atan2 and f64::sin, geometry.rs:684-692,
 * integration.rs:167): which = 0 the builders' correctly rounded atan2(a, b),
 * 1 their correctly rounded sin(a), 2 CUDA's atan2, 3 CUDA's sin. b is unused
 * for sin. Synchronous. */
DG_EXPORT dg_status dg_eval_math(int32_t which, const double *d_a, const double *d_b,
                                 int64_t n, double *d_out);

/* Request loop (continuous batching across plans). Replaces the reference's
 * bounded streaming executor (src/batch/bounded.rs:56-420) for device work:
 * requests are admitted while slots and HBM allow, same-plan requests are
 * coalesced into one launch, results come back through dg_server_poll. */
typedef struct dg_server dg_server;

typedef struct dg_server_config {
    int32_t device;
    int32_t max_inflight_frames; /* admission slots */
    int64_t cache_bytes;         /* HBM budget of the plan cache */
    int32_t max_coalesce;        /* most frames one launch takes */
    int32_t poll_us;             /* worker idle wait */
} dg_server_config;

typedef struct dg_server_stats {
    int64_t submitted, completed, failed, launches, coalesced_frames;
    int64_t plan_builds, plan_hits, plan_evictions, cache_bytes;
    int64_t batch_us;  /* workers' time from a batch's first copy to its results */
    int64_t build_us;  /* time spent building (and tuning) plans */
} dg_server_stats;

DG_EXPORT dg_status dg_server_create(const dg_server_config *config, dg_server **out);
DG_EXPORT dg_status dg_server_destroy(dg_server *server);
/* Registers a plan configuration under `key` (built on first use, rebuilt
 * when evicted). Replaces re-preparing a Cuda1dPlan per geometry. */
DG_EXPORT dg_status dg_server_register(dg_server *server, uint64_t key, const dg_geometry *geometry,
                             const dg_method *method, const uint8_t *mask, int32_t dim1,
                             int32_t dim2, int32_t n_radial, int32_t n_azimuthal,
                             const double *azimuthal_range);
/* Queues one frame (host memory, copied before return) for plan `key`;
 * returns a ticket. DG_TIMEOUT if no slot frees within wait_ms. */
DG_EXPORT dg_status dg_server_submit(dg_server *server, uint64_t key, const void *frame, int32_t dtype,
                           uint32_t flags, int32_t wait_ms, uint64_t *ticket);
/* Waits up to wait_ms for `ticket`; fills n_bins doubles per requested
 * output and the request's latency in microseconds (submit to result). */
DG_EXPORT dg_status dg_server_poll(dg_server *server, uint64_t ticket, int32_t wait_ms,
                         double *out_intensity, double *out_sigma, double *out_std,
                         double *latency_us);
DG_EXPORT dg_status dg_server_stats_get(dg_server *server, dg_server_stats *out);

/* ---- Several plans in one launch (work-queue gather) ----
 * No counterpart in the reference, whose engine launches one plan at a time
 * (src/integration/cuda/device.rs:1417-1584; streaming driver
 * src/batch/bounded.rs:172). A dg_multi integrates batches of device-resident
 * frames of several plans together: a grid of row-warp CTAs (one per tile;
 * resident and claiming for batches of more than 2^24 tiles) takes
 * (plan, row item, block of four frames) tiles from one counter until every
 * plan's table is summed, so plans of very different sizes share the GPU without a launch
 * per plan; each row's results are written by the CTA that sums it (no
 * partial sums, no second pass). The device work of a call (descriptor copy,
 * gather) is a CUDA graph captured on the first call of each (dtype, flags)
 * and replayed after that. Every plan is summed as by lane mapping 10, so
 * each item's results equal dg_integrate_device of that plan with mapping 10
 * selected, bit for bit. DG_UNSUPPORTED for a table of more than 2^31
 * entries. Meant for small batches (a frame pass reads the table once per
 * four frames). No kernel of the call waits on another.
 * Items share one dtype and one set of flags; a plan appears in at most one
 * item of a call; an item carries 0..256 frames. Calls on one dg_multi are
 * serialised (a call waits until the previous one's device work is done
 * before it rewrites the descriptors). Plans are locked for the call, as by
 * dg_integrate_device. */
typedef struct dg_multi dg_multi;
typedef struct dg_multi_item {
    dg_plan *plan;
    const void *d_frames;   /* n_frames frames of the plan's shape, device memory */
    int64_t n_frames;       /* 0..256 */
    double *d_intensity;    /* n_frames x n_bins, device memory */
    double *d_sigma;        /* with DG_ERRORS */
    double *d_std;          /* with DG_AZIMUTHAL_STD (1D plans) */
} dg_multi_item;
DG_EXPORT dg_status dg_multi_create(int32_t device, int32_t max_plans, dg_multi **out);
DG_EXPORT dg_status dg_multi_destroy(dg_multi *multi);
/* Enqueues the items on `stream` (a cudaStream_t; NULL = the multi's own).
 * No synchronisation: the caller owns completion. */
DG_EXPORT dg_status dg_multi_integrate(dg_multi *multi, const dg_multi_item *items,
                                       int32_t n_items, int32_t dtype, uint32_t flags,
                                       void *stream);
/* Test hook: with on != 0, later calls run the resident grid (the CTAs the
 * SMs hold at once, claiming tiles from the queue's counter) that otherwise
 * only batches of more than 2^24 tiles use. Results are the same either way. */
DG_EXPORT dg_status dg_multi_test_resident(dg_multi *multi, int32_t on);

/* Device description; cuda_info (src/integration/cuda.rs:262-329). */
typedef struct dg_device_info {
    int32_t available;
    int32_t device;
    int32_t cc_major, cc_minor;
    int32_t sm_count;
    int64_t total_memory_bytes;
    int32_t driver_version;
    char name[128];
} dg_device_info;
DG_EXPORT dg_status dg_device_info_get(int32_t device, dg_device_info *out);

/* Message of the calling thread's last failed call; returns its length. */
DG_EXPORT int32_t dg_last_error(char *buf, size_t len);

#ifdef __cplusplus
}
#endif
#endif
