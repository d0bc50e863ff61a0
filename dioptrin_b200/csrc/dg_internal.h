// Internal declarations shared by the translation units of libdioptrin_b200.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dioptrin_gpu.h"

namespace dg {

// Error carried from the point of failure to the C ABI, which stores the
// message in the calling thread's last-error slot and returns the status.
struct Error {
    dg_status status;
    std::string message;
};

[[noreturn]] void fail(dg_status status, const std::string &message);
// Stores `message` as the calling thread's dg_last_error text.
void set_last_error(const std::string &message);
void check_cuda(cudaError_t err, const char *what);
#define DG_CUDA(call) ::dg::check_cuda((call), #call)

// Device allocation owned by a plan; freed with the plan.
template <typename T>
struct DeviceArray {
    T *ptr = nullptr;
    size_t count = 0;
    DeviceArray() = default;
    DeviceArray(const DeviceArray &) = delete;
    DeviceArray &operator=(const DeviceArray &) = delete;
    DeviceArray(DeviceArray &&o) noexcept : ptr(o.ptr), count(o.count) {
        o.ptr = nullptr;
        o.count = 0;
    }
    DeviceArray &operator=(DeviceArray &&o) noexcept {
        if (this != &o) {
            release();
            ptr = o.ptr;
            count = o.count;
            o.ptr = nullptr;
            o.count = 0;
        }
        return *this;
    }
    ~DeviceArray() { release(); }
    void alloc(size_t n) {
        release();
        if (n == 0) n = 1;
        cudaError_t e = cudaMalloc(reinterpret_cast<void **>(&ptr), n * sizeof(T));
        if (e != cudaSuccess) {
            ptr = nullptr;
            (void)cudaGetLastError();
            fail(DG_DEVICE, "device allocation of " + std::to_string(n * sizeof(T)) +
                                " bytes failed: " + cudaGetErrorString(e));
        }
        count = n;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
    size_t bytes() const { return count * sizeof(T); }
};

// One int in mapped page-locked host memory: a kernel sets it to report a
// failure without the host synchronising; the host reads it at any time.
struct PinnedFlag {
    int *host = nullptr;
    int *dev = nullptr;
    PinnedFlag() = default;
    PinnedFlag(const PinnedFlag &) = delete;
    PinnedFlag &operator=(const PinnedFlag &) = delete;
    PinnedFlag(PinnedFlag &&o) noexcept : host(o.host), dev(o.dev) {
        o.host = nullptr;
        o.dev = nullptr;
    }
    PinnedFlag &operator=(PinnedFlag &&o) noexcept {
        if (this != &o) {
            release();
            host = o.host;
            dev = o.dev;
            o.host = nullptr;
            o.dev = nullptr;
        }
        return *this;
    }
    ~PinnedFlag() { release(); }
    void alloc() {
        if (host) return;
        void *p = nullptr;
        cudaError_t e = cudaHostAlloc(&p, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable);
        void *d = nullptr;
        if (e == cudaSuccess) e = cudaHostGetDevicePointer(&d, p, 0);
        if (e != cudaSuccess) {
            if (p) cudaFreeHost(p);
            (void)cudaGetLastError();
            fail(DG_DEVICE, std::string("mapped host flag allocation failed: ") +
                                cudaGetErrorString(e));
        }
        host = static_cast<int *>(p);
        dev = static_cast<int *>(d);
        *host = 0;
    }
    void release() {
        if (host) cudaFreeHost(host);
        host = nullptr;
        dev = nullptr;
    }
};

// Geometry scalars the device kernels need. Trigonometric constants and the
// q scale are computed on the host with the C library so that they are the
// same bits the reference computes (geometry.rs:640-660, integration.rs:147-158).
struct GeomParams {
    double pixel1, pixel2, distance, poni1, poni2;
    double s1, c1, s2, c2, s3, c3;
    double wavelength, q_scale;
    int unit;
    int has_pol;
    double pol_factor;
};

GeomParams make_geom_params(const dg_geometry &g, const dg_method &m);

// A CSR table in device memory, as produced by the builders (f64 weights,
// the reference's Lut1d/Lut2d) or compacted for the gather.
struct DeviceCsr {
    int64_t n_rows = 0;
    int64_t nnz = 0;
    DeviceArray<int64_t> row_ptr;  // n_rows + 1
    DeviceArray<int32_t> col;      // nnz
    DeviceArray<double> w;         // nnz
};

struct BuildResult {
    DeviceCsr full;                 // unmasked table
    double hist_min = 0, hist_step = 0;
    int64_t guard_corners = 0;
    int64_t singular_pixels = 0;
    DeviceArray<double> norm;       // per-pixel pol*sa (f64)
    std::vector<double> radial_centres;
    std::vector<double> azimuthal_centres;
};

// Device CSR construction (dg_build.cu).
void build_table(const dg_geometry &g, const dg_method &m, int32_t dim1, int32_t dim2,
                 int32_t n_radial, int32_t n_azimuthal, const double *azimuthal_range,
                 cudaStream_t stream, BuildResult &out);
// Order-preserving mask compaction (fixed_table) + strict f64 denominators.
void compact_table(const DeviceCsr &full, const uint8_t *d_mask, int32_t n_pixels,
                   cudaStream_t stream, DeviceCsr &out);
void denominators(const DeviceCsr &table, const double *d_norm, cudaStream_t stream,
                  double *d_den);
// Device FP64 primitives on arrays: 0 correctly rounded atan2(a, b), 1 its
// sin(a), 2 CUDA atan2, 3 CUDA sin.
void eval_math(int which, const double *a, const double *b, int64_t n, double *out,
               cudaStream_t stream);

// Pairs of CUDA events, created on demand and destroyed with the pool.
// Orders the uses of a plan's scratch by calls on different streams (a
// caller may name any stream): each use records `done` on its stream, and a
// use on another stream waits for it first. Calls on one stream are ordered
// by the stream already.
struct ScratchOrder {
    cudaEvent_t done = nullptr;
    cudaStream_t last = nullptr;
    bool used = false;
    ScratchOrder() = default;
    ScratchOrder(const ScratchOrder &) = delete;
    ScratchOrder &operator=(const ScratchOrder &) = delete;
    ScratchOrder(ScratchOrder &&o) noexcept : done(o.done), last(o.last), used(o.used) {
        o.done = nullptr;
        o.used = false;
    }
    ScratchOrder &operator=(ScratchOrder &&o) noexcept {
        if (this != &o) {
            if (done) cudaEventDestroy(done);
            done = o.done;
            last = o.last;
            used = o.used;
            o.done = nullptr;
            o.used = false;
        }
        return *this;
    }
    ~ScratchOrder() {
        if (done) cudaEventDestroy(done);
    }
    void wait(cudaStream_t s) {
        if (used && last != s) DG_CUDA(cudaStreamWaitEvent(s, done, 0));
    }
    void mark(cudaStream_t s) {
        if (!done) DG_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        DG_CUDA(cudaEventRecord(done, s));
        last = s;
        used = true;
    }
};

struct EventPool {
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
    size_t used = 0;
    EventPool() = default;
    EventPool(const EventPool &) = delete;
    EventPool &operator=(const EventPool &) = delete;
    EventPool(EventPool &&o) noexcept : events(std::move(o.events)), used(o.used) {
        o.events.clear();
        o.used = 0;
    }
    EventPool &operator=(EventPool &&o) noexcept {
        if (this != &o) {
            destroy();
            events = std::move(o.events);
            used = o.used;
            o.events.clear();
            o.used = 0;
        }
        return *this;
    }
    ~EventPool() { destroy(); }
    void destroy() {
        for (auto &e : events) {
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
        events.clear();
        used = 0;
    }
};

// One bin-tile layout (dg_gather.cu): runs of rows whose entries are cut
// into pixel-interval chunks, built on first use.
struct BinTiles {
    bool built = false;
    int32_t n_items = 0;
    DeviceArray<int4> item;        // {first row, rows, first chunk, chunks}, largest first
    // Items 2m and 2m + 1 are neighbouring tiles launched as one 2-CTA
    // cluster per frame group (an odd count ends with an empty item).
    bool paired = false;
    DeviceArray<int32_t> meta;     // per chunk: {pixels, pairs, first pair}, row offsets, pixels
    DeviceArray<int4> org;         // per row {origin entry, first valid entry, row end, 0}
    DeviceArray<float4> pair_a, pair_as, pair_b;
    DeviceArray<float2> pair_c;    // {n_lo 0, n_lo 1} (spread)
    // Per pair {slot 0, slot 1, entry 0, entry 1}, kept to build the
    // per-frame-mask pairs {slot, slot, w, w}, {w*norm, w*norm} on first use.
    DeviceArray<int4> desc;
    DeviceArray<float4> pair_ra, pair_rb;
    bool raw_built = false;
    // Set by k_gather_bins when a wait of its chunk pipeline gave up.
    PinnedFlag wait_err;
    int64_t bytes() const {
        return int64_t(item.bytes() + meta.bytes() + org.bytes() + pair_a.bytes() +
                       pair_as.bytes() + pair_b.bytes() + pair_c.bytes() + desc.bytes() + pair_ra.bytes() +
                       pair_rb.bytes());
    }
};

// Gather-side table (dg_gather.cu). The masked table is cut into segments,
// each a run of one row's entries whose pixels lie in one strip of detector
// rows; segments of the same strip and neighbouring rows are grouped into
// units, one CTA each, so a CTA's warps read the same detector region.
struct GatherTable {
    int32_t n_rows = 0;
    int64_t nnz = 0;
    int32_t n_segments = 0;
    int32_t n_units = 0;
    int32_t unit_cap = 0;             // most entries one unit stages in shared memory
    int32_t strip_rows = 0;           // detector rows per strip
    DeviceArray<int4> seg;            // {row, begin, end, row end}
    DeviceArray<int2> unit;           // {first segment, segment count}
    DeviceArray<int32_t> row_seg;     // n_rows + 1: row r's segments are
    DeviceArray<int32_t> seg_ids;     //   seg_ids[row_seg[r] .. row_seg[r+1]) in strip order
    DeviceArray<int32_t> first_valid; // first entry valid for the spread, per row (-1: none)
    DeviceArray<int32_t> origin;      // the spread's origin entry: the row's heaviest valid (-1: none)
    DeviceArray<int2> entry;          // {col, weight bits} for the I/sigma path
    DeviceArray<float4> entry_std;    // {col bits, c, n, c/n} for the spread path (n in FP32)
    DeviceArray<float> entry_nlo;     // n - FP32(n) per entry: the spread's n as an FP32 pair
    DeviceArray<double> den;          // strict f64 sum w*norm
    DeviceArray<double> den_std;      // sum c*n over entries valid for the spread
    DeviceArray<int32_t> valid_std;   // entries valid for the spread, per row
    DeviceArray<double> partial;      // scratch: per (frame, segment) FP64 sums
    // Frame-lane layout (k_gather_fl): units of segments with a bounded
    // number of distinct pixels, their pixel lists (a fixed stride apart) and
    // the entries in unit order as pairs, columns as indices into the lists.
    int32_t fl_n_units = 0;
    DeviceArray<int4> fl_unit;        // {first segment, segment count, first pair, pixels}
    DeviceArray<int32_t> fl_px;
    DeviceArray<float4> fl_pair_a;    // {index 0 bits, index 1 bits, c0, c1}
    DeviceArray<float4> fl_pair_b;    // {n0, n1, c0/n0, c1/n1} (spread)
    DeviceArray<float2> fl_pair_c;    // {n_lo 0, n_lo 1} (spread)
    DeviceArray<float4> fl_pair_s;    // pair_a with the spread's weights, when they differ
    const float4 *fl_pair_as = nullptr;  // the spread's pair_a (fl_pair_s or fl_pair_a)
    DeviceArray<int32_t> fl_seg_org;  // per segment: its origin pixel's index in the unit list
    // Raw-sum and per-frame-mask gathers, built on first use (prepare_raw):
    // {pixel bits, w, w*norm, 0} per entry and the FP64 weight sum per row.
    DeviceArray<float4> entry_raw;
    DeviceArray<double> cnt;
    // Bin tiles (k_gather_bins), mappings 7 and 8; see dg_gather.cu.
    BinTiles bt[2];
    // Row warps (k_rows), mapping 10: row pointers, rows with more than
    // kRowsLong entries (longest first) then the others, and one item per
    // CTA: {row, 0, entry begin, entry end} for a long row, {first in
    // rw_rows, count <= 8} for rows taken one per warp, {first, -count <= 32}
    // for rows of at most kRowsTiny entries taken eight lanes each.
    int32_t rw_n_items = 0;
    // Per pixel (frame storage order) its norm n as an FP32 pair {n, n - n32},
    // {0, 0} where n is not finite or not positive: the row warps' spread
    // reads the 8-byte entries and gathers n beside the pixel.
    DeviceArray<float2> px_norm;
    DeviceArray<int32_t> rw_row_ptr;
    DeviceArray<int32_t> rw_rows;
    DeviceArray<int4> rw_item;
    int variant = 0;                  // gather lane mapping (dg_gather.cu kVariantCount)
    int withhold_test = 0;            // bin tiles: stall one warp (dg_plan_test_wait_timeout)
    int32_t flip_rows = 0, flip_cols = 0;  // frames stored bottom row first (0: detector order)
    // Optional CUDA-event timing of the gather launches (dg_plan_profile).
    bool profile = false;
    EventPool events;
    ScratchOrder scratch;  // orders uses of `partial` across streams
    int64_t launches = 0;  // every kernel launch of run_gather since the last reset
};

// Sums the recorded gather-kernel event pairs (synchronising on the last);
// reset clears them.
void gather_kernel_time(GatherTable &t, bool reset, double *ms, int64_t *gather_launches,
                        int64_t *launches);

void make_gather_table(const DeviceCsr &table, const double *d_norm, int32_t dim1,
                       int32_t dim2, int32_t strip_rows, cudaStream_t stream, GatherTable &out);
// Enqueues the batched gather for n_frames device-resident frames. With
// `scratch` (scratch_doubles long) the partial sums go there instead of the
// plan's own array, which is then neither allocated nor ordered across
// streams; frames per launch shrink to what the scratch holds.
void run_gather(GatherTable &t, const void *d_frames, int dtype, int64_t n_pixels,
                int64_t n_frames, uint32_t flags, int precision, double *d_i, double *d_sigma,
                double *d_std, cudaStream_t stream, double *scratch = nullptr,
                size_t scratch_doubles = 0);
// Whether the plan's gather writes the results itself (bin tiles: no partial
// sums, no finalize).
bool gather_writes_results(const GatherTable &t);
// Allocates the plan's partial sums for launches of up to n_frames frames of
// this dtype and these flags, ahead of the first call that needs them (not
// for a plan whose bin tiles need none, unless `any_mapping`).
void reserve_partials(GatherTable &t, int64_t n_frames, uint32_t flags, int dtype,
                      bool any_mapping = false);
// Row warps (k_rows, lane mapping 10) over one plan's batch, and the
// work-queue gather over several plans (dg_multi.cu, dg_gather.cu): one
// descriptor per (plan, batch of frames), after a header. The queue's
// persistent CTAs claim (plan, row item, frame block) tiles from `counter`
// until total_items are done; item_first is the prefix index of a plan's
// first tile.
struct QueuePlan {
    const int4 *item;
    const int32_t *rows;
    const int32_t *row_ptr;
    const int2 *entry;
    const float4 *entry_std;
    const float *entry_nlo;
    const float2 *px_norm;
    const int32_t *first_valid;
    const int32_t *origin;
    const double *den;
    const double *den_std;
    const int32_t *valid_std;
    const void *frames;
    double *out_i, *out_s, *out_d;
    int64_t n_pixels;
    int32_t n_frames, n_rows;
    int32_t n_items;       // row items
    int32_t frame_blocks;  // blocks of up to four frames (one pass each)
    int32_t item_first;    // the work queue: first (item, frame block) tile
    int32_t pad;
};
struct QueueHeader {
    int32_t n_plans, total_items, counter, pad;  // counter: 0 before each launch
};
// Fills a descriptor from a plan's gather table (item_first left 0); n_items
// is 0 when the table has no row-warp items (more than 2^31 entries).
QueuePlan queue_plan(const GatherTable &t, const void *d_frames, int64_t n_pixels, int n_frames,
                     double *oi, double *os, double *od);
// Enqueues the work-queue gather for descriptors already in device memory
// (`hdr` followed by the descriptors) on `s`, at its resident capacity (the
// request's grid is set per call, queue_grid).
void queue_launch(int dtype, uint32_t flags, QueueHeader *hdr, const QueuePlan *plans,
                  cudaStream_t s);
// The work-queue gather's grid for a call of total_tiles tiles: one CTA per
// tile, or (beyond 2^24 tiles, or with `resident`) the CTAs the SMs hold at
// once, which then claim tiles until the queue is empty.
int queue_grid(int dtype, uint32_t flags, int64_t total_tiles, bool resident = false);
// The allocation-free path's fixed device array (dg_gather.cu): its address
// on the current device, looked up on every call, and its size in doubles.
double *noalloc_scratch(size_t *n_doubles);
// Raw sums and per-frame masks. prepare_raw builds the entries once (from the
// plan's masked f64 table and per-pixel norm). run_gather_raw: with d_masks
// (n_frames masks mask_stride bytes apart, 0 = one mask for every frame;
// nonzero bytes mask a pixel) sums over the unmasked entries of each frame,
// else over the table; raw: o0..o3 = signal, norm, variance (DG_ERRORS),
// count; otherwise o0, o1 = intensity and sigma (DG_ERRORS) normalised by
// the frame's own denominators (needs d_masks).
// InputOrder::FlipVertical: remaps the pixel indices of a built gather table
// to frames whose rows come in reverse order (entry order unchanged).
void flip_gather_rows(GatherTable &t, int32_t dim1, int32_t dim2, cudaStream_t s);
// Bin tiles of lane mapping `variant` (7 or 8), built from the plan's masked
// table on first use (the autotuner, or selecting the mapping); idempotent.
void ensure_bin_tiles(GatherTable &t, const DeviceCsr &table, int variant, cudaStream_t s);
bool gather_variant_needs_tiles(int variant);
// Throws DG_TIMEOUT (once) when a bin-tile launch of this table gave up a
// pipeline wait; bin_tile_wait_failed only reports and clears it.
bool bin_tile_wait_failed(const GatherTable &t);
void check_bin_tile_waits(const GatherTable &t);
// Whether the autotuner times bin-tile mapping `variant` (7 or 8) for a
// batch of n_frames: a launch must give every SM at least two CTAs (tiles
// times frame groups) and fill at least half of each CTA's frames.
bool bin_tiles_fill_gpu(const GatherTable &t, int variant, int64_t n_frames);
void prepare_raw(GatherTable &t, const DeviceCsr &table, const double *d_norm, cudaStream_t s);
void run_gather_raw(GatherTable &t, const void *d_frames, int dtype, int64_t n_pixels,
                    int64_t n_frames, const uint8_t *d_masks, int64_t mask_stride, uint32_t flags,
                    bool raw, double *o0, double *o1, double *o2, double *o3, cudaStream_t s);
// Number of gather kernel launches run_gather enqueues (for launch counting).
int gather_launches_per_call();
// Lane-mapping variants of the gather, and the per-plan autotuner: times each
// variant's gather launch on the given frames and keeps the fastest in
// t.variant (returned; `each` receives every variant's time in ms).
int gather_variant_count();
bool gather_variant_available(const GatherTable &t, int variant);
int autotune_gather(GatherTable &t, const void *d_frames, int dtype, int64_t n_pixels,
                    int64_t n_frames, uint32_t flags, cudaStream_t stream,
                    std::vector<double> *each);

// Exclusive scans (dg_scan.cu). `temp` sizing via scan_temp_bytes.
size_t scan_temp_bytes(int64_t n);
void exclusive_scan_i32_to_i64(const int32_t *in, int64_t *out, int64_t n, void *temp,
                               cudaStream_t stream);
void exclusive_scan_i64(const int64_t *in, int64_t *out, int64_t n, void *temp,
                        cudaStream_t stream);

}  // namespace dg

struct dg_plan;
namespace dg {
// Frees the Bitshuffle/LZ4 staging, copy stream and events of a plan (dg_bslz4.cu).
void bslz4_release(dg_plan *plan);
// Creates the plan's copy stream and its two pairs of slot events if missing
// (dg_bslz4.cu).
void ensure_copy_pipeline(dg_plan *plan);
}  // namespace dg

struct dg_plan {
    std::mutex mu;
    int32_t device = 0;
    cudaStream_t stream = nullptr;
    dg_geometry geometry{};
    dg_method method{};
    int32_t dim1 = 0, dim2 = 0, n_radial = 0, n_azimuthal = 0;
    int64_t n_bins = 0;
    double hist_min = 0, hist_step = 0;
    double build_ms = 0;
    int64_t guard_corners = 0, singular_pixels = 0;
    int64_t full_entries = 0;
    std::vector<double> radial, azimuthal;
    dg::DeviceCsr full;      // kept with DG_PLAN_KEEP_TABLES
    dg::DeviceCsr table;     // masked, f64 weights (export)
    dg::DeviceArray<double> norm;
    dg::GatherTable gather;
    int64_t max_batch_frames = 0;
    // staging for host-memory calls
    dg::DeviceArray<unsigned char> stage_in;
    dg::DeviceArray<double> stage_out;
    dg::DeviceArray<unsigned char> stage_mask;  // per-frame masks (dg_integrate_dynamic / _raw)
    // compressed frames and their block descriptors (dg_integrate_bslz4)
    dg::DeviceArray<unsigned char> stage_comp;
    dg::DeviceArray<unsigned char> stage_desc;
    // Host-to-device copies of the two-slot host pipelines (dg_integrate's
    // frames, dg_integrate_bslz4's compressed bytes): per slot, copied (the
    // slot landed) and decoded (the device is done reading it).
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t bs_copied[2] = {nullptr, nullptr};
    cudaEvent_t bs_decoded[2] = {nullptr, nullptr};
    dg::EventPool decode_events;  // decode-kernel timing (dg_plan_decode_time)
    size_t decode_smem[2] = {0, 0};  // shared memory granted to the u16 / u32 decoders
    int64_t device_bytes() const;
    ~dg_plan() {
        dg::bslz4_release(this);
        if (stream) cudaStreamDestroy(stream);
    }
};
