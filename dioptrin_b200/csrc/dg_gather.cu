// Per-frame gather: CSR (bins x pixels) times a stack of frames.
//
// Layout. The masked table is cut into row segments of at most `seg_len`
// entries (a row never shares a segment with another row). One CTA owns one
// segment: it stages the segment's packed entries in shared memory once and
// then sweeps every frame of the call over them, so the table crosses HBM
// once per call however many frames there are. Warps take frames four at a
// time; a lane reads one staged entry (col, weight[, norm, weight/norm]) and
// applies it to four frames, gathering the four pixel values with independent
// loads. Pixels shared by neighbouring bins are read by neighbouring segments
// at nearly the same time, so the second read is served by L2.
//
// Arithmetic. Sums are FP32 products accumulated in short plain-FP32 blocks
// (at most kFlush terms per lane) that are folded into a double-word (hi, lo)
// FP32 accumulator with TwoSum, then merged across lanes with TwoSum and across
// segments in a fixed order in the finalize pass, which divides in FP64. The
// reduction order depends only on the table, never on how many frames a call
// carries, so one frame alone and the same frame inside a batch give
// bit-identical results.
//
// Azimuthal spread (azimuthal.rs:48-118): with x = s/n, w = c*n and origin
// o = x of the row's first valid entry, t = s - o*n (one FMA) gives
// w*(x - o) = c*t and w*(x - o)^2 = (c/n)*t*t, so the shifted moments
// A = sum c*t and B = sum (c/n)*t*t need no division per pixel and
// m2 = B - A^2 / sum(w).
#include <algorithm>
#include <type_traits>

#include "dg_internal.h"

namespace dg {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kFramesPerPass = 4;
constexpr int kFlush = 16;

enum Mode { kIntensity = 0, kErrors = 1, kSpread = 2 };

template <int MODE>
struct NAcc {
    static constexpr int value = MODE == kIntensity ? 1 : MODE == kErrors ? 2 : 6;
};

// Double-word FP32 accumulator with a plain FP32 block in front.
struct AccDW {
    float p, hi, lo;
    __device__ __forceinline__ void zero() { p = hi = lo = 0.f; }
    __device__ __forceinline__ void fma(float a, float b) { p = __fmaf_rn(a, b, p); }
    __device__ __forceinline__ void add(float a) { p = __fadd_rn(p, a); }
    __device__ __forceinline__ void flush() {
        float s = __fadd_rn(hi, p);
        float bp = __fsub_rn(s, hi);
        float e = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bp)), __fsub_rn(p, bp));
        hi = s;
        lo = __fadd_rn(lo, e);
        p = 0.f;
    }
    // (hi, lo) += (h2, l2), hi keeps the rounded sum.
    __device__ __forceinline__ void merge(float h2, float l2) {
        float s = __fadd_rn(hi, h2);
        if (!(fabsf(s) <= 3.40282347e+38f)) {  // inf or NaN: keep it
            hi = s;
            lo = 0.f;
            return;
        }
        float bp = __fsub_rn(s, hi);
        float e = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bp)), __fsub_rn(h2, bp));
        float t = __fadd_rn(__fadd_rn(e, lo), l2);
        hi = __fadd_rn(s, t);
        lo = __fsub_rn(t, __fsub_rn(hi, s));
    }
};

template <typename P>
__device__ __forceinline__ float load_px(const P *__restrict__ f, uint32_t i) {
    return float(__ldg(f + i));
}
template <>
__device__ __forceinline__ float load_px<double>(const double *__restrict__ f, uint32_t i) {
    return __double2float_rn(__ldg(f + i));
}

template <typename P>
constexpr bool is_float_px() {
    return std::is_same<P, float>::value || std::is_same<P, double>::value;
}

// One CTA per segment; see the file comment.
template <int MODE, typename P>
__global__ void __launch_bounds__(kThreads)
    k_gather(const int4 *__restrict__ segs, const int2 *__restrict__ entry,
             const float4 *__restrict__ entry_std, const int32_t *__restrict__ first_valid,
             const P *__restrict__ frames, int64_t n_pixels, int n_frames, int n_segments,
             float *__restrict__ partial) {
    constexpr int NA = NAcc<MODE>::value;
    extern __shared__ __align__(16) unsigned char smem[];
    const int4 sg = segs[blockIdx.x];
    const int row = sg.x, begin = sg.y, len = sg.z - sg.y;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    // Stage the segment's entries (16-byte vector copies).
    if (MODE == kSpread) {
        float4 *st = reinterpret_cast<float4 *>(smem);
        for (int j = threadIdx.x; j < len; j += kThreads) st[j] = entry_std[begin + j];
    } else {
        int2 *st = reinterpret_cast<int2 *>(smem);
        for (int j = threadIdx.x; j < len; j += kThreads) st[j] = entry[begin + j];
    }
    __syncthreads();

    const int groups = (n_frames + kFramesPerPass - 1) / kFramesPerPass;
    for (int grp = warp; grp < groups; grp += kWarps) {
        const int f0 = grp * kFramesPerPass;
        const P *fr[kFramesPerPass];
        bool fv[kFramesPerPass];
#pragma unroll
        for (int q = 0; q < kFramesPerPass; ++q) {
            fv[q] = f0 + q < n_frames;
            fr[q] = frames + int64_t(fv[q] ? f0 + q : f0) * n_pixels;
        }
        float origin[kFramesPerPass];
        if (MODE == kSpread) {
            // o = s/n of the row's first valid entry (azimuthal.rs:80-82).
            const int fvi = first_valid[row];
#pragma unroll
            for (int q = 0; q < kFramesPerPass; ++q) {
                origin[q] = 0.f;
                if (fvi >= 0) {
                    int k = fvi;
                    float4 e = entry_std[k];
                    float s = load_px<P>(fr[q], uint32_t(__float_as_int(e.x)));
                    if (is_float_px<P>()) {
                        // Skip entries whose pixel is not finite in this frame.
                        const int row_end = sg.w;
                        while (!isfinite(s) && ++k < row_end) {
                            e = entry_std[k];
                            if (e.y > 0.f) s = load_px<P>(fr[q], uint32_t(__float_as_int(e.x)));
                        }
                    }
                    origin[q] = __fdiv_rn(s, e.z);
                }
            }
        }
        AccDW acc[kFramesPerPass][NA];
#pragma unroll
        for (int q = 0; q < kFramesPerPass; ++q)
#pragma unroll
            for (int a = 0; a < NA; ++a) acc[q][a].zero();

        int since = 0;
        for (int j = lane; j < len; j += 32) {
            if (MODE == kSpread) {
                const float4 e = reinterpret_cast<const float4 *>(smem)[j];
                const uint32_t col = uint32_t(__float_as_int(e.x));
                const float c = e.y, n = e.z, cr = e.w;
                const float c2 = __fmul_rn(c, c);
                float s[kFramesPerPass];
#pragma unroll
                for (int q = 0; q < kFramesPerPass; ++q) s[q] = load_px<P>(fr[q], col);
#pragma unroll
                for (int q = 0; q < kFramesPerPass; ++q) {
                    float v = s[q];
                    if (is_float_px<P>() && !isfinite(v)) {
                        acc[q][4].add(__fmul_rn(c, n));
                        acc[q][5].add(c > 0.f ? 1.f : 0.f);
                        continue;
                    }
                    acc[q][0].fma(c, v);
                    acc[q][1].fma(c2, fmaxf(v, 0.f));
                    const float t = __fmaf_rn(-origin[q], n, v);
                    acc[q][2].fma(c, t);
                    acc[q][3].fma(__fmul_rn(cr, t), t);
                }
            } else {
                const int2 e = reinterpret_cast<const int2 *>(smem)[j];
                const uint32_t col = uint32_t(e.x);
                const float c = __int_as_float(e.y);
                float s[kFramesPerPass];
#pragma unroll
                for (int q = 0; q < kFramesPerPass; ++q) s[q] = load_px<P>(fr[q], col);
#pragma unroll
                for (int q = 0; q < kFramesPerPass; ++q) {
                    acc[q][0].fma(c, s[q]);
                    if (MODE == kErrors) acc[q][1].fma(__fmul_rn(c, c), fmaxf(s[q], 0.f));
                }
            }
            if (++since == kFlush) {
                since = 0;
#pragma unroll
                for (int q = 0; q < kFramesPerPass; ++q)
#pragma unroll
                    for (int a = 0; a < NA; ++a) acc[q][a].flush();
            }
        }
#pragma unroll
        for (int q = 0; q < kFramesPerPass; ++q)
#pragma unroll
            for (int a = 0; a < NA; ++a) acc[q][a].flush();
        // Fixed butterfly-free tree: lane i takes lane i + o for o = 16..1.
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int q = 0; q < kFramesPerPass; ++q)
#pragma unroll
                for (int a = 0; a < NA; ++a) {
                    float h2 = __shfl_down_sync(0xffffffffu, acc[q][a].hi, o);
                    float l2 = __shfl_down_sync(0xffffffffu, acc[q][a].lo, o);
                    acc[q][a].merge(h2, l2);
                }
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < kFramesPerPass; ++q) {
                if (!fv[q]) continue;
                float *out = partial + (int64_t(f0 + q) * n_segments + blockIdx.x) * (2 * NA);
#pragma unroll
                for (int a = 0; a < NA; ++a) {
                    out[2 * a] = acc[q][a].hi;
                    out[2 * a + 1] = acc[q][a].lo;
                }
            }
        }
    }
}

// One thread per (frame, row): fold the row's segment partials in order and
// normalise in FP64 (normalize_bin, prepared.rs:985-996; the spread's
// closing formulas, azimuthal.rs:96-104).
template <int MODE>
__global__ void k_finalize(const float *__restrict__ partial, const int32_t *__restrict__ row_seg,
                           const double *__restrict__ den, const double *__restrict__ den_std,
                           const int32_t *__restrict__ valid_std, int n_rows, int n_segments,
                           int n_frames, double *__restrict__ out_i, double *__restrict__ out_s,
                           double *__restrict__ out_d) {
    constexpr int NA = NAcc<MODE>::value;
    int64_t id = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (id >= int64_t(n_rows) * n_frames) return;
    int f = int(id / n_rows), r = int(id % n_rows);
    AccDW acc[NA];
    for (int a = 0; a < NA; ++a) acc[a].zero();
    for (int sgi = row_seg[r]; sgi < row_seg[r + 1]; ++sgi) {
        const float *p = partial + (int64_t(f) * n_segments + sgi) * (2 * NA);
        for (int a = 0; a < NA; ++a) acc[a].merge(p[2 * a], p[2 * a + 1]);
    }
    double v[NA];
    for (int a = 0; a < NA; ++a) v[a] = double(acc[a].hi) + double(acc[a].lo);
    int64_t o = int64_t(f) * n_rows + r;
    if (MODE != kSpread) {
        double n = den[r];
        out_i[o] = n == 0.0 ? 0.0 : v[0] / n;
        if (MODE == kErrors) {
            double q = n == 0.0 ? 0.0 : v[1] / (n * n);
            out_s[o] = sqrt(q > 0.0 ? q : 0.0);
        }
        return;
    }
    int valid = valid_std[r] - int(acc[5].hi + acc[5].lo + 0.5f);
    double sw = den_std[r] - v[4];
    if (valid <= 0 || !(sw > 0.0)) {
        out_i[o] = 0.0;
        if (out_s) out_s[o] = 0.0;
        out_d[o] = __longlong_as_double(0x7ff8000000000000ll);
        return;
    }
    out_i[o] = v[0] / sw;
    if (out_s) out_s[o] = sqrt(v[1] > 0.0 ? v[1] : 0.0) / sw;
    double mean = v[2] / sw;
    double m2 = v[3] - mean * v[2];
    double q = m2 / sw;
    out_d[o] = sqrt(q > 0.0 ? q : 0.0);
}

// Packs the masked f64 table into the gather's entry formats and computes
// the spread's denominators over its valid entries (c > 0, n > 0, finite).
__global__ void k_pack(const int64_t *__restrict__ row_ptr, int n_rows,
                       const int32_t *__restrict__ col, const double *__restrict__ w,
                       const double *__restrict__ norm, int2 *__restrict__ entry,
                       float4 *__restrict__ entry_std, double *__restrict__ den_std,
                       int32_t *__restrict__ valid_std, int32_t *__restrict__ first_valid) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    double sw = 0.0;
    int valid = 0, first = -1;
    for (int64_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
        int32_t j = col[k];
        double c = w[k], n = norm[j];
        double ww = c * n;
        bool ok = isfinite(n) && n > 0.0 && isfinite(c) && c > 0.0 && isfinite(ww) && ww > 0.0;
        float cf = __double2float_rn(c);
        entry[k] = make_int2(j, __float_as_int(cf));
        float nf = __double2float_rn(n);
        entry_std[k] = make_float4(__int_as_float(j), ok ? cf : 0.f, ok ? nf : 1.f,
                                   ok ? __double2float_rn(c / n) : 0.f);
        if (ok) {
            sw += ww;
            ++valid;
            if (first < 0) first = int(k);
        }
    }
    den_std[r] = sw;
    valid_std[r] = valid;
    first_valid[r] = first;
}

template <typename P>
void launch_typed(GatherTable &t, const void *frames, int64_t n_pixels, int n_frames, int mode,
                  cudaStream_t s) {
    const int threads = kThreads;
    const size_t smem = size_t(t.seg_len) * (mode == kSpread ? 16 : 8);
    const P *fp = static_cast<const P *>(frames);
    if (mode == kSpread) {
        k_gather<kSpread, P><<<t.n_segments, threads, smem, s>>>(
            t.seg.ptr, t.entry.ptr, t.entry_std.ptr, t.row_seg.ptr + t.n_rows + 1, fp, n_pixels,
            n_frames, t.n_segments, t.partial.ptr);
    } else if (mode == kErrors) {
        k_gather<kErrors, P><<<t.n_segments, threads, smem, s>>>(
            t.seg.ptr, t.entry.ptr, t.entry_std.ptr, nullptr, fp, n_pixels, n_frames,
            t.n_segments, t.partial.ptr);
    } else {
        k_gather<kIntensity, P><<<t.n_segments, threads, smem, s>>>(
            t.seg.ptr, t.entry.ptr, t.entry_std.ptr, nullptr, fp, n_pixels, n_frames,
            t.n_segments, t.partial.ptr);
    }
    DG_CUDA(cudaGetLastError());
}

}  // namespace

int gather_launches_per_call() { return 2; }

void gather_kernel_time(GatherTable &t, bool reset, double *ms, int64_t *gather_launches,
                        int64_t *launches) {
    double total = 0.0;
    if (t.events_used) DG_CUDA(cudaEventSynchronize(t.events[t.events_used - 1].second));
    for (size_t i = 0; i < t.events_used; ++i) {
        float m = 0.f;
        DG_CUDA(cudaEventElapsedTime(&m, t.events[i].first, t.events[i].second));
        total += m;
    }
    if (ms) *ms = total;
    if (gather_launches) *gather_launches = int64_t(t.events_used);
    if (launches) *launches = t.launches;
    if (reset) {
        t.events_used = 0;
        t.launches = 0;
    }
}

void make_gather_table(const DeviceCsr &table, const double *d_norm, int32_t seg_len,
                       cudaStream_t s, GatherTable &out) {
    out.n_rows = int32_t(table.n_rows);
    out.nnz = table.nnz;
    out.seg_len = seg_len;
    out.entry.alloc(size_t(table.nnz));
    out.entry_std.alloc(size_t(table.nnz));
    out.den.alloc(size_t(table.n_rows));
    out.den_std.alloc(size_t(table.n_rows));
    out.valid_std.alloc(size_t(table.n_rows));
    denominators(table, d_norm, s, out.den.ptr);
    // Segments: rows cut into pieces of at most seg_len entries, on the host
    // from the row pointers (a few thousand to a few hundred thousand rows).
    std::vector<int64_t> rp(size_t(table.n_rows) + 1);
    DG_CUDA(cudaMemcpyAsync(rp.data(), table.row_ptr.ptr, rp.size() * 8, cudaMemcpyDeviceToHost,
                            s));
    DG_CUDA(cudaStreamSynchronize(s));
    std::vector<int4> segs;
    std::vector<int32_t> row_seg(size_t(table.n_rows) + 1);
    for (int64_t r = 0; r < table.n_rows; ++r) {
        row_seg[size_t(r)] = int32_t(segs.size());
        for (int64_t b = rp[size_t(r)]; b < rp[size_t(r) + 1]; b += seg_len) {
            int64_t e = std::min<int64_t>(b + seg_len, rp[size_t(r) + 1]);
            segs.push_back(make_int4(int(r), int(b), int(e), int(rp[size_t(r) + 1])));
        }
    }
    row_seg[size_t(table.n_rows)] = int32_t(segs.size());
    out.n_segments = int32_t(segs.size());
    out.seg.alloc(std::max<size_t>(segs.size(), 1));
    if (!segs.empty())
        DG_CUDA(cudaMemcpyAsync(out.seg.ptr, segs.data(), segs.size() * sizeof(int4),
                                cudaMemcpyHostToDevice, s));
    // row_seg followed by first_valid (n_rows) in one allocation.
    out.row_seg.alloc(size_t(2 * table.n_rows + 1));
    DG_CUDA(cudaMemcpyAsync(out.row_seg.ptr, row_seg.data(), row_seg.size() * 4,
                            cudaMemcpyHostToDevice, s));
    k_pack<<<unsigned((table.n_rows + 127) / 128), 128, 0, s>>>(
        table.row_ptr.ptr, int(table.n_rows), table.col.ptr, table.w.ptr, d_norm, out.entry.ptr,
        out.entry_std.ptr, out.den_std.ptr, out.valid_std.ptr,
        out.row_seg.ptr + table.n_rows + 1);
    DG_CUDA(cudaGetLastError());
    DG_CUDA(cudaStreamSynchronize(s));
}

void run_gather(GatherTable &t, const void *d_frames, int dtype, int64_t n_pixels,
                int64_t n_frames, uint32_t flags, int precision, double *d_i, double *d_sigma,
                double *d_std, cudaStream_t s) {
    (void)precision;
    if (n_frames <= 0) return;
    const int mode = (flags & DG_AZIMUTHAL_STD) ? kSpread : (flags & DG_ERRORS) ? kErrors
                                                                                : kIntensity;
    const int na = mode == kSpread ? 6 : mode == kErrors ? 2 : 1;
    // Frames per launch bounded by the partial-sum scratch (256 frames).
    const int64_t chunk = 256;
    const int64_t need = std::max<int64_t>(1, t.n_segments) * chunk * 2 * 6;
    if (t.partial.count < size_t(need)) t.partial.alloc(size_t(need));
    if (dtype < DG_U16 || dtype > DG_F64) fail(DG_INVALID_INPUT, "unknown pixel dtype");
    const size_t esize = dtype == DG_U16 ? 2 : dtype == DG_F64 ? 8 : 4;
    for (int64_t f0 = 0; f0 < n_frames; f0 += chunk) {
        const int nf = int(std::min<int64_t>(chunk, n_frames - f0));
        const void *fp = static_cast<const unsigned char *>(d_frames) + f0 * n_pixels * esize;
        if (t.n_segments > 0) {
            std::pair<cudaEvent_t, cudaEvent_t> *ev = nullptr;
            if (t.profile) {
                if (t.events_used == t.events.size()) {
                    std::pair<cudaEvent_t, cudaEvent_t> e{};
                    DG_CUDA(cudaEventCreate(&e.first));
                    DG_CUDA(cudaEventCreate(&e.second));
                    t.events.push_back(e);
                }
                ev = &t.events[t.events_used++];
                DG_CUDA(cudaEventRecord(ev->first, s));
            }
            ++t.launches;
            switch (dtype) {
            case DG_U16: launch_typed<uint16_t>(t, fp, n_pixels, nf, mode, s); break;
            case DG_U32: launch_typed<uint32_t>(t, fp, n_pixels, nf, mode, s); break;
            case DG_I32: launch_typed<int32_t>(t, fp, n_pixels, nf, mode, s); break;
            case DG_F32: launch_typed<float>(t, fp, n_pixels, nf, mode, s); break;
            case DG_F64: launch_typed<double>(t, fp, n_pixels, nf, mode, s); break;
            }
            if (ev) DG_CUDA(cudaEventRecord(ev->second, s));
        }
        const int64_t total = int64_t(t.n_rows) * nf;
        const unsigned blocks = unsigned((total + 255) / 256);
        double *oi = d_i + f0 * t.n_rows;
        double *os = d_sigma ? d_sigma + f0 * t.n_rows : nullptr;
        double *od = d_std ? d_std + f0 * t.n_rows : nullptr;
        if (total > 0) {
            ++t.launches;
            if (mode == kSpread)
                k_finalize<kSpread><<<blocks, 256, 0, s>>>(t.partial.ptr, t.row_seg.ptr, t.den.ptr,
                                                           t.den_std.ptr, t.valid_std.ptr, t.n_rows,
                                                           t.n_segments, nf, oi, os, od);
            else if (mode == kErrors)
                k_finalize<kErrors><<<blocks, 256, 0, s>>>(t.partial.ptr, t.row_seg.ptr, t.den.ptr,
                                                           t.den_std.ptr, t.valid_std.ptr, t.n_rows,
                                                           t.n_segments, nf, oi, os, od);
            else
                k_finalize<kIntensity><<<blocks, 256, 0, s>>>(
                    t.partial.ptr, t.row_seg.ptr, t.den.ptr, t.den_std.ptr, t.valid_std.ptr,
                    t.n_rows, t.n_segments, nf, oi, os, od);
            DG_CUDA(cudaGetLastError());
        }
        (void)na;
    }
}

}  // namespace dg
