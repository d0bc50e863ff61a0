// Per-frame gather: CSR (bins x pixels) times a stack of frames.
//
// Layout. The masked table is cut into segments: a segment is a run of one
// row's entries whose pixels lie in one strip of `strip_rows` detector rows
// (rows list pixels in ascending order, so this is a contiguous range), split
// further to at most kSegMax entries. Within a strip, the segments of
// neighbouring rows are grouped into units of at most kWarps segments and
// unit_cap entries. One CTA owns one unit: it stages the unit's packed entries
// in shared memory once and sweeps every frame of the call over them, so the
// table crosses HBM once per call however many frames there are. Neighbouring
// bins share most pixels (a split pixel falls in ~2.6 bins), and a unit's
// bins cover the same strip of the detector: warps take (segment, frame
// group) tasks in frame-major order, so at any time the CTA's warps read the
// same few kilobytes of the same frames and the repeats are served by L1
// instead of each costing an L2 sector.
//
// A task is (segment, group of kFrameLanes frames); lane (frame, slice)
// reads every kSlices-th staged entry (col, weight[, norm, weight/norm]) and
// gathers that pixel of its frame, kUnroll independent loads at a time; the
// kSlices lanes of a frame then fold their sums.
//
// Arithmetic. Sums are FP32 products accumulated in short plain-FP32 blocks
// (at most kFlush terms per lane) that are folded into a double-word (hi, lo)
// FP32 accumulator with TwoSum; each lane's double-word sum is exact in FP64,
// and lanes, then segments, are added in FP64 in a fixed order. The
// reduction order depends only on the table, never on how many frames a call
// carries, so one frame alone and the same frame inside a batch give
// bit-identical results.
//
// Azimuthal spread (azimuthal.rs:48-118): with x = s/n, w = c*n and origin
// o = x of the row's first valid entry, t = s - o*n (one FMA) gives
// w*(x - o) = c*t and w*(x - o)^2 = (c/n)*t*t, so the shifted moments
// B = sum (c/n)*t*t needs no division per pixel, A = sum c*t equals
// S - o*sum(c*n) and is formed once per row in the finalize, and
// m2 = B - A^2 / sum(w).
#include <algorithm>
#include <type_traits>

#include "dg_internal.h"

namespace dg {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kFlush = 16;  // terms per lane between double-word folds
// Gather lane mappings a plan chooses from (launch_gather), as
// (entry slices per frame group, frames per lane, entries per lane per step):
// 0 (32,4,4), 1 (32,2,8), 2 (8,2,4), 3 (4,1,8), 4 (16,4,2).
constexpr int kVariantCount = 5;
constexpr int kSegMax = 1024;
constexpr int kUnitCap = 3008;  // 16-byte entries in the 48 KB default shared memory

enum Mode { kIntensity = 0, kErrors = 1, kSpread = 2 };

template <typename P>
constexpr bool is_float_px() {
    return std::is_same<P, float>::value || std::is_same<P, double>::value;
}

// Accumulators per (segment, frame): S = sum c*s, then V = sum c^2*max(s,0),
// then for the spread B = sum (c/n)*t^2, then for float pixels the weight
// c*n and the count of non-finite pixels. The spread's first moment
// A = sum c*t = S - o*sum c*n is formed in the finalize.
template <int MODE, typename P>
struct NAcc {
    static constexpr int value =
        MODE == kIntensity ? 1 : MODE == kErrors ? 2 : (is_float_px<P>() ? 5 : 3);
};

template <typename P>
constexpr bool is_unsigned_px() {
    return std::is_same<P, uint16_t>::value || std::is_same<P, uint32_t>::value;
}

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

// Origin o = s/n of the row's first valid entry in this frame
// (azimuthal.rs:80-82): entries that are statically invalid carry c = 0, and
// for float pixels a non-finite value moves on to the next entry.
template <typename P>
__device__ __forceinline__ float row_origin(const float4 *__restrict__ entry_std, int first,
                                            int row_end, const P *__restrict__ frame) {
    if (first < 0) return 0.f;
    int k = first;
    float4 e = entry_std[k];
    float s = load_px<P>(frame, uint32_t(__float_as_int(e.x)));
    if (is_float_px<P>()) {
        while (!isfinite(s) && ++k < row_end) {
            e = entry_std[k];
            if (e.y > 0.f) s = load_px<P>(frame, uint32_t(__float_as_int(e.x)));
        }
    }
    return __fdiv_rn(s, e.z);
}

// Reduce-scatter of V values (a power of two, <= 32) across the 32 lanes of
// a warp by a fixed butterfly: after the call, lanes 2i and 2i+1 (V = 16),
// or lanes with (lane >> log2(32/V)) == i in general, hold value i summed over
// all lanes. IEEE addition is commutative, so the result does not depend on
// which partner adds which.
template <int V>
__device__ __forceinline__ double reduce_scatter(double (&v)[V], int lane) {
    int cur = V;
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) {
        if (cur > 1) {
            const bool hi = (lane & m) != 0;
            const int half = cur / 2;
#pragma unroll
            for (int i = 0; i < V / 2; ++i) {
                if (i < half) {
                    const double send = hi ? v[i] : v[i + half];
                    const double keep = hi ? v[i + half] : v[i];
                    v[i] = __dadd_rn(keep, __shfl_xor_sync(0xffffffffu, send, m));
                }
            }
            cur = half;
        } else {
            v[0] = __dadd_rn(v[0], __shfl_xor_sync(0xffffffffu, v[0], m));
        }
    }
    return v[0];
}

// One CTA per unit; see the file comment. Template parameters choose the
// lane mapping: SLICES lanes split a segment's entries (lane sl takes entries
// sl, sl + SLICES, ...), 32 / SLICES lane groups take different frames, and
// each lane carries FPL frames, so a task is (segment, 32 / SLICES * FPL
// frames). U entries per lane per step have all their loads in flight.
template <int MODE, typename P, int SLICES, int FPL, int U>
__global__ void __launch_bounds__(kThreads)
    k_gather(const int2 *__restrict__ units, const int4 *__restrict__ segs,
             const int2 *__restrict__ entry, const float4 *__restrict__ entry_std,
             const int32_t *__restrict__ first_valid, const P *__restrict__ frames,
             int64_t n_pixels, int n_frames, int n_segments, double *__restrict__ partial) {
    constexpr int NA = NAcc<MODE, P>::value;
    constexpr int GROUPS = 32 / SLICES;         // frame lane groups per warp
    constexpr int TASK_FRAMES = GROUPS * FPL;  // frames per task
    static_assert(kFlush % U == 0, "flush cadence must be a multiple of the unroll");
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_off[kWarps + 1];
    const int2 un = units[blockIdx.x];
    const int seg0 = un.x, nseg = un.y;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        int o = 0;
        for (int i = 0; i < nseg; ++i) {
            s_off[i] = o;
            const int4 sg = segs[seg0 + i];
            o += sg.z - sg.y;
        }
        s_off[nseg] = o;
    }
    __syncthreads();
    // Stage the unit's entries (16- or 8-byte vector copies, segment by segment).
    for (int i = 0; i < nseg; ++i) {
        const int4 sg = segs[seg0 + i];
        const int len = sg.z - sg.y, off = s_off[i];
        if (MODE == kSpread) {
            float4 *st = reinterpret_cast<float4 *>(smem) + off;
            for (int j = threadIdx.x; j < len; j += kThreads) st[j] = entry_std[sg.y + j];
        } else {
            int2 *st = reinterpret_cast<int2 *>(smem) + off;
            for (int j = threadIdx.x; j < len; j += kThreads) st[j] = entry[sg.y + j];
        }
    }
    __syncthreads();

    const int sl = lane % SLICES, fg = lane / SLICES;
    const int groups = (n_frames + TASK_FRAMES - 1) / TASK_FRAMES;
    int grp = 0, si = warp;
    // Frame-major task order: the CTA's warps work on the same frames at once.
    for (;; si += kWarps) {
        while (si >= nseg) {
            si -= nseg;
            ++grp;
        }
        if (grp >= groups) break;
        const int4 sg = segs[seg0 + si];
        const int row = sg.x, len = sg.z - sg.y, off = s_off[si];
        const int fbase = grp * TASK_FRAMES + fg * FPL;
        const P *fr[FPL];
        bool fv[FPL];
#pragma unroll
        for (int q = 0; q < FPL; ++q) {
            fv[q] = fbase + q < n_frames;
            fr[q] = frames + int64_t(fv[q] ? fbase + q : 0) * n_pixels;
        }
        float origin[FPL];
#pragma unroll
        for (int q = 0; q < FPL; ++q)
            origin[q] = MODE == kSpread ? row_origin<P>(entry_std, first_valid[row], sg.w, fr[q])
                                        : 0.f;
        AccDW acc[FPL][NA];
#pragma unroll
        for (int q = 0; q < FPL; ++q)
#pragma unroll
            for (int a = 0; a < NA; ++a) acc[q][a].zero();

        // One step: U entries of this lane, all loads issued before use.
        // CHECK is true only for the last, partial step, whose entries past
        // the segment end contribute zero without touching the frame.
        auto step = [&](int j0, auto check) {
            constexpr bool CHECK = decltype(check)::value;
            if (MODE == kSpread) {
                float4 e[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int j = j0 + SLICES * u;
                    if (CHECK)
                        e[u] = j < len ? reinterpret_cast<const float4 *>(smem)[off + j]
                                       : make_float4(0.f, 0.f, 1.f, 0.f);
                    else
                        e[u] = reinterpret_cast<const float4 *>(smem)[off + j];
                }
                float sv[U][FPL];
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int q = 0; q < FPL; ++q)
                        sv[u][q] = !CHECK || j0 + SLICES * u < len
                                       ? load_px<P>(fr[q], uint32_t(__float_as_int(e[u].x)))
                                       : 0.f;
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const float c = e[u].y, n = e[u].z, cr = e[u].w;
                    const float c2 = __fmul_rn(c, c);
#pragma unroll
                    for (int q = 0; q < FPL; ++q) {
                        const float v = sv[u][q];
                        if (is_float_px<P>() && !isfinite(v)) {
                            acc[q][NA - 2].add(__fmul_rn(c, n));
                            acc[q][NA - 1].add(c > 0.f ? 1.f : 0.f);
                            continue;
                        }
                        acc[q][0].fma(c, v);
                        acc[q][1].fma(c2, is_unsigned_px<P>() ? v : fmaxf(v, 0.f));
                        const float t = __fmaf_rn(-origin[q], n, v);
                        acc[q][2].fma(__fmul_rn(cr, t), t);
                    }
                }
            } else {
                int2 e[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int j = j0 + SLICES * u;
                    if (CHECK)
                        e[u] = j < len ? reinterpret_cast<const int2 *>(smem)[off + j]
                                       : make_int2(0, 0);
                    else
                        e[u] = reinterpret_cast<const int2 *>(smem)[off + j];
                }
                float sv[U][FPL];
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int q = 0; q < FPL; ++q)
                        sv[u][q] = !CHECK || j0 + SLICES * u < len
                                       ? load_px<P>(fr[q], uint32_t(e[u].x))
                                       : 0.f;
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const float c = __int_as_float(e[u].y);
                    const float c2 = __fmul_rn(c, c);
#pragma unroll
                    for (int q = 0; q < FPL; ++q) {
                        acc[q][0].fma(c, sv[u][q]);
                        if (MODE == kErrors)
                            acc[q][1].fma(c2, is_unsigned_px<P>() ? sv[u][q] : fmaxf(sv[u][q], 0.f));
                    }
                }
            }
        };
        int since = 0;
        const int full = len / (SLICES * U) * (SLICES * U);
        int j0 = sl;
        for (; j0 < full; j0 += SLICES * U) {
            step(j0, std::false_type{});
            since += U;
            if (since == kFlush) {
                since = 0;
#pragma unroll
                for (int q = 0; q < FPL; ++q)
#pragma unroll
                    for (int a = 0; a < NA; ++a) acc[q][a].flush();
            }
        }
        if (full < len) step(j0, std::true_type{});
#pragma unroll
        for (int q = 0; q < FPL; ++q)
#pragma unroll
            for (int a = 0; a < NA; ++a) acc[q][a].flush();

        // Each lane's double-word sums are exact in FP64; the SLICES lanes of
        // a frame group are added by a fixed tree.
        if constexpr (SLICES == 32) {
            constexpr int V0 = FPL * NA;
            constexpr int V = V0 <= 1 ? 1 : V0 <= 2 ? 2 : V0 <= 4 ? 4 : V0 <= 8 ? 8 : V0 <= 16 ? 16 : 32;
            double d[V];
#pragma unroll
            for (int i = 0; i < V; ++i) d[i] = 0.0;
#pragma unroll
            for (int q = 0; q < FPL; ++q)
#pragma unroll
                for (int a = 0; a < NA; ++a)
                    d[q * NA + a] = double(acc[q][a].hi) + double(acc[q][a].lo);
            const double mine = reduce_scatter<V>(d, lane);
            const int idx = lane / (32 / V);
            if (lane % (32 / V) == 0 && idx < V0) {
                const int q = idx / NA, a = idx % NA;
                if (fbase + q < n_frames)
                    partial[(int64_t(fbase + q) * n_segments + seg0 + si) * NA + a] = mine;
            }
        } else {
            double d[FPL][NA];
#pragma unroll
            for (int q = 0; q < FPL; ++q)
#pragma unroll
                for (int a = 0; a < NA; ++a) {
                    double x = double(acc[q][a].hi) + double(acc[q][a].lo);
#pragma unroll
                    for (int o = SLICES / 2; o > 0; o >>= 1)
                        x = __dadd_rn(x, __shfl_down_sync(0xffffffffu, x, o));
                    d[q][a] = x;
                }
            if (sl == 0) {
#pragma unroll
                for (int q = 0; q < FPL; ++q) {
                    if (!fv[q]) continue;
                    double *out = partial + (int64_t(fbase + q) * n_segments + seg0 + si) * NA;
#pragma unroll
                    for (int a = 0; a < NA; ++a) out[a] = d[q][a];
                }
            }
        }
    }
}

// One thread per (frame, row): fold the row's segment partials in strip
// order in FP64 and normalise (normalize_bin, prepared.rs:985-996; the
// spread's closing formulas, azimuthal.rs:96-104).
template <int MODE, typename P>
__global__ void k_finalize(const double *__restrict__ partial, const int32_t *__restrict__ row_seg,
                           const int32_t *__restrict__ seg_ids, const int4 *__restrict__ segs,
                           const double *__restrict__ den, const double *__restrict__ den_std,
                           const double *__restrict__ den_f32,
                           const int32_t *__restrict__ valid_std,
                           const int32_t *__restrict__ first_valid,
                           const float4 *__restrict__ entry_std, const P *__restrict__ frames,
                           int64_t n_pixels, int n_rows, int n_segments, int n_frames,
                           double *__restrict__ out_i, double *__restrict__ out_s,
                           double *__restrict__ out_d) {
    constexpr int NA = NAcc<MODE, P>::value;
    int64_t id = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (id >= int64_t(n_rows) * n_frames) return;
    int f = int(id / n_rows), r = int(id % n_rows);
    double v[NA];
    for (int a = 0; a < NA; ++a) v[a] = 0.0;
    const int k0 = row_seg[r], k1 = row_seg[r + 1];
    for (int k = k0; k < k1; ++k) {
        const double *p = partial + (int64_t(f) * n_segments + seg_ids[k]) * NA;
        for (int a = 0; a < NA; ++a) v[a] = __dadd_rn(v[a], p[a]);
    }
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
    int valid = valid_std[r];
    double sw = den_std[r], wf = den_f32[r];
    if (NA == 5) {
        valid -= int(v[4] + 0.5);
        sw -= v[3];
        wf -= v[3];
    }
    if (valid <= 0 || !(sw > 0.0)) {
        out_i[o] = 0.0;
        if (out_s) out_s[o] = 0.0;
        out_d[o] = __longlong_as_double(0x7ff8000000000000ll);
        return;
    }
    // A = sum c*(s - o*n) = S - o * sum c*n over the same FP32 weights.
    const int row_end = k0 < k1 ? segs[seg_ids[k0]].w : 0;
    const float org = row_origin<P>(entry_std, first_valid[r], row_end, frames + int64_t(f) * n_pixels);
    const double a1 = v[0] - double(org) * wf;
    out_i[o] = v[0] / sw;
    if (out_s) out_s[o] = sqrt(v[1] > 0.0 ? v[1] : 0.0) / sw;
    const double mean = a1 / sw;
    const double m2 = v[2] - mean * a1;
    const double q = m2 / sw;
    out_d[o] = sqrt(q > 0.0 ? q : 0.0);
}

// Packs the masked f64 table into the gather's entry formats and computes
// the spread's denominators over its valid entries (c > 0, n > 0, finite).
__global__ void k_pack(const int64_t *__restrict__ row_ptr, int n_rows,
                       const int32_t *__restrict__ col, const double *__restrict__ w,
                       const double *__restrict__ norm, int2 *__restrict__ entry,
                       float4 *__restrict__ entry_std, double *__restrict__ den_std,
                       double *__restrict__ den_f32, int32_t *__restrict__ valid_std,
                       int32_t *__restrict__ first_valid) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    double sw = 0.0, swf = 0.0;
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
            swf += double(cf) * double(nf);
            ++valid;
            if (first < 0) first = int(k);
        }
    }
    den_std[r] = sw;
    den_f32[r] = swf;
    valid_std[r] = valid;
    first_valid[r] = first;
}

// bounds[r * (n_strips + 1) + s]: first entry of row r whose pixel lies in
// strip s or later (columns within a row are ascending).
__global__ void k_strip_bounds(const int64_t *__restrict__ row_ptr, int n_rows,
                               const int32_t *__restrict__ col, int n_strips, int64_t strip_px,
                               int32_t *__restrict__ bounds) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    int64_t b = row_ptr[r], e = row_ptr[r + 1];
    int32_t *out = bounds + int64_t(r) * (n_strips + 1);
    for (int s = 0; s <= n_strips; ++s) {
        int64_t key = int64_t(s) * strip_px, lo = b, hi = e;
        while (lo < hi) {
            int64_t mid = (lo + hi) >> 1;
            if (int64_t(col[mid]) < key) lo = mid + 1;
            else hi = mid;
        }
        out[s] = int32_t(lo);
    }
}

// Launches lane-mapping variant `variant` of the gather (kVariantCount) with
// its partial sums in `partial`.
template <int MODE, typename P>
void launch_gather(const GatherTable &t, int variant, const P *fp, int64_t n_pixels, int nf,
                   double *partial, cudaStream_t s) {
    const size_t smem = size_t(t.unit_cap) * (MODE == kSpread ? 16 : 8);
#define DG_GATHER_ARGS                                                                        \
    t.unit.ptr, t.seg.ptr, t.entry.ptr, t.entry_std.ptr, t.first_valid.ptr, fp, n_pixels, nf, \
        t.n_segments, partial
    switch (variant) {
    case 0: k_gather<MODE, P, 32, 4, 4><<<t.n_units, kThreads, smem, s>>>(DG_GATHER_ARGS); break;
    case 1: k_gather<MODE, P, 32, 2, 8><<<t.n_units, kThreads, smem, s>>>(DG_GATHER_ARGS); break;
    case 2: k_gather<MODE, P, 8, 2, 4><<<t.n_units, kThreads, smem, s>>>(DG_GATHER_ARGS); break;
    case 3: k_gather<MODE, P, 4, 1, 8><<<t.n_units, kThreads, smem, s>>>(DG_GATHER_ARGS); break;
    default: k_gather<MODE, P, 16, 4, 2><<<t.n_units, kThreads, smem, s>>>(DG_GATHER_ARGS); break;
    }
#undef DG_GATHER_ARGS
    DG_CUDA(cudaGetLastError());
}

template <typename P>
void launch_typed(GatherTable &t, const void *frames, int64_t n_pixels, int n_frames, int mode,
                  cudaStream_t s) {
    const P *fp = static_cast<const P *>(frames);
    if (mode == kSpread) launch_gather<kSpread, P>(t, t.variant, fp, n_pixels, n_frames, t.partial.ptr, s);
    else if (mode == kErrors) launch_gather<kErrors, P>(t, t.variant, fp, n_pixels, n_frames, t.partial.ptr, s);
    else launch_gather<kIntensity, P>(t, t.variant, fp, n_pixels, n_frames, t.partial.ptr, s);
}

template <int MODE, typename P>
void launch_finalize(GatherTable &t, const void *frames, int64_t n_pixels, int nf, double *oi,
                     double *os, double *od, cudaStream_t s) {
    const int64_t total = int64_t(t.n_rows) * nf;
    const unsigned blocks = unsigned((total + 255) / 256);
    k_finalize<MODE, P><<<blocks, 256, 0, s>>>(
        t.partial.ptr, t.row_seg.ptr, t.seg_ids.ptr, t.seg.ptr, t.den.ptr, t.den_std.ptr,
        t.den_f32.ptr, t.valid_std.ptr, t.first_valid.ptr, t.entry_std.ptr,
        static_cast<const P *>(frames), n_pixels, t.n_rows, t.n_segments, nf, oi, os, od);
    DG_CUDA(cudaGetLastError());
}

template <typename P>
void finalize_typed(GatherTable &t, int mode, const void *frames, int64_t n_pixels, int nf,
                    double *oi, double *os, double *od, cudaStream_t s) {
    if (mode == kSpread) launch_finalize<kSpread, P>(t, frames, n_pixels, nf, oi, os, od, s);
    else if (mode == kErrors) launch_finalize<kErrors, P>(t, frames, n_pixels, nf, oi, os, od, s);
    else launch_finalize<kIntensity, P>(t, frames, n_pixels, nf, oi, os, od, s);
}

}  // namespace

int gather_launches_per_call() { return 2; }

void gather_kernel_time(GatherTable &t, bool reset, double *ms, int64_t *gather_launches,
                        int64_t *launches) {
    double total = 0.0;
    EventPool &p = t.events;
    if (p.used) DG_CUDA(cudaEventSynchronize(p.events[p.used - 1].second));
    for (size_t i = 0; i < p.used; ++i) {
        float m = 0.f;
        DG_CUDA(cudaEventElapsedTime(&m, p.events[i].first, p.events[i].second));
        total += m;
    }
    if (ms) *ms = total;
    if (gather_launches) *gather_launches = int64_t(p.used);
    if (launches) *launches = t.launches;
    if (reset) {
        p.used = 0;
        t.launches = 0;
    }
}

void make_gather_table(const DeviceCsr &table, const double *d_norm, int32_t dim1, int32_t dim2,
                       int32_t strip_rows, cudaStream_t s, GatherTable &out) {
    out.n_rows = int32_t(table.n_rows);
    out.nnz = table.nnz;
    out.unit_cap = kUnitCap;
    out.strip_rows = strip_rows;
    out.entry.alloc(size_t(table.nnz));
    out.entry_std.alloc(size_t(table.nnz));
    out.den.alloc(size_t(table.n_rows));
    out.den_std.alloc(size_t(table.n_rows));
    out.den_f32.alloc(size_t(table.n_rows));
    out.valid_std.alloc(size_t(table.n_rows));
    out.first_valid.alloc(size_t(table.n_rows));
    denominators(table, d_norm, s, out.den.ptr);
    const unsigned rb = unsigned((table.n_rows + 127) / 128);
    if (table.n_rows > 0)
        k_pack<<<rb, 128, 0, s>>>(table.row_ptr.ptr, int(table.n_rows), table.col.ptr, table.w.ptr,
                                  d_norm, out.entry.ptr, out.entry_std.ptr, out.den_std.ptr,
                                  out.den_f32.ptr, out.valid_std.ptr, out.first_valid.ptr);
    DG_CUDA(cudaGetLastError());

    // Segments: (row, strip) runs from per-row strip bounds found on the
    // device; grouped into units on the host (a few hundred thousand at most).
    const int n_strips = (dim1 + strip_rows - 1) / strip_rows;
    const int64_t nb = table.n_rows;
    DeviceArray<int32_t> bounds;
    bounds.alloc(size_t(nb * (n_strips + 1)));
    if (nb > 0)
        k_strip_bounds<<<rb, 128, 0, s>>>(table.row_ptr.ptr, int(nb), table.col.ptr, n_strips,
                                          int64_t(strip_rows) * dim2, bounds.ptr);
    DG_CUDA(cudaGetLastError());
    std::vector<int32_t> hb(size_t(nb * (n_strips + 1)));
    std::vector<int64_t> rp(size_t(nb) + 1);
    if (!hb.empty())
        DG_CUDA(cudaMemcpyAsync(hb.data(), bounds.ptr, hb.size() * 4, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaMemcpyAsync(rp.data(), table.row_ptr.ptr, rp.size() * 8, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));

    std::vector<int4> segs;
    std::vector<int2> units;
    std::vector<int32_t> seg_count(size_t(nb), 0);
    for (int st = 0; st < n_strips; ++st) {
        int unit_first = int(segs.size()), unit_entries = 0;
        auto close_unit = [&]() {
            if (int(segs.size()) > unit_first)
                units.push_back(make_int2(unit_first, int(segs.size()) - unit_first));
            unit_first = int(segs.size());
            unit_entries = 0;
        };
        for (int64_t r = 0; r < nb; ++r) {
            const int32_t *b = hb.data() + r * (n_strips + 1);
            for (int32_t lo = b[st]; lo < b[st + 1]; lo += kSegMax) {
                int32_t hi = std::min<int32_t>(lo + kSegMax, b[st + 1]);
                int len = hi - lo;
                if (int(segs.size()) - unit_first == kWarps || unit_entries + len > kUnitCap)
                    close_unit();
                segs.push_back(make_int4(int(r), lo, hi, int(rp[size_t(r) + 1])));
                unit_entries += len;
                seg_count[size_t(r)]++;
            }
        }
        close_unit();
    }
    // Row -> its segments, in strip order (the finalize's fixed fold order).
    std::vector<int32_t> row_seg(size_t(nb) + 1, 0), seg_ids(segs.size());
    for (int64_t r = 0; r < nb; ++r) row_seg[size_t(r) + 1] = row_seg[size_t(r)] + seg_count[size_t(r)];
    std::vector<int32_t> fill(row_seg.begin(), row_seg.end() - 1);
    for (size_t i = 0; i < segs.size(); ++i) seg_ids[size_t(fill[size_t(segs[i].x)]++)] = int32_t(i);
    out.n_segments = int32_t(segs.size());
    out.n_units = int32_t(units.size());
    out.seg.alloc(std::max<size_t>(segs.size(), 1));
    out.unit.alloc(std::max<size_t>(units.size(), 1));
    out.seg_ids.alloc(std::max<size_t>(seg_ids.size(), 1));
    out.row_seg.alloc(row_seg.size());
    if (!segs.empty()) {
        DG_CUDA(cudaMemcpyAsync(out.seg.ptr, segs.data(), segs.size() * sizeof(int4),
                                cudaMemcpyHostToDevice, s));
        DG_CUDA(cudaMemcpyAsync(out.unit.ptr, units.data(), units.size() * sizeof(int2),
                                cudaMemcpyHostToDevice, s));
        DG_CUDA(cudaMemcpyAsync(out.seg_ids.ptr, seg_ids.data(), seg_ids.size() * 4,
                                cudaMemcpyHostToDevice, s));
    }
    DG_CUDA(cudaMemcpyAsync(out.row_seg.ptr, row_seg.data(), row_seg.size() * 4,
                            cudaMemcpyHostToDevice, s));
    DG_CUDA(cudaStreamSynchronize(s));
}

void run_gather(GatherTable &t, const void *d_frames, int dtype, int64_t n_pixels,
                int64_t n_frames, uint32_t flags, int precision, double *d_i, double *d_sigma,
                double *d_std, cudaStream_t s) {
    (void)precision;
    if (n_frames <= 0) return;
    if (dtype < DG_U16 || dtype > DG_F64) fail(DG_INVALID_INPUT, "unknown pixel dtype");
    const int mode = (flags & DG_AZIMUTHAL_STD) ? kSpread : (flags & DG_ERRORS) ? kErrors
                                                                                : kIntensity;
    // Frames per launch bounded by the partial-sum scratch (256 frames).
    const int64_t chunk = 256;
    const int64_t need = std::max<int64_t>(1, t.n_segments) * chunk * 5;
    if (t.partial.count < size_t(need)) t.partial.alloc(size_t(need));
    const size_t esize = dtype == DG_U16 ? 2 : dtype == DG_F64 ? 8 : 4;
    for (int64_t f0 = 0; f0 < n_frames; f0 += chunk) {
        const int nf = int(std::min<int64_t>(chunk, n_frames - f0));
        const void *fp = static_cast<const unsigned char *>(d_frames) + f0 * n_pixels * esize;
        if (t.n_units > 0) {
            std::pair<cudaEvent_t, cudaEvent_t> *ev = nullptr;
            if (t.profile) {
                EventPool &p = t.events;
                if (p.used == p.events.size()) {
                    std::pair<cudaEvent_t, cudaEvent_t> e{};
                    DG_CUDA(cudaEventCreate(&e.first));
                    DG_CUDA(cudaEventCreate(&e.second));
                    p.events.push_back(e);
                }
                ev = &p.events[p.used++];
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
        double *oi = d_i + f0 * t.n_rows;
        double *os = d_sigma ? d_sigma + f0 * t.n_rows : nullptr;
        double *od = d_std ? d_std + f0 * t.n_rows : nullptr;
        if (t.n_rows > 0) {
            ++t.launches;
            switch (dtype) {
            case DG_U16: finalize_typed<uint16_t>(t, mode, fp, n_pixels, nf, oi, os, od, s); break;
            case DG_U32: finalize_typed<uint32_t>(t, mode, fp, n_pixels, nf, oi, os, od, s); break;
            case DG_I32: finalize_typed<int32_t>(t, mode, fp, n_pixels, nf, oi, os, od, s); break;
            case DG_F32: finalize_typed<float>(t, mode, fp, n_pixels, nf, oi, os, od, s); break;
            case DG_F64: finalize_typed<double>(t, mode, fp, n_pixels, nf, oi, os, od, s); break;
            }
        }
    }
}

namespace {

template <typename P>
void launch_mode(GatherTable &t, int variant, int mode, const void *frames, int64_t n_pixels,
                 int nf, cudaStream_t s) {
    const P *fp = static_cast<const P *>(frames);
    if (mode == kSpread) launch_gather<kSpread, P>(t, variant, fp, n_pixels, nf, t.partial.ptr, s);
    else if (mode == kErrors) launch_gather<kErrors, P>(t, variant, fp, n_pixels, nf, t.partial.ptr, s);
    else launch_gather<kIntensity, P>(t, variant, fp, n_pixels, nf, t.partial.ptr, s);
}

}  // namespace

int gather_variant_count() { return kVariantCount; }

int autotune_gather(GatherTable &t, const void *d_frames, int dtype, int64_t n_pixels,
                    int64_t n_frames, uint32_t flags, cudaStream_t s,
                    std::vector<double> *each) {
    if (dtype < DG_U16 || dtype > DG_F64) fail(DG_INVALID_INPUT, "unknown pixel dtype");
    if (n_frames <= 0) fail(DG_INVALID_INPUT, "autotuning needs at least one frame");
    const int mode = (flags & DG_AZIMUTHAL_STD) ? kSpread : (flags & DG_ERRORS) ? kErrors
                                                                                : kIntensity;
    const int nf = int(std::min<int64_t>(n_frames, 256));
    const int64_t need = std::max<int64_t>(1, t.n_segments) * 256 * 5;
    if (t.partial.count < size_t(need)) t.partial.alloc(size_t(need));
    if (each) each->assign(size_t(kVariantCount), 0.0);
    if (t.n_units == 0) return t.variant;
    cudaEvent_t a = nullptr, b = nullptr;
    DG_CUDA(cudaEventCreate(&a));
    DG_CUDA(cudaEventCreate(&b));
    int best = t.variant;
    float best_t = 3.4e38f;
    try {
        for (int v = 0; v < kVariantCount; ++v) {
            float vt = 3.4e38f;
            for (int rep = 0; rep < 4; ++rep) {
                DG_CUDA(cudaEventRecord(a, s));
                switch (dtype) {
                case DG_U16: launch_mode<uint16_t>(t, v, mode, d_frames, n_pixels, nf, s); break;
                case DG_U32: launch_mode<uint32_t>(t, v, mode, d_frames, n_pixels, nf, s); break;
                case DG_I32: launch_mode<int32_t>(t, v, mode, d_frames, n_pixels, nf, s); break;
                case DG_F32: launch_mode<float>(t, v, mode, d_frames, n_pixels, nf, s); break;
                case DG_F64: launch_mode<double>(t, v, mode, d_frames, n_pixels, nf, s); break;
                }
                DG_CUDA(cudaEventRecord(b, s));
                DG_CUDA(cudaEventSynchronize(b));
                float ms = 0.f;
                DG_CUDA(cudaEventElapsedTime(&ms, a, b));
                if (rep > 0 && ms < vt) vt = ms;  // first launch warms caches
            }
            if (each) (*each)[size_t(v)] = vt;
            if (vt < best_t) {
                best_t = vt;
                best = v;
            }
        }
    } catch (...) {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        throw;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    t.variant = best;
    return best;
}

}  // namespace dg

// ---------------------------------------------------------------------------
// Allocation-free integration (dg_integrate_device_noalloc).
//
// For callers that must not allocate device memory while they integrate: a
// real-time acquisition loop with a fixed memory budget, a host thread that
// may not enter the CUDA allocator, or code running where cudaMalloc is not
// permitted. dg_integrate_device allocates its per-segment partial sums on
// first use; this variant keeps them in one fixed array in the library
// instead, so after the plan exists nothing is allocated. The plan itself is
// created beforehand with dg_plan_create, which does allocate.
//
// The array is a file-scope __device__ variable of kNoAllocScratchBytes. Host
// code cannot use its name as a device address, so its address is obtained
// with cudaGetSymbolAddress once per device, with that device current, on
// the first call on that device; make that first call before any stream
// capture. Every call on a device shares the one array: calls that overlap on
// the GPU (from different streams or threads) race on it, so serialise them.
// Every partial sum the finalize reads is written by the gather kernel of the
// same call, so nothing needs clearing between calls.
namespace dg {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB per device
constexpr size_t kNoAllocScratchDoubles = kNoAllocScratchBytes / sizeof(double);
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_partial[kNoAllocScratchDoubles];

std::mutex g_noalloc_mu;
double *g_noalloc_ptr[kNoAllocMaxDevices] = {};

// The array's device address on `device` (current), resolved once.
double *noalloc_scratch(int device) {
    if (device < 0 || device >= kNoAllocMaxDevices)
        fail(DG_UNSUPPORTED, "device ordinal beyond the allocation-free path's table");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partial);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            fail(DG_DEVICE, std::string("cudaGetSymbolAddress of the scratch array failed: ") +
                                cudaGetErrorString(e));
        }
        g_noalloc_ptr[device] = static_cast<double *>(p);
    }
    return g_noalloc_ptr[device];
}

template <typename P>
void noalloc_launch(const GatherTable &t, double *partial, const void *frames, int64_t n_pixels,
                    int nf, int mode, double *oi, double *os, double *od, cudaStream_t s) {
    const P *fp = static_cast<const P *>(frames);
    if (t.n_units > 0) {
        if (mode == kSpread) launch_gather<kSpread, P>(t, t.variant, fp, n_pixels, nf, partial, s);
        else if (mode == kErrors) launch_gather<kErrors, P>(t, t.variant, fp, n_pixels, nf, partial, s);
        else launch_gather<kIntensity, P>(t, t.variant, fp, n_pixels, nf, partial, s);
    }
    if (t.n_rows > 0) {
        const unsigned blocks = unsigned((int64_t(t.n_rows) * nf + 255) / 256);
#define DG_NOALLOC_FINALIZE(M)                                                                 \
    k_finalize<M, P><<<blocks, 256, 0, s>>>(                                                   \
        partial, t.row_seg.ptr, t.seg_ids.ptr, t.seg.ptr, t.den.ptr, t.den_std.ptr,           \
        t.den_f32.ptr, t.valid_std.ptr, t.first_valid.ptr, t.entry_std.ptr, fp, n_pixels,      \
        t.n_rows, t.n_segments, nf, oi, os, od)
        if (mode == kSpread) DG_NOALLOC_FINALIZE(kSpread);
        else if (mode == kErrors) DG_NOALLOC_FINALIZE(kErrors);
        else DG_NOALLOC_FINALIZE(kIntensity);
#undef DG_NOALLOC_FINALIZE
        DG_CUDA(cudaGetLastError());
    }
}

}  // namespace
}  // namespace dg

extern "C" dg_status dg_integrate_device_noalloc(dg_plan *plan, const void *d_frames,
                                                 int32_t dtype, int64_t n_frames, uint32_t flags,
                                                 double *d_i, double *d_s, double *d_d,
                                                 void *stream) {
    using namespace dg;
    try {
        if (!plan) fail(DG_INVALID_INPUT, "plan must not be NULL");
        if (dtype < DG_U16 || dtype > DG_F64) fail(DG_INVALID_INPUT, "unknown pixel dtype");
        if (n_frames < 0) fail(DG_INVALID_INPUT, "frame count must not be negative");
        if (flags & ~(DG_ERRORS | DG_AZIMUTHAL_STD)) fail(DG_INVALID_INPUT, "unknown flags");
        if (n_frames == 0) return DG_OK;
        if (!d_frames || !d_i) fail(DG_INVALID_INPUT, "frames and intensity must not be NULL");
        if ((flags & DG_ERRORS) && !d_s) fail(DG_INVALID_INPUT, "errors requested without an output");
        if ((flags & DG_AZIMUTHAL_STD) && !d_d)
            fail(DG_INVALID_INPUT, "azimuthal_std requested without an output");
        if ((flags & DG_AZIMUTHAL_STD) && plan->n_azimuthal != 0)
            fail(DG_UNSUPPORTED, "azimuthal_std is defined for 1D tables only");
        std::lock_guard<std::mutex> lock(plan->mu);
        int previous = -1;
        DG_CUDA(cudaGetDevice(&previous));
        if (previous != plan->device) DG_CUDA(cudaSetDevice(plan->device));
        struct Restore {
            int dev;
            ~Restore() {
                int now = -1;
                if (dev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != dev) cudaSetDevice(dev);
            }
        } restore{previous};
        double *scratch = noalloc_scratch(plan->device);
        const GatherTable &t = plan->gather;
        const int mode = (flags & DG_AZIMUTHAL_STD) ? kSpread : (flags & DG_ERRORS) ? kErrors
                                                                                    : kIntensity;
        const bool fpx = dtype == DG_F32 || dtype == DG_F64;
        const int na = mode == kIntensity ? 1 : mode == kErrors ? 2 : (fpx ? 5 : 3);
        const int64_t per_frame = std::max<int64_t>(1, t.n_segments) * na;
        const int64_t chunk = std::min<int64_t>(int64_t(kNoAllocScratchDoubles) / per_frame, 256);
        if (chunk < 1)
            fail(DG_UNSUPPORTED,
                 "this plan needs " + std::to_string(per_frame * 8) +
                     " bytes of partial sums per frame; the allocation-free path holds " +
                     std::to_string(kNoAllocScratchBytes) + " bytes (use dg_integrate_device)");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : plan->stream;
        const int64_t npix = int64_t(plan->dim1) * plan->dim2;
        const size_t es = dtype == DG_U16 ? 2 : dtype == DG_F64 ? 8 : 4;
        for (int64_t f0 = 0; f0 < n_frames; f0 += chunk) {
            const int nf = int(std::min<int64_t>(chunk, n_frames - f0));
            const void *fp = static_cast<const unsigned char *>(d_frames) + f0 * npix * int64_t(es);
            double *oi = d_i + f0 * t.n_rows;
            double *os = (flags & DG_ERRORS) ? d_s + f0 * t.n_rows : nullptr;
            double *od = (flags & DG_AZIMUTHAL_STD) ? d_d + f0 * t.n_rows : nullptr;
            switch (dtype) {
            case DG_U16: noalloc_launch<uint16_t>(t, scratch, fp, npix, nf, mode, oi, os, od, s); break;
            case DG_U32: noalloc_launch<uint32_t>(t, scratch, fp, npix, nf, mode, oi, os, od, s); break;
            case DG_I32: noalloc_launch<int32_t>(t, scratch, fp, npix, nf, mode, oi, os, od, s); break;
            case DG_F32: noalloc_launch<float>(t, scratch, fp, npix, nf, mode, oi, os, od, s); break;
            case DG_F64: noalloc_launch<double>(t, scratch, fp, npix, nf, mode, oi, os, od, s); break;
            }
        }
        return DG_OK;
    } catch (const Error &e) {
        set_last_error(e.message);
        return e.status;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return DG_DEVICE;
    } catch (...) {
        set_last_error("unknown failure");
        return DG_DEVICE;
    }
}
