// Per-frame gather: CSR (bins x pixels) times a stack of frames.
//
// Three families of lane mappings, chosen per plan by timing (the
// autotuner): entry-lane units (k_gather, mappings 0-4, described first
// below), frame-lane units (k_gather_fl, 5-6) and bin tiles (k_gather_bins,
// 7-8). The first two leave per-segment partial sums that k_finalize folds;
// the bin tiles keep each bin's sums in registers for the whole batch and
// write the results themselves.
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
// o = x of one valid entry of the row, t = s - o*n gives w*(x - o) = c*t
// and w*(x - o)^2 = (c/n)*t*t, so the shifted moments A = sum c*t and
// B = sum (c/n)*t*t need no division per pixel, and the reference's second
// pass sum w*((x - o) - A/W)^2 equals m2 = B - A^2/W with W = sum w. The
// shift is exact to the last bit of t: n is kept as an FP32 pair
// (n_hi, n_lo) with n_hi + n_lo = n to 2^-48, t = (s - o*n_hi) - o*n_lo by
// two FMAs, and A is accumulated from the same t (forming it as S - o*W
// instead loses the products' rounding of S to the cancellation). Any
// constant origin gives the same m2 and o only has to be the same for every
// entry of a row, so its FP32 rounding is harmless; its distance from the
// mean sets the cancellation in m2, so o is the row's heaviest valid entry
// (row_origin) rather than the reference's first one.
#include <algorithm>
#include <climits>
#include <type_traits>

#include <array>
#include <atomic>
#include <memory>
#include <thread>

#include "dg_internal.h"

namespace dg {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kFlush = 16;  // terms per lane between double-word folds
// Gather lane mappings a plan chooses from (launch_gather). Entry-lane
// mappings, as (entry slices per frame group, frames per lane, entries per
// lane per step): 0 (32,4,4), 1 (32,2,8), 2 (8,2,4), 3 (4,1,8), 4 (16,4,2),
// and 9 (32,1,8), whose 32 lanes all take entries of one frame (the
// one-frame launches of the plain path); frame-lane mappings (k_gather_fl),
// 2 CTAs per SM (5) or 1 CTA per SM with the next frames prefetched while the
// current ones are summed (6); bin tiles (k_gather_bins: 7, one frame per
// lane; 8, two), which write the results themselves; row warps (k_rows, 10)
// for launches of a few frames, which write them too.
constexpr int kVariantCount = 11;
constexpr int kSegMax = 256;
constexpr int kUnitCap = 3008;  // 16-byte entries in the 48 KB default shared memory

// kRaw: the per-frame-mask gather (entries {pixel, w, w*norm}); it sums
// S = sum w*s, V = sum w^2*max(s,0), N = sum w*norm and C = sum w over the
// entries whose pixel the frame's mask leaves unmasked.
enum Mode { kIntensity = 0, kErrors = 1, kSpread = 2, kRaw = 3 };

template <typename P>
constexpr bool is_float_px() {
    return std::is_same<P, float>::value || std::is_same<P, double>::value;
}

// Accumulators per (segment, frame): S = sum c*s, then V = sum c^2*max(s,0),
// then for the spread B = sum (c/n)*t^2 and A = sum c*t, then for float
// pixels the weight c*n and the count of non-finite pixels.
template <int MODE, typename P>
struct NAcc {
    static constexpr int value = MODE == kIntensity ? 1
                                 : MODE == kErrors  ? 2
                                 : MODE == kRaw     ? 4
                                                    : (is_float_px<P>() ? 6 : 4);
};
constexpr int kSpreadA = 3;  // index of A among the spread's accumulators
constexpr int kMaxAcc = 6;   // accumulators per (segment, frame), at most
static_assert(NAcc<kSpread, float>::value <= kMaxAcc && NAcc<kRaw, float>::value <= kMaxAcc,
              "partial sums are sized for kMaxAcc accumulators");

// Accumulators per frame of a mode, for sizing partial sums at run time.
inline int n_accumulators(int mode, bool float_px) {
    return mode == kIntensity ? 1 : mode == kErrors ? 2 : mode == kRaw ? 4 : (float_px ? 6 : 4);
}

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

// Origin o = s/n of the spread's shift in this frame. The reference shifts
// by the row's first valid entry (azimuthal.rs:80-82); the spread does not
// depend on the shift, only its rounding does: the moments lose to
// cancellation about (mean - o)^2 / variance, so this build shifts by the
// row's heaviest valid entry (largest c*n, chosen at plan time), which sits
// at the mean of a bin dominated by one pixel. A float pixel that is not
// finite there hands the origin to the row's first valid finite entry
// (entries that are statically invalid carry c = 0).
template <typename P>
__device__ __forceinline__ float row_origin(const float4 *__restrict__ entry_std, int origin,
                                            int first, int row_end,
                                            const P *__restrict__ frame) {
    if (origin < 0) return 0.f;
    float4 e = entry_std[origin];
    float s = load_px<P>(frame, uint32_t(__float_as_int(e.x)));
    if (is_float_px<P>() && !isfinite(s)) {
        for (int k = first; k < row_end; ++k) {
            const float4 ek = entry_std[k];
            if (!(ek.y > 0.f)) continue;
            e = ek;
            s = load_px<P>(frame, uint32_t(__float_as_int(e.x)));
            if (isfinite(s)) break;
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
// One unit of the entry-lane gather, run by the whole CTA (k_gather runs unit
// blockIdx.x; the work-queue gather runs the units it claims, several per
// CTA). It ends with a CTA barrier, so the next unit may restage the shared
// memory at once.
template <int MODE, typename P, int SLICES, int FPL, int U>
__device__ __forceinline__ void gather_unit(
    int unit, const int2 *__restrict__ units, const int4 *__restrict__ segs,
    const int2 *__restrict__ entry, const float4 *__restrict__ entry_std,
    const float *__restrict__ entry_nlo, const int32_t *__restrict__ first_valid,
    const int32_t *__restrict__ origin_entry, const P *__restrict__ frames, int64_t n_pixels,
    int n_frames, int n_segments, double *__restrict__ partial,
    const uint8_t *__restrict__ masks, int64_t mask_stride) {
    constexpr int NA = NAcc<MODE, P>::value;
    constexpr bool WIDE = MODE == kSpread || MODE == kRaw;  // 16-byte entries
    constexpr int GROUPS = 32 / SLICES;         // frame lane groups per warp
    constexpr int TASK_FRAMES = GROUPS * FPL;  // frames per task
    static_assert(kFlush % U == 0, "flush cadence must be a multiple of the unroll");
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_off[kWarps + 1];
    const int2 un = units[unit];
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
        if (WIDE) {
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
        const uint8_t *mk[FPL];
        bool fv[FPL];
#pragma unroll
        for (int q = 0; q < FPL; ++q) {
            fv[q] = fbase + q < n_frames;
            fr[q] = frames + int64_t(fv[q] ? fbase + q : 0) * n_pixels;
            mk[q] = MODE == kRaw ? masks + int64_t(fv[q] ? fbase + q : 0) * mask_stride : nullptr;
        }
        float origin[FPL];
#pragma unroll
        for (int q = 0; q < FPL; ++q)
            origin[q] = MODE == kSpread ? row_origin<P>(entry_std, origin_entry[row],
                                                        first_valid[row], sg.w, fr[q])
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
            if (MODE == kRaw) {
                float4 e[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int j = j0 + SLICES * u;
                    if (CHECK)
                        e[u] = j < len ? reinterpret_cast<const float4 *>(smem)[off + j]
                                       : make_float4(0.f, 0.f, 0.f, 0.f);
                    else
                        e[u] = reinterpret_cast<const float4 *>(smem)[off + j];
                }
                float sv[U][FPL];
                bool live[U][FPL];
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                    for (int q = 0; q < FPL; ++q) {
                        const uint32_t col = uint32_t(__float_as_int(e[u].x));
                        const bool in = !CHECK || j0 + SLICES * u < len;
                        sv[u][q] = in ? load_px<P>(fr[q], col) : 0.f;
                        live[u][q] = in && __ldg(mk[q] + col) == 0;
                    }
#pragma unroll
                for (int u = 0; u < U; ++u) {
#pragma unroll
                    for (int q = 0; q < FPL; ++q) {
                        // a masked pixel adds nothing, whatever its value
                        const float c = live[u][q] ? e[u].y : 0.f;
                        const float cn = live[u][q] ? e[u].z : 0.f;
                        const float v = live[u][q] ? sv[u][q] : 0.f;
                        acc[q][0].fma(c, v);
                        acc[q][1].fma(__fmul_rn(c, c), is_unsigned_px<P>() ? v : fmaxf(v, 0.f));
                        acc[q][2].add(cn);
                        acc[q][3].add(c);
                    }
                }
            } else if (MODE == kSpread) {
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
                float sv[U][FPL], nlo[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const bool in = !CHECK || j0 + SLICES * u < len;
                    nlo[u] = in ? __ldg(entry_nlo + sg.y + j0 + SLICES * u) : 0.f;
#pragma unroll
                    for (int q = 0; q < FPL; ++q)
                        sv[u][q] = in ? load_px<P>(fr[q], uint32_t(__float_as_int(e[u].x))) : 0.f;
                }
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
                        const float t = __fmaf_rn(-origin[q], nlo[u], __fmaf_rn(-origin[q], n, v));
                        acc[q][2].fma(__fmul_rn(cr, t), t);
                        acc[q][kSpreadA].fma(c, t);
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
                    partial[(int64_t(seg0 + si) * NA + a) * n_frames + fbase + q] = mine;
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
#pragma unroll
                    for (int a = 0; a < NA; ++a)
                        partial[(int64_t(seg0 + si) * NA + a) * n_frames + fbase + q] = d[q][a];
                }
            }
        }
    }
    __syncthreads();
}

template <int MODE, typename P, int SLICES, int FPL, int U>
__global__ void __launch_bounds__(kThreads)
    k_gather(const int2 *__restrict__ units, const int4 *__restrict__ segs,
             const int2 *__restrict__ entry, const float4 *__restrict__ entry_std,
             const float *__restrict__ entry_nlo,
             const int32_t *__restrict__ first_valid, const int32_t *__restrict__ origin_entry,
             const P *__restrict__ frames, int64_t n_pixels, int n_frames, int n_segments,
             double *__restrict__ partial, const uint8_t *__restrict__ masks,
             int64_t mask_stride) {
    gather_unit<MODE, P, SLICES, FPL, U>(blockIdx.x, units, segs, entry, entry_std, entry_nlo,
                                         first_valid, origin_entry, frames, n_pixels, n_frames,
                                         n_segments, partial, masks, mask_stride);
}

// ---------------------------------------------------------------------------
// Row warps (lane mapping 10): launches of a few frames. A batch amortises
// the table over its frames; one frame reads every entry once, so what
// counts there is keeping enough loads in flight and doing nothing else: no
// staging, no partial sums, no second launch. A row of at most kRowsLong
// entries is one warp's (eight rows per CTA), a longer one the whole CTA's
// (largest first, so the long rows start early). Threads stride the row's
// entries (coalesced), kRowsU of them in flight each, load the pixels of F
// frames per entry and sum in FP64; the warp (then the CTA's warps in a fixed
// order) adds the threads' sums by a fixed butterfly and one thread writes the
// results (normalize_bin, prepared.rs:985-996; the spread's closing formulas,
// azimuthal.rs:96-104). The spread is shifted by the row's origin as in the
// other mappings, in FP64: t = s - o*n with n the entry's FP32 pair.
constexpr int kRowsLong = 512;
constexpr int kRowsTiny = 64;  // rows of at most this many entries take 8 lanes
#ifndef DG_ROWS_U
#define DG_ROWS_U 4
#endif
constexpr int kRowsU = DG_ROWS_U;
constexpr int kRowsThreads = 256;

template <typename P>
__device__ __forceinline__ double load_px_d(const P *__restrict__ f, uint32_t i) {
    return double(__ldg(f + i));
}

// Butterfly sum over the 32 lanes: every lane ends with the same value (IEEE
// addition is commutative, so partners compute the same sums).
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) v = __dadd_rn(v, __shfl_xor_sync(0xffffffffu, v, m));
    return v;
}
// The same over each group of 8 lanes (the warp's four tiny rows).
__device__ __forceinline__ double group8_sum_d(double v) {
#pragma unroll
    for (int m = 4; m > 0; m >>= 1) v = __dadd_rn(v, __shfl_xor_sync(0xffffffffu, v, m));
    return v;
}

// Shared memory of a row-warp CTA: the warps' sums of a long row.
constexpr int kRowsWarps = kRowsThreads / 32;
using RowsRed = double[kRowsWarps][4 * kMaxAcc];

// One row-warp item of a plan's batch (q.item[k]); every thread of the CTA
// calls it. F frames per pass over the entries.
template <int MODE, typename P, int F>
__device__ __forceinline__ void rows_item(const QueuePlan &qp, int k, int fb, RowsRed &s_red) {
    constexpr int NA = NAcc<MODE, P>::value;
    constexpr bool SPREAD = MODE == kSpread;
    constexpr int NW = kRowsWarps;
    const int4 *__restrict__ items = qp.item;
    const int32_t *__restrict__ rows = qp.rows;
    const int32_t *__restrict__ row_ptr = qp.row_ptr;
    const int2 *__restrict__ entry = qp.entry;
    const float4 *__restrict__ entry_std = qp.entry_std;
    const float2 *__restrict__ px_norm = qp.px_norm;
    const int32_t *__restrict__ first_valid = qp.first_valid;
    const int32_t *__restrict__ origin_entry = qp.origin;
    const double *__restrict__ den = qp.den;
    const double *__restrict__ den_std = qp.den_std;
    const int32_t *__restrict__ valid_std = qp.valid_std;
    const P *__restrict__ frames = static_cast<const P *>(qp.frames);
    const int64_t n_pixels = qp.n_pixels;
    const int n_frames = qp.n_frames, n_rows = qp.n_rows;
    double *__restrict__ out_i = qp.out_i;
    double *__restrict__ out_s = qp.out_s;
    double *__restrict__ out_d = qp.out_d;
    const int4 it = items[k];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // {row, 0, begin, end}: one long row for the whole CTA, its entry range
    // inline; {first, n > 0}: a row per warp; {first, -n}: tiny rows, 8 lanes
    // each (four per warp), rows[first ..] and their row pointers.
    const bool whole = it.y == 0, tiny = it.y < 0;
    if (!whole && !tiny && warp >= it.y) return;  // no CTA-wide barrier in this case
    const int sub = int(threadIdx.x) >> 3;
    if (tiny && (sub & ~3) >= -it.y) return;  // a warp whose four rows are all past the end
    const bool live = !tiny || sub < -it.y;    // lanes past the end still shuffle
    const int row = whole ? it.x : rows[it.x + (tiny ? (live ? sub : 0) : warp)];
    const int e0 = whole ? it.z : row_ptr[row];
    const int e1 = whole ? it.w : live ? row_ptr[row + 1] : e0;
    const int li = whole ? int(threadIdx.x) : tiny ? (lane & 7) : lane;
    const int nl = whole ? kRowsThreads : tiny ? 8 : 32;
    const int org = SPREAD ? origin_entry[row] : -1, fvalid = SPREAD ? first_valid[row] : -1;
    // frames [F*fb, F*fb + F) of the batch, one pass
    for (int f0 = F * fb; f0 < n_frames && f0 < F * fb + F; f0 += F) {
        const P *fr[F];
#pragma unroll
        for (int q = 0; q < F; ++q) fr[q] = frames + int64_t(min(f0 + q, n_frames - 1)) * n_pixels;
        double o[F];
#pragma unroll
        for (int q = 0; q < F; ++q)
            o[q] = SPREAD ? double(row_origin<P>(entry_std, org, fvalid, e1, fr[q])) : 0.0;
        double acc[F][NA];
#pragma unroll
        for (int q = 0; q < F; ++q)
#pragma unroll
            for (int a = 0; a < NA; ++a) acc[q][a] = 0.0;
        for (int j0 = e0 + li; j0 < e1; j0 += nl * kRowsU) {
            float2 nn[kRowsU];
            int2 en[kRowsU];
            double x[kRowsU][F];
#pragma unroll
            for (int u = 0; u < kRowsU; ++u) {
                const int j = j0 + nl * u;
                const bool in = j < e1;
                en[u] = in ? entry[j] : make_int2(0, 0);
                const uint32_t col = uint32_t(en[u].x);
                if constexpr (SPREAD) nn[u] = in ? px_norm[col] : make_float2(0.f, 0.f);
#pragma unroll
                for (int q = 0; q < F; ++q) x[u][q] = in ? load_px_d<P>(fr[q], col) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kRowsU; ++u) {
                if (j0 + nl * u >= e1) break;
                if constexpr (SPREAD) {
                    // valid for the spread (azimuthal.rs:62-75): c > 0 and n
                    // finite and > 0 ({0, 0} marks an invalid n); an invalid
                    // entry adds nothing
                    const float cf = __int_as_float(en[u].y);
                    const bool ok = nn[u].x > 0.f && cf > 0.f && cf <= 3.40282347e+38f;
                    const double c = ok ? double(cf) : 0.0;
                    const double cr = ok ? double(__fdiv_rn(cf, nn[u].x)) : 0.0;
                    const double n = ok ? __dadd_rn(double(nn[u].x), double(nn[u].y)) : 1.0;
                    const double c2 = __dmul_rn(c, c);
#pragma unroll
                    for (int q = 0; q < F; ++q) {
                        const double v = x[u][q];
                        if (is_float_px<P>() && !isfinite(v)) {
                            acc[q][NA - 2] = __dadd_rn(acc[q][NA - 2], __dmul_rn(c, n));
                            acc[q][NA - 1] = __dadd_rn(acc[q][NA - 1], c > 0.0 ? 1.0 : 0.0);
                            continue;
                        }
                        acc[q][0] = __fma_rn(c, v, acc[q][0]);
                        acc[q][1] = __fma_rn(c2, is_unsigned_px<P>() ? v : fmax(v, 0.0), acc[q][1]);
                        const double t = __fma_rn(-o[q], n, v);
                        acc[q][2] = __fma_rn(__dmul_rn(cr, t), t, acc[q][2]);
                        acc[q][kSpreadA] = __fma_rn(c, t, acc[q][kSpreadA]);
                    }
                } else {
                    const double c = __int_as_float(en[u].y);
                    const double c2 = __dmul_rn(c, c);
#pragma unroll
                    for (int q = 0; q < F; ++q) {
                        acc[q][0] = __fma_rn(c, x[u][q], acc[q][0]);
                        if (MODE == kErrors)
                            acc[q][1] = __fma_rn(c2, is_unsigned_px<P>() ? x[u][q] : fmax(x[u][q], 0.0),
                                                 acc[q][1]);
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < F; ++q)
#pragma unroll
            for (int a = 0; a < NA; ++a)
                acc[q][a] = tiny ? group8_sum_d(acc[q][a]) : warp_sum_d(acc[q][a]);
        if (whole) {
            if (lane == 0)
#pragma unroll
                for (int q = 0; q < F; ++q)
#pragma unroll
                    for (int a = 0; a < NA; ++a) s_red[warp][q * NA + a] = acc[q][a];
            __syncthreads();
            if (threadIdx.x == 0)
#pragma unroll
                for (int q = 0; q < F; ++q)
#pragma unroll
                    for (int a = 0; a < NA; ++a) {
                        double v = s_red[0][q * NA + a];
                        for (int w = 1; w < NW; ++w) v = __dadd_rn(v, s_red[w][q * NA + a]);
                        acc[q][a] = v;
                    }
            __syncthreads();  // s_red is rewritten by the next frames
            if (threadIdx.x != 0) continue;
        } else if (tiny ? ((lane & 7) != 0 || !live) : lane != 0) {
            continue;
        }
#pragma unroll
        for (int q = 0; q < F; ++q) {
            if (f0 + q >= n_frames) break;
            const double *v = acc[q];
            const int64_t oo = int64_t(f0 + q) * n_rows + row;
            if constexpr (!SPREAD) {
                const double n = den[row];
                out_i[oo] = n == 0.0 ? 0.0 : v[0] / n;
                if (MODE == kErrors) {
                    const double s2 = n == 0.0 ? 0.0 : v[1] / (n * n);
                    out_s[oo] = sqrt(s2 > 0.0 ? s2 : 0.0);
                }
            } else {
                int valid = valid_std[row];
                double sw = den_std[row];
                if (NA == 6) {
                    valid -= int(v[NA - 1] + 0.5);
                    sw -= v[NA - 2];
                }
                if (valid <= 0 || !(sw > 0.0)) {
                    out_i[oo] = 0.0;
                    if (out_s) out_s[oo] = 0.0;
                    out_d[oo] = __longlong_as_double(0x7ff8000000000000ll);
                    continue;
                }
                const double a1 = v[kSpreadA];
                out_i[oo] = v[0] / sw;
                if (out_s) out_s[oo] = sqrt(v[1] > 0.0 ? v[1] : 0.0) / sw;
                const double mean = a1 / sw;
                const double q2 = (v[2] - mean * a1) / sw;
                // one valid contribution: its deviation from itself is exactly 0
                out_d[oo] = valid == 1 ? 0.0 : sqrt(q2 > 0.0 ? q2 : 0.0);
            }
        }
    }
}

// Lane mapping 10 for one plan's batch: one CTA per (item, frame block).
// Resident CTAs per SM the compiler must allow for (0: as many as the
// registers it chooses leave; the spread's one-frame form takes 64, four CTAs).
#ifndef DG_ROWS_MINB
#define DG_ROWS_MINB 0
#endif
#if DG_ROWS_MINB > 0
#define DG_ROWS_BOUNDS __launch_bounds__(kRowsThreads, DG_ROWS_MINB)
#else
#define DG_ROWS_BOUNDS __launch_bounds__(kRowsThreads)
#endif
template <int MODE, typename P, int F>
__global__ void DG_ROWS_BOUNDS k_rows(const QueuePlan q) {
    __shared__ RowsRed s_red;
    rows_item<MODE, P, F>(q, blockIdx.x, blockIdx.y, s_red);
}

// Frames per pass (and per frame block) of a row-warp launch of nf frames.
__host__ __device__ constexpr int rows_pass_frames(int nf) { return nf <= 1 ? 1 : nf <= 2 ? 2 : 4; }

// Tiles a resident work-queue CTA claims at once (one atomic add per claim),
// and the most tiles a call runs as one CTA per tile.
constexpr int kQueueClaim = 4;
constexpr int64_t kQueueDirectTiles = int64_t(1) << 24;

// Work-queue gather over several plans (dg_multi_integrate). A persistent
// grid of row-warp CTAs claims (plan, row item, frame block) tiles from one
// counter until every plan's tiles are summed, so plans of very different
// sizes and batch sizes share one launch and the GPU stays full to the last
// tile. A plan's results are those
// of lane mapping 10 launched for that plan alone, bit for bit. No CTA waits
// on another: a claim is one atomic add, and a CTA that finds the counter
// past the end returns.
template <int MODE, typename P>
__global__ void __launch_bounds__(kRowsThreads)
    k_rows_queue(QueueHeader *__restrict__ hdr, const QueuePlan *__restrict__ plans) {
    __shared__ RowsRed s_red;
    __shared__ int s_item;
    const int n_plans = hdr->n_plans, total = hdr->total_items;
    // A grid that covers every tile takes tile blockIdx.x; a smaller one (a
    // batch beyond the grid limit) stays resident and claims tiles.
    const bool direct = int64_t(gridDim.x) >= int64_t(total);
    for (int pass = 0;; ++pass) {
        int first;
        if (direct) {
            first = int(blockIdx.x);
            if (pass > 0 || first >= total) return;
        } else {
            if (threadIdx.x == 0) s_item = atomicAdd(&hdr->counter, kQueueClaim);
            __syncthreads();
            first = s_item;
            __syncthreads();  // every thread has read s_item before it is claimed again
            if (first >= total) return;
        }
        // the last descriptor whose first tile is at most `first` (plans with
        // no tiles share the next one's prefix and are skipped)
        int lo = 0, hi = n_plans - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (plans[mid].item_first <= first) lo = mid;
            else hi = mid - 1;
        }
        const int last = direct ? first + 1 : min(first + kQueueClaim, total);
        for (int item = first; item < last; ++item) {
            while (lo + 1 < n_plans && plans[lo + 1].item_first <= item) ++lo;
            const QueuePlan &q = plans[lo];
            // (row item, frame block) tiles of the plan, the frame blocks of
            // an item one after another (its entries are still in L2 for the
            // next)
            const int local = item - q.item_first;
            const int k = local / q.frame_blocks, fb = local - k * q.frame_blocks;
            switch (rows_pass_frames(q.n_frames)) {
            case 1: rows_item<MODE, P, 1>(q, k, fb, s_red); break;
            case 2: rows_item<MODE, P, 2>(q, k, fb, s_red); break;
            default: rows_item<MODE, P, 4>(q, k, fb, s_red); break;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Frame-lane gather. Lane = frame: for 32 frames at a time, a unit's distinct
// pixels (at most kFlDCap, listed at plan time) are staged in shared memory,
// 4-byte pixel types by cp.async and the others converted to FP32 on the way,
// frame rows kFlStride words apart (odd, so the 32 lanes reading one pixel of
// their own frames hit 32 banks). Every lane of a warp walks the same entries
// against its own frame, so a frame's sums need no cross-lane reduction.
//
// Entries go in pairs, {index 0, index 1, c0, c1} and for the spread
// {n0, n1, c0/n0, c1/n1}, their columns rewritten at plan time as indices
// into the unit's pixel list; a segment of odd length ends with a padding
// entry of weight 0 whose index names column kFlDCap, which staging never
// writes and which holds 0. Sums use packed FP32x2 arithmetic: the even
// entries of a segment accumulate in one half, the odd ones in the other,
// each in a double-word accumulator folded every kFlFlushPairs pairs.
//
// A unit's pairs are cut into kWarps equal pieces, one per warp. A segment
// inside one piece is written straight to the partial sums; a piece's first
// and last segments go to shared-memory slots, and the slots of a segment
// cut by piece boundaries are added in warp order. Results depend on the
// table alone, not on the frames around them in a batch.

#ifndef DG_FL_DCAP
#define DG_FL_DCAP 384
#endif
constexpr int kFlSegs = 32;               // segments per frame-lane unit, at most
constexpr int kFlDCap = DG_FL_DCAP;       // distinct pixels per frame-lane unit (even)
constexpr int kFlECap = 2 * kFlDCap;      // entries per frame-lane unit before padding
constexpr int kFlPairCap = (kFlECap + kFlSegs) / 2;
constexpr int kFlStride = kFlDCap + 1;    // odd; column kFlDCap stays 0
constexpr int kFlSlots = 2 * kWarps;      // first and last segment of each piece
constexpr int kFlFlushPairs = 16;         // pairs per lane between double-word folds
constexpr int kFlSortMax = 2048;          // keys one unit sorts at plan time
static_assert(kFlECap + kFlSegs <= kFlSortMax, "frame-lane units must fit the plan-time sort");
static_assert(kFlSegs <= 32, "the unit set-up scans segment lengths in one warp");
static_assert(kSegMax <= kFlDCap, "a single segment must fit a frame-lane unit");

template <typename P>
using StagedPx = typename std::conditional<sizeof(P) == 4, P, float>::type;

__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
// The same with the shared-memory address as a 32-bit integer, and a 32-bit
// shared-memory load: address arithmetic stays in 32 bits.
__device__ __forceinline__ void cp_async4_s(unsigned d, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
// L2 eviction priority of the bin tiles' 4-byte pixel copies: 0 the default
// policy, 1 evict-first (frame sectors stream through L2 and leave it to the
// entry-pair records that a tile's frame groups share), 2 evict-last.
#ifndef DG_BT_L2HINT
#define DG_BT_L2HINT 0
#endif
__device__ __forceinline__ uint64_t bt_l2_policy() {
    uint64_t p = 0;
    if constexpr (DG_BT_L2HINT == 1)
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
    else if constexpr (DG_BT_L2HINT == 2)
        asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
    return p;
}
__device__ __forceinline__ void cp_async4_sp(unsigned d, const void *src, uint64_t policy) {
    if constexpr (DG_BT_L2HINT == 0) {
        cp_async4_s(d, src);
    } else {
        asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 4, %2;\n" ::"r"(d),
                     "l"(src), "l"(policy)
                     : "memory");
    }
}
__device__ __forceinline__ uint32_t lds32(unsigned a) {
    uint32_t v;
    asm volatile("ld.shared.b32 %0, [%1];\n" : "=r"(v) : "r"(a));
    return v;
}
// A staged 4-byte pixel from its bits.
template <typename S>
__device__ __forceinline__ float staged_value(uint32_t b) {
    if constexpr (std::is_same<S, float>::value) return __uint_as_float(b);
    else if constexpr (std::is_same<S, int32_t>::value) return float(int32_t(b));
    else return float(b);
}

// Packed FP32x2 arithmetic (round to nearest, per element as the scalar
// operations).
typedef unsigned long long f2;
__device__ __forceinline__ f2 pk(float a, float b) {
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float2 upk(f2 v) {
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
    return r;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
    f2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
    f2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
    f2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
    f2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// Two double-word FP32 accumulators (even and odd entries) with a plain
// FP32 block in front; the fold is AccDW::flush on each half.
struct Acc2 {
    f2 p, hi, lo;
    __device__ __forceinline__ void zero() { p = hi = lo = 0ull; }
    __device__ __forceinline__ void flush() {
        const f2 s = add2(hi, p);
        const f2 bp = sub2(s, hi);
        const f2 e = add2(sub2(hi, sub2(s, bp)), sub2(p, bp));
        hi = s;
        lo = add2(lo, e);
        p = 0ull;
    }
    // Both halves' exact sums added in FP64 (even + odd).
    __device__ __forceinline__ double value() const {
        const float2 h = upk(hi), l = upk(lo);
        return __dadd_rn(double(h.x) + double(l.x), double(h.y) + double(l.y));
    }
};

// The same packed partial folded into one FP64 sum instead (both halves
// added in FP64, even then odd): four registers instead of six.
struct AccP64 {
    f2 p;
    double d;
    __device__ __forceinline__ void zero() {
        p = 0ull;
        d = 0.0;
    }
    __device__ __forceinline__ void flush() {
        const float2 h = upk(p);
        d = __dadd_rn(__dadd_rn(d, double(h.x)), double(h.y));
        p = 0ull;
    }
    __device__ __forceinline__ double value() const { return d; }
};


// Dynamic shared memory of k_gather_fl: entry pairs, pixel list, one or
// (double-buffered) two sets of 32 frame rows, piece-boundary slots.
template <int MODE>
constexpr size_t fl_pair_bytes() {
    return MODE == kSpread ? 40 : 16;  // pair A, and B and C for the spread
}
template <int MODE, typename P, bool DB>
constexpr size_t fl_smem_bytes() {
    return size_t(kFlPairCap) * fl_pair_bytes<MODE>() + size_t(kFlDCap) * 4 +
           size_t(DB ? 64 : 32) * kFlStride * 4 + size_t(kFlSlots) * NAcc<MODE, P>::value * 32 * 8;
}

// CTAs per SM the frame-lane gather's shared memory allows (227 KB per CTA,
// 228 KB per SM with 1 KB reserved per CTA), for its launch bounds.
template <int MODE, typename P, bool DB>
constexpr int fl_ctas_per_sm() {
    return fl_smem_bytes<MODE, P, DB>() + 6 * 1024 <= 113 * 1024 ? 2 : 1;
}

template <int MODE, typename P, int U2, bool DB>
__global__ void __launch_bounds__(kThreads, (fl_ctas_per_sm<MODE, P, DB>()))
    k_gather_fl(const int4 *__restrict__ units, const int4 *__restrict__ segs,
                const int32_t *__restrict__ unit_px, const float4 *__restrict__ pair_a,
                const float4 *__restrict__ pair_b, const float2 *__restrict__ pair_c,
                const float4 *__restrict__ entry_std,
                const int32_t *__restrict__ first_valid, const int32_t *__restrict__ origin_entry,
                const int32_t *__restrict__ seg_org,
                const P *__restrict__ frames, int64_t n_pixels, int n_frames, int n_segments,
                double *__restrict__ partial) {
    using S = StagedPx<P>;
    constexpr int NA = NAcc<MODE, P>::value;
    constexpr bool SPREAD = MODE == kSpread;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_off[kFlSegs + 1], s_first[kFlSegs], s_rend[kFlSegs], s_oidx[kFlSegs],
        s_oent[kFlSegs];
    __shared__ float s_on[kFlSegs];
    __shared__ int s_sa[kWarps], s_sb[kWarps];
    __shared__ int s_nb, s_bseg[kFlSlots], s_bwlo[kFlSlots], s_bwhi[kFlSlots];
    float4 *s_pa = reinterpret_cast<float4 *>(smem);
    float4 *s_pb = s_pa + kFlPairCap;
    float2 *s_pc = reinterpret_cast<float2 *>(s_pb + kFlPairCap);
    int32_t *s_px = reinterpret_cast<int32_t *>(smem + size_t(kFlPairCap) * fl_pair_bytes<MODE>());
    S *s_buf = reinterpret_cast<S *>(s_px + kFlDCap);
    double *s_red = reinterpret_cast<double *>(s_buf + (DB ? 64 : 32) * kFlStride);

    const int4 un = units[blockIdx.x];
    const int seg0 = un.x, nseg = un.y, D = un.w;
    const int64_t poff = un.z;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (warp == 0) {
        int plen = 0;
        if (lane < nseg) {
            const int4 sg = segs[seg0 + lane];
            plen = (sg.z - sg.y + 1) & ~1;
            const int first = first_valid[sg.x], oe = origin_entry[sg.x];
            s_first[lane] = first;
            s_rend[lane] = sg.w;
            s_oent[lane] = oe;
            if (SPREAD) {
                s_oidx[lane] = seg_org[seg0 + lane];
                s_on[lane] = oe >= 0 ? entry_std[oe].z : 1.f;
            }
        }
        int inc = plen;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane < nseg) s_off[lane + 1] = inc;
        if (lane == 0) s_off[0] = 0;
    }
    __syncthreads();
    const int np = s_off[nseg] >> 1;
    for (int j = tid; j < np; j += kThreads) {
        s_pa[j] = pair_a[poff + j];
        if (SPREAD) {
            s_pb[j] = pair_b[poff + j];
            s_pc[j] = pair_c[poff + j];
        }
    }
    for (int j = tid; j < D; j += kThreads) s_px[j] = unit_px[int64_t(blockIdx.x) * kFlDCap + j];
    // Column kFlDCap of every frame row is read by padding entries and must
    // hold 0; staging writes columns below D <= kFlDCap only.
    for (int j = tid; j < (DB ? 64 : 32); j += kThreads) s_buf[j * kFlStride + kFlDCap] = S(0);
    // This warp's piece [lo, hi) (entries; pair aligned) and the segments
    // sa..sb it meets.
    const int lo = 2 * int(int64_t(warp) * np / kWarps);
    const int hi = 2 * int(int64_t(warp + 1) * np / kWarps);
    int sa = 0, sb = -1;
    if (lo < hi) {
        while (s_off[sa + 1] <= lo) ++sa;
        sb = sa;
        while (s_off[sb + 1] < hi) ++sb;
    }
    if (lane == 0) {
        s_sa[warp] = sa;
        s_sb[warp] = sb;
    }
    __syncthreads();
    if (tid == 0) {
        // Segments at piece boundaries, ascending, with their warps.
        int nb = 0;
        for (int w = 0; w < kWarps; ++w) {
            if (s_sb[w] < 0) continue;
            for (int e = 0; e < 2; ++e) {
                const int b = e == 0 ? s_sa[w] : s_sb[w];
                if (e == 1 && b == s_sa[w]) break;
                if (nb > 0 && s_bseg[nb - 1] == b) {
                    s_bwhi[nb - 1] = w;
                } else {
                    s_bseg[nb] = b;
                    s_bwlo[nb] = w;
                    s_bwhi[nb] = w;
                    ++nb;
                }
            }
        }
        s_nb = nb;
    }
    __syncthreads();

    // Stage pixel s_px[k] of frames f0.. into frame rows of `buf`; rows of
    // frames past the end keep stale values (their lanes are never written
    // out). 4-byte pixels are copied asynchronously as one commit group.
    auto stage = [&](int f0, S *buf) {
        const int nv = min(32, n_frames - f0);
        for (int k = tid; k < D; k += kThreads) {
            const P *src = frames + int64_t(f0) * n_pixels + s_px[k];
            S *dst = buf + k;
            if constexpr (sizeof(P) == 4) {
#pragma unroll 8
                for (int f = 0; f < nv; ++f) cp_async4(dst + f * kFlStride, src + int64_t(f) * n_pixels);
            } else {
#pragma unroll 8
                for (int f = 0; f < nv; ++f)
                    dst[f * kFlStride] = load_px<P>(src + int64_t(f) * n_pixels, 0u);
            }
        }
        if constexpr (sizeof(P) == 4) asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    const int groups = (n_frames + 31) / 32;
    if (DB) stage(0, s_buf);
    for (int g = 0; g < groups; ++g) {
        const int f0 = g * 32;
        const int nv = min(32, n_frames - f0);
        S *cur = DB && (g & 1) ? s_buf + 32 * kFlStride : s_buf;
        if (!DB) {
            stage(f0, cur);
            if constexpr (sizeof(P) == 4) asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        } else if (g + 1 < groups) {
            // Prefetch the next group into the other buffer, last read by the
            // previous group's compute (finished at its closing barrier).
            stage(f0 + 32, (g & 1) ? s_buf : s_buf + 32 * kFlStride);
            if constexpr (sizeof(P) == 4) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        } else {
            if constexpr (sizeof(P) == 4) asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();
        const S *px = cur + lane * kFlStride;

        for (int i = sa; i <= sb; ++i) {
            const int p0 = max(lo, s_off[i]) >> 1, p1 = min(hi, s_off[i + 1]) >> 1;
            // Origin o = s/n of the row's origin entry (row_origin): its pixel
            // is staged with the unit's; a non-finite float pixel there sends
            // the lane to the row's entries in global memory.
            float org = 0.f;
            if constexpr (SPREAD) {
                const float so = float(px[s_oidx[i]]);
                org = __fdiv_rn(so, s_on[i]);
                if (is_float_px<P>() && !isfinite(so)) {
                    const int fi = min(f0 + lane, n_frames - 1);
                    org = row_origin<P>(entry_std, s_oent[i], s_first[i], s_rend[i],
                                        frames + int64_t(fi) * n_pixels);
                }
            }
            const f2 norg = pk(-org, -org);
            Acc2 acc[NA];
#pragma unroll
            for (int a = 0; a < NA; ++a) acc[a].zero();

            // UU pairs from p, all shared-memory reads issued before use.
            auto body = [&](int p, auto unroll) {
                constexpr int UU = decltype(unroll)::value;
                float4 ea[UU], eb[UU];
                f2 ec[UU];
#pragma unroll
                for (int u = 0; u < UU; ++u) {
                    ea[u] = s_pa[p + u];
                    if constexpr (SPREAD) {
                        eb[u] = s_pb[p + u];
                        ec[u] = reinterpret_cast<const f2 *>(s_pc)[p + u];
                    }
                }
                float v0[UU], v1[UU];
#pragma unroll
                for (int u = 0; u < UU; ++u) {
                    v0[u] = float(px[__float_as_int(ea[u].x)]);
                    v1[u] = float(px[__float_as_int(ea[u].y)]);
                }
#pragma unroll
                for (int u = 0; u < UU; ++u) {
                    const f2 c = pk(ea[u].z, ea[u].w);
                    if constexpr (SPREAD && is_float_px<P>()) {
                      if (!(isfinite(v0[u]) && isfinite(v1[u]))) {
                        // A non-finite pixel adds its weight c*n to the
                        // spread's excluded sums instead (azimuthal.rs:68-70).
                        const bool ok0 = isfinite(v0[u]), ok1 = isfinite(v1[u]);
                        const float x0 = ok0 ? v0[u] : 0.f, x1 = ok1 ? v1[u] : 0.f;
                        const f2 ce = pk(ok0 ? ea[u].z : 0.f, ok1 ? ea[u].w : 0.f);
                        const f2 x = pk(x0, x1), n = pk(eb[u].x, eb[u].y);
                        const f2 cre = pk(ok0 ? eb[u].z : 0.f, ok1 ? eb[u].w : 0.f);
                        acc[0].p = fma2(ce, x, acc[0].p);
                        acc[1].p = fma2(mul2(ce, ce), pk(fmaxf(x0, 0.f), fmaxf(x1, 0.f)), acc[1].p);
                        const f2 t = fma2(norg, ec[u], fma2(norg, n, x));
                        acc[2].p = fma2(mul2(cre, t), t, acc[2].p);
                        acc[kSpreadA].p = fma2(ce, t, acc[kSpreadA].p);
                        acc[NA - 2].p = add2(acc[NA - 2].p,
                                             pk(ok0 ? 0.f : __fmul_rn(ea[u].z, eb[u].x),
                                                ok1 ? 0.f : __fmul_rn(ea[u].w, eb[u].y)));
                        acc[NA - 1].p = add2(acc[NA - 1].p, pk(!ok0 && ea[u].z > 0.f ? 1.f : 0.f,
                                                               !ok1 && ea[u].w > 0.f ? 1.f : 0.f));
                        continue;
                      }
                    }
                    const f2 x = pk(v0[u], v1[u]);
                    acc[0].p = fma2(c, x, acc[0].p);
                    if constexpr (MODE != kIntensity) {
                        const f2 xp = is_unsigned_px<P>()
                                          ? x
                                          : pk(fmaxf(v0[u], 0.f), fmaxf(v1[u], 0.f));
                        acc[1].p = fma2(mul2(c, c), xp, acc[1].p);
                    }
                    if constexpr (SPREAD) {
                        const f2 n = pk(eb[u].x, eb[u].y), cr = pk(eb[u].z, eb[u].w);
                        const f2 t = fma2(norg, ec[u], fma2(norg, n, x));
                        acc[2].p = fma2(mul2(cr, t), t, acc[2].p);
                        acc[kSpreadA].p = fma2(c, t, acc[kSpreadA].p);
                    }
                }
            };
            int p = p0, since = 0;
            for (; p + U2 <= p1; p += U2) {
                body(p, std::integral_constant<int, U2>{});
                since += U2;
                if (since == kFlFlushPairs) {
                    since = 0;
#pragma unroll
                    for (int a = 0; a < NA; ++a) acc[a].flush();
                }
            }
            for (; p < p1; ++p) body(p, std::integral_constant<int, 1>{});
            double val[NA];
#pragma unroll
            for (int a = 0; a < NA; ++a) {
                acc[a].flush();
                val[a] = acc[a].value();
            }
            if (i != sa && i != sb) {
                if (lane < nv) {
#pragma unroll
                    for (int a = 0; a < NA; ++a)
                        partial[(int64_t(seg0 + i) * NA + a) * n_frames + f0 + lane] = val[a];
                }
            } else {
                const int slot = 2 * warp + (i == sa ? 0 : 1);
#pragma unroll
                for (int a = 0; a < NA; ++a) s_red[(slot * NA + a) * 32 + lane] = val[a];
            }
        }
        __syncthreads();

        // Segments at piece boundaries: their pieces added in warp order.
        const int items = s_nb * NA * 32;
        for (int idx = tid; idx < items; idx += kThreads) {
            const int f = idx & 31, rest = idx >> 5;
            const int a = rest % NA, bi = rest / NA;
            const int b = s_bseg[bi];
            double v = 0.0;
            for (int w = s_bwlo[bi]; w <= s_bwhi[bi]; ++w) {
                if (s_sb[w] < 0) continue;  // an empty piece (units of < kWarps pairs)
                const int slot = 2 * w + (b == s_sa[w] ? 0 : 1);
                v = __dadd_rn(v, s_red[(slot * NA + a) * 32 + f]);
            }
            if (f < nv) partial[(int64_t(seg0 + b) * NA + a) * n_frames + f0 + f] = v;
        }
    }
}

// Frame-lane units at plan time: one CTA per unit sorts the unit's pixel
// indices and its segments' origin pixels (bitonic, kFlSortMax keys),
// writes each segment's origin index into seg_org (kFlDCap, the zero column,
// for a row without valid entries), counts the distinct ones into out_d
// and, with fill (and D <= kFlDCap), writes the distinct list and the
// unit's entry pairs: A {index 0, index 1, c0, c1} with the table's FP32
// weights, B {n0, n1, c0/n0, c1/n1}, C {n_lo 0, n_lo 1} and, when pair_as is
// given, A with the spread's weights (0 for entries the spread excludes).
// Each segment's origin pixel is its row's origin entry's.
__global__ void __launch_bounds__(256)
    k_fl_units(const int4 *__restrict__ units, const int4 *__restrict__ segs,
               const int32_t *__restrict__ col, const int32_t *__restrict__ origin_entry,
               int fill, int32_t *__restrict__ out_d, int32_t *__restrict__ unit_px,
               const int2 *__restrict__ entry, const float4 *__restrict__ entry_std,
               const float *__restrict__ entry_nlo, float4 *__restrict__ pair_a,
               float4 *__restrict__ pair_b, float2 *__restrict__ pair_c,
               float4 *__restrict__ pair_as, int32_t *__restrict__ seg_org) {
    constexpr int N = kFlSortMax, T = 256, PER = N / T;
    __shared__ int s_key[N];
    __shared__ int s_uniq[kFlDCap];
    __shared__ int s_off[kFlSegs + 1], s_poff[kFlSegs + 1];
    __shared__ int s_warp[T / 32 + 1];
    const int4 un = units[blockIdx.x];
    const int tid = threadIdx.x;
    if (tid == 0) {
        int o = 0, po = 0;
        for (int i = 0; i < un.y; ++i) {
            const int4 sg = segs[un.x + i];
            s_off[i] = o;
            s_poff[i] = po;
            o += sg.z - sg.y;
            po += (sg.z - sg.y + 1) & ~1;
        }
        s_off[un.y] = o;
        s_poff[un.y] = po;
    }
    __syncthreads();
    // Keys: the entries' pixels, then each segment's origin pixel (the
    // pixel of its row's first entry valid for the spread).
    const int E = s_off[un.y];
    for (int i = 0; i < un.y; ++i) {
        const int4 sg = segs[un.x + i];
        for (int j = tid; j < sg.z - sg.y; j += T) s_key[s_off[i] + j] = col[sg.y + j];
    }
    if (tid < un.y) {
        const int fv = origin_entry[segs[un.x + tid].x];
        s_key[E + tid] = fv >= 0 ? col[fv] : INT_MAX;
    }
    for (int j = E + un.y + tid; j < N; j += T) s_key[j] = INT_MAX;
    __syncthreads();
    for (int k = 2; k <= N; k <<= 1) {
        for (int jj = k >> 1; jj > 0; jj >>= 1) {
            for (int i = tid; i < N; i += T) {
                const int ixj = i ^ jj;
                if (ixj > i) {
                    const int a = s_key[i], b = s_key[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        s_key[i] = b;
                        s_key[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    // Distinct keys: flags over PER consecutive keys per thread, block scan.
    int cnt = 0;
    for (int t = 0; t < PER; ++t) {
        const int i = tid * PER + t;
        const int key = s_key[i];
        cnt += key != INT_MAX && (i == 0 || key != s_key[i - 1]);
    }
    const int lane = tid & 31, w = tid >> 5;
    int inc = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[w] = inc;
    __syncthreads();
    if (tid == 0) {
        int run = 0;
        for (int i = 0; i < T / 32; ++i) {
            const int x = s_warp[i];
            s_warp[i] = run;
            run += x;
        }
        s_warp[T / 32] = run;
    }
    __syncthreads();
    const int D = s_warp[T / 32];
    if (tid == 0) out_d[blockIdx.x] = D;
    if (!fill || D > kFlDCap) return;
    int pos = s_warp[w] + inc - cnt;
    for (int t = 0; t < PER; ++t) {
        const int i = tid * PER + t;
        const int key = s_key[i];
        if (key != INT_MAX && (i == 0 || key != s_key[i - 1])) {
            s_uniq[pos] = key;
            unit_px[int64_t(blockIdx.x) * kFlDCap + pos] = key;
            ++pos;
        }
    }
    __syncthreads();
    if (tid < un.y) {
        const int fv = origin_entry[segs[un.x + tid].x];
        int a = kFlDCap;
        if (fv >= 0) {
            const int cc = col[fv];
            int b = D;
            a = 0;
            while (a < b) {
                const int m = (a + b) >> 1;
                if (s_uniq[m] < cc) a = m + 1;
                else b = m;
            }
        }
        seg_org[un.x + tid] = a;
    }
    float *pa = reinterpret_cast<float *>(pair_a + un.z);
    float *pb = reinterpret_cast<float *>(pair_b + un.z);
    float *pc = reinterpret_cast<float *>(pair_c + un.z);
    float *ps = pair_as ? reinterpret_cast<float *>(pair_as + un.z) : nullptr;
    for (int i = 0; i < un.y; ++i) {
        const int4 sg = segs[un.x + i];
        const int len = sg.z - sg.y, padded = (len + 1) & ~1;
        for (int j = tid; j < padded; j += T) {
            const int p = s_poff[i] + j, rec = (p >> 1) * 4, h = p & 1;
            int idx = kFlDCap;
            float c = 0.f, cs = 0.f, n = 1.f, cr = 0.f, nlo = 0.f;
            if (j < len) {
                const int k = sg.y + j, cc = col[k];
                int a = 0, b = D;
                while (a < b) {
                    const int m = (a + b) >> 1;
                    if (s_uniq[m] < cc) a = m + 1;
                    else b = m;
                }
                idx = a;
                c = __int_as_float(entry[k].y);
                const float4 es = entry_std[k];
                cs = es.y;
                n = es.z;
                cr = es.w;
                nlo = entry_nlo[k];
            }
            pa[rec + h] = __int_as_float(idx);
            pa[rec + 2 + h] = c;
            pb[rec + h] = n;
            pb[rec + 2 + h] = cr;
            pc[(p >> 1) * 2 + h] = nlo;
            if (ps) {
                ps[rec + h] = __int_as_float(idx);
                ps[rec + 2 + h] = cs;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Bin-tile gathers (mappings 7 and 8). A tile is ROWS consecutive rows
// (bins) of the table and 32 * F2 frames (lane = frame; F2 frames per lane,
// 32 apart). The tile's entries, merged over its rows in pixel order, are cut
// into chunks of at most DCap distinct pixels and PCap entry pairs; a row's
// entries inside a chunk are a contiguous run of its CSR row. The CTA walks
// the tile's chunks in order through a ring of buffers: while chunk k is
// summed, the next chunk's pixels (4-byte cp.async into frame rows Stride
// words apart, every warp staging an equal share) and entry pairs (16-byte
// cp.async) are in flight. There is no CTA-wide barrier per chunk: each
// buffer has mbarriers for "landed" (every thread's copies) and "summed"
// (every warp), so a warp whose row has many entries in one chunk can finish
// it while the others start the next one; a row's load evens out over the
// tile (rows of a tile hold nearly equal entry counts; their shares of one
// chunk do not). Every wait is bounded (kBtWaitNs); a warp that gives up
// ends the tile and sets a flag in mapped host memory that the host reports
// as DG_TIMEOUT. Warp w owns row w of the tile and keeps its sums in
// registers for the whole tile (double-word FP32, folded every kBtFoldPairs
// pairs of the row), then normalises and writes the results itself: no
// partial sums, no finalize launch. Every row is summed in the same order for
// every frame and batch.
// With two frames per lane (mapping 8) every entry pair read from shared
// memory serves 64 frames: half the broadcast reads per frame, at half the
// chunk size.
// The same kernel writes raw sums instead (flag `raw`: S and V, with the
// row's strict N and C), and in mode kRaw applies per-frame masks on mapping
// 8's tiles (BtR: two frames per lane, one for 2-byte pixels): a chunk's mask
// bytes are staged
// next to its pixels, and a masked entry adds nothing to S, V, N or C. Bytes
// the kernel loads rather than copies (masks, 2-byte pixels) are loaded with
// a chunk's copies and stored after the warp has summed the chunk before it.

// One bin-tile layout: rows per tile (= warps per CTA: warp w owns row w),
// chunk capacities, frames per lane, pairs per unrolled step and the chunk
// pipeline: BUFS pixel/pair buffers, pixels staged AHEAD chunks before they
// are summed and records MAHEAD chunks before their pixels. Per-chunk
// record, fixed size: {pixels D, pairs, first pair, 0}, the rows' pair
// offsets (ROWS + 1, padded to a multiple of 4 words), then D pixel indices.
template <int ROWS, int DCAP, int PCAP, int F2, int U2, int BUFS = 3, int AHEAD = 1,
          int MAHEAD = 1>
struct BtCfg {
    static constexpr int kRows = ROWS;
    static constexpr int kThreads = ROWS * 32;
    static constexpr int kU2 = U2;
    static constexpr int kBufs = BUFS;
    static constexpr int kAhead = AHEAD;
    static constexpr int kMetaAhead = MAHEAD;
    // A record slot is rewritten only after every warp has summed the chunk
    // it held (the buffer waits guarantee that for BUFS + MAHEAD slots).
    static constexpr int kMetaBufs = BUFS + MAHEAD;
    // How many chunks a warp may fall behind the fastest one.
    static constexpr int kLag = AHEAD < MAHEAD ? (AHEAD < BUFS - AHEAD - 1 ? AHEAD : BUFS - AHEAD - 1)
                                               : (MAHEAD < BUFS - AHEAD - 1 ? MAHEAD : BUFS - AHEAD - 1);
    static_assert(AHEAD >= 1 && MAHEAD >= 1 && kLag >= 0, "pipeline depths");
    static_assert(ROWS <= 32, "tile rows are packed in 5 bits at plan time");
    static constexpr int kDCap = DCAP;          // distinct pixels per chunk
    static constexpr int kStride = DCAP + 1;    // odd frame-row stride; column DCAP stays 0
    static constexpr int kPCap = PCAP;          // entry pairs per chunk
    static constexpr int kF2 = F2;              // frames per lane
    static constexpr int kFrames = 32 * F2;     // frames per CTA
    static constexpr int kMetaHead = (4 + ROWS + 1 + 3) / 4 * 4;
    static constexpr int kMetaWords = kMetaHead + DCAP;
    // Staging shares: the chunk's pixels are cut into kSlices slices and warp
    // w stages slice w % kSlices of kStageFrames frames (w / kSlices + j *
    // ROWS / kSlices), so every warp issues the same number of copies and
    // reads each pixel index once for all its frames.
    static constexpr int kSlices = ROWS % 3 == 0 ? 3 : 1;
    static constexpr int kStageFrames = kFrames * kSlices / ROWS;
    static_assert(ROWS % kSlices == 0 && (kFrames * kSlices) % ROWS == 0,
                  "staging shares must divide evenly");
    static_assert(kMetaWords % 4 == 0, "records are copied in 16-byte pieces");
    static_assert(kStride % 2 == 1, "frame rows must start in different banks");
    // Per-frame masks (mode kRaw): a byte per slot, frame rows an odd number
    // of words apart (32 lanes reading one slot of their frames hit 32 banks).
    static constexpr int kMStride = 4 * (((DCAP + 4) / 4) | 1);
    // Entry pairs: A, then B (spread, masks), then C (spread).
    template <int MODE>
    static constexpr size_t pair_bytes() {
        return MODE == kSpread ? 40 : MODE == kRaw ? 32 : 16;
    }
    template <int MODE>
    static constexpr size_t buf_bytes() {
        return size_t(kFrames) * kStride * 4 + size_t(PCAP) * pair_bytes<MODE>() +
               (MODE == kRaw ? size_t(kFrames) * kMStride : 0);
    }
    // Buffers, records, then the mbarriers: full[BUFS], empty[BUFS], record[kMetaBufs].
    template <int MODE>
    static constexpr size_t bar_offset() {
        return size_t(BUFS) * buf_bytes<MODE>() + size_t(kMetaBufs) * kMetaWords * 4;
    }
    template <int MODE>
    static constexpr size_t smem_bytes() {
        return bar_offset<MODE>() + size_t(2 * BUFS + kMetaBufs) * 8;
    }
};
// Mapping 8's layout can be changed at build time for measurements
// (-DDG_BT8_ROWS=24, -DDG_BT8_DCAP=128 -DDG_BT8_PCAP=200 -DDG_BT8_BUFS=4 -DDG_BT8_AHEAD=2).
#ifndef DG_BT8_ROWS
#define DG_BT8_ROWS 16
#endif
#ifndef DG_BT8_DCAP
#define DG_BT8_DCAP 160
#endif
#ifndef DG_BT8_PCAP
#define DG_BT8_PCAP 256
#endif
#ifndef DG_BT8_BUFS
#define DG_BT8_BUFS 3
#endif
#ifndef DG_BT8_AHEAD
#define DG_BT8_AHEAD 1
#endif
// 2-byte pixels of the bin tiles loaded with a chunk's copies and stored
// after the chunk before it is summed (1), or stored as they arrive (0).
#ifndef DG_BT_DEFER_PX
#define DG_BT_DEFER_PX 1
#endif
// With two frames per lane, the lane's two frames stored side by side in
// shared memory (1: one 8-byte load per slot) or in separate frame rows (0).
#ifndef DG_BT_PAIRED
#define DG_BT_PAIRED 0
#endif
// Shared-memory addresses of the bin tiles' pixel copies and pixel loads
// kept as 32-bit integers (1) or left to the compiler (0).
#ifndef DG_BT_SADDR
#define DG_BT_SADDR 1
#endif
// Bin-tile sums per (row, frame): packed FP32 partials folded into an FP64
// sum (1) or into double-word FP32 sums (0).
#ifndef DG_BT_ACC64
#define DG_BT_ACC64 1
#endif
using BtAcc = std::conditional<DG_BT_ACC64 != 0, AccP64, Acc2>::type;
// Mapping 8's neighbouring tiles launched as 2-CTA clusters (1) or one CTA
// per tile (0).
#ifndef DG_BT_CLUSTER_PAIRS
#define DG_BT_CLUSTER_PAIRS 0
#endif
// Bin tiles run largest first (1) or in bin order (0).
#ifndef DG_BT_LARGEST_FIRST
#define DG_BT_LARGEST_FIRST 1
#endif
// Pairs of a row summed in plain FP32 (each half of a packed accumulator
// takes one entry per pair) before they are folded into the double-word sums.
#ifndef DG_BT_FOLD_PAIRS
#define DG_BT_FOLD_PAIRS 32
#endif
constexpr int kBtFoldPairs = DG_BT_FOLD_PAIRS;
constexpr bool kBtClusterPairs = DG_BT_CLUSTER_PAIRS != 0;
using Bt7 = BtCfg<24, 384, 640, 1, 4>;  // mapping 7
using Bt8 = BtCfg<DG_BT8_ROWS, DG_BT8_DCAP, DG_BT8_PCAP, 2, (DG_BT8_ROWS > 16 ? 2 : 4),
                  DG_BT8_BUFS, DG_BT8_AHEAD>;  // mapping 8
static_assert(Bt7::smem_bytes<kSpread>() <= 227 * 1024, "mapping 7 fits shared memory");
static_assert(Bt8::smem_bytes<kSpread>() <= 227 * 1024, "mapping 8 fits shared memory");
// Per-frame masks on mapping 8's tiles (same rows and chunks, so the same
// records): one frame per lane leaves registers for the four sums.
// Two frames per lane for 4-byte pixels (the FP64 folds leave the registers
// for four sums of two frames: 76 k against 72 k frames/s on the Eiger-4M
// batch); 2-byte pixels, whose mask and pixel loads are deferred in
// registers, keep one.
template <typename P>
using BtR = BtCfg<DG_BT8_ROWS, DG_BT8_DCAP, DG_BT8_PCAP, sizeof(P) == 2 ? 1 : 2, 4, DG_BT8_BUFS,
                  DG_BT8_AHEAD>;
static_assert(BtR<float>::kMetaWords == Bt8::kMetaWords &&
                  BtR<uint16_t>::kMetaWords == Bt8::kMetaWords &&
                  BtR<float>::kMetaHead == Bt8::kMetaHead,
              "masked tiles read mapping 8's chunk records");
static_assert(BtR<float>::smem_bytes<kRaw>() <= 227 * 1024 &&
                  BtR<uint16_t>::smem_bytes<kRaw>() <= 227 * 1024,
              "masked tiles fit shared memory");

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}

// Shared-memory mbarriers of the bin-tile chunk pipeline.
__device__ __forceinline__ unsigned smem_addr(const void *p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(b)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(b)) : "memory");
}
// Arrives (without raising the expected count) once all of this thread's
// earlier cp.async copies have landed.
__device__ __forceinline__ void mbar_arrive_copies(uint64_t *b) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(smem_addr(b))
                 : "memory");
}
// Waits for the phase of the given parity to complete; gives up (false)
// after kBtWaitNs of global time, so a lost arrival cannot hang the GPU.
// (A suspend-time hint on the try, 1 ms, measured 2% slower on mapping 8.)
constexpr uint64_t kBtWaitNs = 1000000000ull;
// Tries between two reads of the global timer, and the pause (ns) after a
// failed try (0: none), of a waiting warp.
#ifndef DG_BT_WAIT_TRIES
#define DG_BT_WAIT_TRIES 1
#endif
#ifndef DG_BT_WAIT_SLEEP
#define DG_BT_WAIT_SLEEP 0
#endif
__device__ __forceinline__ bool mbar_try(unsigned a, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    return now;
}
__device__ __forceinline__ bool mbar_wait(uint64_t *b, unsigned parity) {
    const unsigned a = smem_addr(b);
    if (mbar_try(a, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
#pragma unroll 1
        for (int n = 0; n < DG_BT_WAIT_TRIES; ++n) {
            if (DG_BT_WAIT_SLEEP > 0) __nanosleep(DG_BT_WAIT_SLEEP);
            if (mbar_try(a, parity)) return true;
        }
        if (global_ns() - t0 > kBtWaitNs) return false;
    }
}

template <int MODE, typename P, class CFG>
__global__ void __launch_bounds__(CFG::kThreads, 1)
    k_gather_bins(const int4 *__restrict__ items, const int32_t *__restrict__ meta,
                  const float4 *__restrict__ pair_a, const float4 *__restrict__ pair_b,
                  const float2 *__restrict__ pair_c,
                  const int4 *__restrict__ org, const float4 *__restrict__ entry_std,
                  const double *__restrict__ den, const double *__restrict__ den_std,
                  const int32_t *__restrict__ valid_std,
                  const P *__restrict__ frames, int64_t n_pixels, int n_frames, int n_rows,
                  double *__restrict__ out_i, double *__restrict__ out_s,
                  double *__restrict__ out_d, int *__restrict__ wait_err, int withhold,
                  const double *__restrict__ raw_cnt, double *__restrict__ out_c, int raw,
                  const uint8_t *__restrict__ masks, int64_t mask_stride, int paired) {
    using S = StagedPx<P>;
    constexpr int NA = NAcc<MODE, P>::value;
    constexpr bool SPREAD = MODE == kSpread;
    constexpr int F2 = CFG::kF2, STRIDE = CFG::kStride, DCAP = CFG::kDCap, PCAP = CFG::kPCap;
    // Float pixels with the spread keep five sums per frame (the excluded
    // non-finite weights): half the unroll keeps them in registers.
#ifndef DG_BT_FLOAT_SPREAD_U2
#define DG_BT_FLOAT_SPREAD_U2 2
#endif
    constexpr int U2 = (SPREAD && is_float_px<P>() && CFG::kU2 > DG_BT_FLOAT_SPREAD_U2)
                           ? DG_BT_FLOAT_SPREAD_U2
                           : CFG::kU2;
    constexpr int NT = CFG::kThreads, NW = CFG::kRows;
    constexpr int NB = CFG::kBufs, NM = CFG::kMetaBufs, AH = CFG::kAhead, MA = CFG::kMetaAhead;
    constexpr int MH = CFG::kMetaHead, MW = CFG::kMetaWords;
    constexpr size_t BUF = CFG::template buf_bytes<MODE>();
    constexpr bool WIDE = SPREAD || MODE == kRaw;  // 32-byte entry pairs
    constexpr int MS = CFG::kMStride;
    extern __shared__ __align__(16) unsigned char smem[];
    const int groups = (n_frames + CFG::kFrames - 1) / CFG::kFrames;
    // Paired tiles: the two CTAs of a cluster take neighbouring tiles 2m and
    // 2m + 1 for the same frames.
    int item_idx, group;
    if (paired) {
        const int per = 2 * groups, m = int(blockIdx.x) / per, rm = int(blockIdx.x) % per;
        item_idx = 2 * m + (rm & 1);
        group = rm >> 1;
    } else {
        item_idx = int(blockIdx.x) / groups;
        group = int(blockIdx.x) % groups;
    }
    const int4 it = items[item_idx];
    const int f0 = group * CFG::kFrames;
    const int nv = min(CFG::kFrames, n_frames - f0);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int row0 = it.x, nrows = it.y, ch0 = it.z, nch = it.w;
    // Failure-detection check (dg_plan_test_wait_timeout): warp 0 of the first
    // CTA never reports a chunk summed, so the waits for its buffers run out.
    const bool signal = !(withhold && blockIdx.x == 0 && warp == 0);

    auto pxbuf = [&](int b) { return reinterpret_cast<S *>(smem + size_t(b) * BUF); };
    // Staged pixel of (local frame f, slot k). With two frames per lane the
    // lane's frames l and l + 32 can sit side by side (PAIRED: one 8-byte
    // shared load reads a slot for both; rows of 2 * STRIDE words, STRIDE odd,
    // so the 16 lanes of a half-warp hit 16 distinct bank pairs).
    constexpr bool PAIRED = DG_BT_PAIRED && F2 == 2 && MODE != kRaw;
    auto pxi = [&](int f, int k) {
        return PAIRED ? (f & 31) * 2 * STRIDE + 2 * k + (f >> 5) : f * STRIDE + k;
    };
    auto pabuf = [&](int b) {
        return reinterpret_cast<float4 *>(smem + size_t(b) * BUF +
                                          size_t(CFG::kFrames) * STRIDE * 4);
    };
    auto mbuf = [&](int c) {
        return reinterpret_cast<int32_t *>(smem + size_t(NB) * BUF) + (c % NM) * MW;
    };
    auto mkbuf = [&](int b) {  // mask rows (mode kRaw)
        return smem + size_t(b) * BUF + size_t(CFG::kFrames) * STRIDE * 4 + size_t(PCAP) * 32;
    };
    auto pcbuf = [&](int b) {  // pairs C (spread)
        return reinterpret_cast<f2 *>(smem + size_t(b) * BUF + size_t(CFG::kFrames) * STRIDE * 4 +
                                      size_t(PCAP) * 32);
    };
    // full[b]: chunk in buffer b landed (every thread's copies and stores);
    // empty[b]: every warp has summed the chunk in buffer b; rec[m]: the
    // record in slot m landed.
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + CFG::template bar_offset<MODE>());
    uint64_t *empty = full + NB, *rec = full + 2 * NB;
    if (tid == 0) {
        for (int b = 0; b < NB; ++b) {
            mbar_init(full + b, NT);
            mbar_init(empty + b, NW);
        }
        for (int m = 0; m < NM; ++m) mbar_init(rec + m, NT);
    }
    // Column DCAP of every frame row is read by padding pairs and holds 0.
    for (int j = tid; j < NB * CFG::kFrames; j += NT) {
        pxbuf(j / CFG::kFrames)[pxi(j % CFG::kFrames, DCAP)] = S(0);
        if constexpr (MODE == kRaw) mkbuf(j / CFG::kFrames)[(j % CFG::kFrames) * MS + DCAP] = 0;
    }
    __syncthreads();

    // Copy chunk c's record into its slot; every thread arrives on the
    // slot's barrier once its copies have landed (all threads arriving, not
    // only the copying ones, measured faster: 2.03 against 2.67 ms).
    auto stage_meta = [&](int c) {
        const int4 *src = reinterpret_cast<const int4 *>(meta + int64_t(ch0 + c) * MW);
        int4 *dst = reinterpret_cast<int4 *>(mbuf(c));
        for (int j = tid; j < MW / 4; j += NT) cp_async16(dst + j, src + j);
        mbar_arrive_copies(rec + c % NM);
    };
    // Stage chunk c into buffer c % NB (its record is in shared memory); every
    // thread arrives on the buffer's full barrier, counted once its copies
    // have landed and ordering its plain stores (2-byte pixels) before it.
    // Mode kRaw: a chunk's mask bytes, loaded with its copies and stored into
    // shared memory only after the warp has summed the chunk before it, so
    // the loads' latency hides behind that work.
    constexpr int KS = CFG::kSlices, FS = CFG::kStageFrames, FSTEP = CFG::kRows / KS;
    constexpr int KSTEP = ((DCAP + KS - 1) / KS + 31) / 32;
    unsigned mv[MODE == kRaw ? KSTEP : 1][FS];
    // 2-byte pixels are loaded, not copied: their loads are deferred the same
    // way where the registers allow it (512 threads, no spread).
    constexpr bool DEFER_PX = DG_BT_DEFER_PX && sizeof(P) != 4 && MODE != kSpread && NT <= 512;
    constexpr bool DEFER = MODE == kRaw || DEFER_PX;
    S pv[DEFER_PX ? KSTEP : 1][FS];
    // The first of two halves of staging chunk c: mask loads and copies.
    // The frames this warp stages (4-byte pixels), found once per tile.
    const P *stage_frame[FS];
    const uint64_t l2pol = bt_l2_policy();
#pragma unroll
    for (int j = 0; j < FS; ++j)
        stage_frame[j] = frames + int64_t(f0 + min(warp / KS + j * FSTEP, max(nv - 1, 0))) * n_pixels;
    auto stage_issue = [&](int c, int b) {  // b = c % NB
        const int32_t *mb = mbuf(c);
        const int4 ch = make_int4(0, mb[0], mb[2], mb[1]);  // {-, pixels, first pair, pairs}
        const int per = (ch.y + KS - 1) / KS, s0 = (warp % KS) * per;
        const int k1 = min(ch.y, s0 + per), fw = warp / KS;
        S *dst = pxbuf(b);
        const P *base = frames + int64_t(f0 + fw) * n_pixels;
        if constexpr (MODE == kRaw) {
#pragma unroll
            for (int i = 0; i < KSTEP; ++i) {
                const int k = s0 + lane + 32 * i;
#pragma unroll
                for (int j = 0; j < FS; ++j) {
                    const int f = fw + j * FSTEP;
                    mv[i][j] = k < k1 && f < nv
                                   ? unsigned(__ldg(masks + int64_t(f0 + f) * mask_stride + mb[MH + k]))
                                   : 0u;
                }
            }
        }
        if constexpr (DEFER_PX) {
#pragma unroll
            for (int i = 0; i < KSTEP; ++i) {
                const int k = s0 + lane + 32 * i;
#pragma unroll
                for (int j = 0; j < FS; ++j)
                    pv[i][j] = k < k1 && fw + j * FSTEP < nv
                                   ? load_px<P>(base + mb[MH + k] + int64_t(j * FSTEP) * n_pixels, 0u)
                                   : S(0);
            }
        } else if constexpr (sizeof(P) == 4) {
            // This lane's slots s0 + lane + 32 i and their pixel indices, read
            // once; then frame by frame, one address add and one copy per
            // (slot, frame).
            uint32_t boff[KSTEP];  // byte offsets of the slots' pixels in a frame
            bool kin[KSTEP];
#pragma unroll
            for (int i = 0; i < KSTEP; ++i) {
                const int k = s0 + lane + 32 * i;
                kin[i] = k < k1;
                boff[i] = kin[i] ? uint32_t(mb[MH + k]) * uint32_t(sizeof(P)) : 0u;
            }
#pragma unroll
            for (int j = 0; j < FS; ++j) {
                const int f = fw + j * FSTEP;
                if (f >= nv) break;
#if DG_BT_SADDR
                const char *fsrc = reinterpret_cast<const char *>(stage_frame[j]);
                const unsigned drow = smem_addr(dst + pxi(f, s0 + lane));
                constexpr unsigned kStep = 4u * (PAIRED ? 64u : 32u);  // 32 slots on
#pragma unroll
                for (int i = 0; i < KSTEP; ++i)
                    if (kin[i]) cp_async4_sp(drow + kStep * unsigned(i), fsrc + boff[i], l2pol);
#else
                const P *fsrc = base + int64_t(j * FSTEP) * n_pixels;
                int idx[KSTEP];
#pragma unroll
                for (int i = 0; i < KSTEP; ++i) idx[i] = int(boff[i] / uint32_t(sizeof(P)));
#pragma unroll
                for (int i = 0; i < KSTEP; ++i)
                    if (kin[i]) cp_async4(dst + pxi(f, s0 + lane + 32 * i), fsrc + idx[i]);
#endif
            }
        } else {
            for (int k = s0 + lane; k < k1; k += 32) {
                const P *src = base + mb[MH + k];
#pragma unroll
                for (int j = 0; j < FS; ++j) {
                    if (fw + j * FSTEP >= nv) break;
                    dst[pxi(fw + j * FSTEP, k)] = load_px<P>(src + int64_t(j * FSTEP) * n_pixels, 0u);
                }
            }
        }
        float4 *pa = pabuf(b);
        f2 *pc = pcbuf(b);
        for (int j = tid; j < ch.w; j += NT) {
            cp_async16(pa + j, pair_a + ch.z + j);
            if (WIDE) cp_async16(pa + PCAP + j, pair_b + ch.z + j);
            if (SPREAD) cp_async8(pc + j, pair_c + ch.z + j);
        }
    };
    // The second half: mask stores, then this thread's arrival on the
    // buffer's full barrier.
    auto stage_finish = [&](int c, int b) {
        if constexpr (DEFER_PX) {
            const int dn = mbuf(c)[0];
            const int per = (dn + KS - 1) / KS, s0 = (warp % KS) * per;
            const int k1 = min(dn, s0 + per), fw = warp / KS;
            S *dst = pxbuf(b);
#pragma unroll
            for (int i = 0; i < KSTEP; ++i) {
                const int k = s0 + lane + 32 * i;
#pragma unroll
                for (int j = 0; j < FS; ++j)
                    if (k < k1 && fw + j * FSTEP < nv) dst[pxi(fw + j * FSTEP, k)] = pv[i][j];
            }
        }
        if constexpr (MODE == kRaw) {
            const int32_t *mb = mbuf(c);
            const int dn = mb[0];
            const int per = (dn + KS - 1) / KS, s0 = (warp % KS) * per;
            const int k1 = min(dn, s0 + per), fw = warp / KS;
            unsigned char *md = mkbuf(b);
#pragma unroll
            for (int i = 0; i < KSTEP; ++i) {
                const int k = s0 + lane + 32 * i;
#pragma unroll
                for (int j = 0; j < FS; ++j) {
                    const int f = fw + j * FSTEP;
                    if (k < k1 && f < nv) md[f * MS + k] = static_cast<unsigned char>(mv[i][j]);
                }
            }
        }
        asm volatile("cp.async.mbarrier.arrive.shared::cta.b64 [%0];\n" ::"r"(smem_addr(full + b))
                     : "memory");
        mbar_arrive(full + b);
    };
    auto stage = [&](int c, int b) {
        stage_issue(c, b);
        stage_finish(c, b);
    };

    // This warp's row: accumulators, fold counter and origin of each of the
    // lane's frames.
    BtAcc acc[F2][NA];
#pragma unroll
    for (int h = 0; h < F2; ++h)
#pragma unroll
        for (int a = 0; a < NA; ++a) acc[h][a].zero();
    int since = 0;
    const int r = warp;  // row of the tile
    // Origin of the spread's shift, per frame of the lane: the row's origin
    // entry {origin, first valid, row end} read from the frames before the
    // first chunk (row_origin).
    float orgv[F2];
#pragma unroll
    for (int h = 0; h < F2; ++h) orgv[h] = 0.f;
    if constexpr (SPREAD) {
        if (r < nrows) {
            const int4 o = org[row0 + r];
#pragma unroll
            for (int h = 0; h < F2; ++h) {
                const int fi = min(f0 + lane + 32 * h, n_frames - 1);
                orgv[h] = row_origin<P>(entry_std, o.x, o.y, o.z, frames + int64_t(fi) * n_pixels);
            }
        }
    }
    f2 norg[F2];
#pragma unroll
    for (int h = 0; h < F2; ++h) norg[h] = pk(-orgv[h], -orgv[h]);

    // Pipeline without a CTA-wide barrier: in step c a warp stages its share
    // of chunk c + AH (once every warp has summed the chunk that buffer held)
    // and of record c + AH + MA, then sums chunk c once all its shares have
    // landed. A warp may fall kLag chunks behind the fastest, so rows whose
    // entries are unevenly spread over the chunks even out over the tile.
    bool ok = true;
    for (int j = 0; j < AH + MA && j < nch; ++j) stage_meta(j);
    static_assert(AH < NB, "the first chunks go to buffers 0..AH-1");
    for (int j = 0; j < AH && j < nch; ++j) {
        if (ok) ok = mbar_wait(rec + j % NM, unsigned(j / NM) & 1u);
        if (ok) stage(j, j);
    }
    // Buffers and phases of chunks c and j = c + AH, kept as counters (c % NB
    // and c / NB without a division per chunk).
    int cb = 0, cq = 0, jb = AH, jq = 0;
    for (int c = 0; c < nch; ++c) {
        const int j = c + AH;
        bool pending = false;  // chunk j's second staging half, after chunk c
        if (j < nch) {
            if (ok && j >= NB) ok = mbar_wait(empty + jb, unsigned(jq - 1) & 1u);
            if (ok && j + MA < nch) stage_meta(j + MA);
            if (ok) ok = mbar_wait(rec + j % NM, unsigned(j / NM) & 1u);
            if (ok) {
                if constexpr (DEFER) {
                    stage_issue(j, jb);
                    pending = true;
                } else {
                    stage(j, jb);
                }
            }
        }
        if (ok) ok = mbar_wait(full + cb, unsigned(cq) & 1u);
        if (!__all_sync(0xffffffffu, ok)) {
            ok = false;
            break;
        }
        const int b = cb, pb = jb;  // pb: chunk j's buffer, for its second half
        if (++cb == NB) {
            cb = 0;
            ++cq;
        }
        if (++jb == NB) {
            jb = 0;
            ++jq;
        }
        if (r >= nrows) {
            if (pending) stage_finish(j, pb);
            if (lane == 0 && signal) mbar_arrive(empty + b);
            continue;
        }
        const S *px[F2];
        unsigned pxa[F2];  // the same as 32-bit shared-memory addresses
#pragma unroll
        for (int h = 0; h < F2; ++h) {
            px[h] = pxbuf(b) + pxi(lane + 32 * h, 0);
            pxa[h] = smem_addr(px[h]);
        }
        const float4 *s_pa = pabuf(b);
        const float4 *s_pb = s_pa + PCAP;
        const f2 *s_pc = pcbuf(b);
        const unsigned char *mk[F2];  // this lane's mask rows (mode kRaw)
#pragma unroll
        for (int h = 0; h < F2; ++h) mk[h] = mkbuf(b) + (lane + 32 * h) * MS;
        const int32_t *cp = mbuf(c) + 4;
        const int p0 = cp[r], p1 = cp[r + 1];
        auto body = [&](int p, auto unroll) {
            constexpr int UU = decltype(unroll)::value;
            float4 ea[UU], eb[UU];
            f2 ec[UU];
#pragma unroll
            for (int u = 0; u < UU; ++u) {
                ea[u] = s_pa[p + u];
                if constexpr (WIDE) eb[u] = s_pb[p + u];
                if constexpr (SPREAD) ec[u] = s_pc[p + u];
            }
            // the pair's pixels for this lane's frames
            float vv0[F2][UU], vv1[F2][UU];
            if constexpr (PAIRED) {
#pragma unroll
                for (int u = 0; u < UU; ++u) {
                    using S2 = typename std::conditional<std::is_same<S, float>::value, float2,
                               typename std::conditional<std::is_same<S, int32_t>::value, int2,
                                                         uint2>::type>::type;
                    const S2 a = *reinterpret_cast<const S2 *>(px[0] + 2 * __float_as_int(ea[u].x));
                    const S2 b2 = *reinterpret_cast<const S2 *>(px[0] + 2 * __float_as_int(ea[u].y));
                    vv0[0][u] = float(a.x);
                    vv0[F2 - 1][u] = float(a.y);
                    vv1[0][u] = float(b2.x);
                    vv1[F2 - 1][u] = float(b2.y);
                }
            } else if constexpr (DG_BT_SADDR && MODE != kRaw) {
#pragma unroll
                for (int h = 0; h < F2; ++h)
#pragma unroll
                    for (int u = 0; u < UU; ++u) {
                        vv0[h][u] = staged_value<S>(
                            lds32(pxa[h] + 4u * unsigned(__float_as_int(ea[u].x))));
                        vv1[h][u] = staged_value<S>(
                            lds32(pxa[h] + 4u * unsigned(__float_as_int(ea[u].y))));
                    }
            } else {
#pragma unroll
                for (int h = 0; h < F2; ++h)
#pragma unroll
                    for (int u = 0; u < UU; ++u) {
                        vv0[h][u] = float(px[h][__float_as_int(ea[u].x)]);
                        vv1[h][u] = float(px[h][__float_as_int(ea[u].y)]);
                    }
            }
#pragma unroll
            for (int h = 0; h < F2; ++h) {
                float(&v0)[UU] = vv0[h];
                float(&v1)[UU] = vv1[h];
                if constexpr (MODE == kRaw) {
                    // Per-frame masks: {slot, slot, w, w}, {w*norm, w*norm, 0, 0};
                    // a masked entry adds nothing to S, V, N or C, whatever its
                    // pixel holds.
#pragma unroll
                    for (int u = 0; u < UU; ++u) {
                        const bool l0 = mk[h][__float_as_int(ea[u].x)] == 0;
                        const bool l1 = mk[h][__float_as_int(ea[u].y)] == 0;
                        const f2 cc = pk(l0 ? ea[u].z : 0.f, l1 ? ea[u].w : 0.f);
                        const float x0 = l0 ? v0[u] : 0.f, x1 = l1 ? v1[u] : 0.f;
                        const f2 x = pk(x0, x1);
                        acc[h][0].p = fma2(cc, x, acc[h][0].p);
                        const f2 xp = is_unsigned_px<P>() ? x : pk(fmaxf(x0, 0.f), fmaxf(x1, 0.f));
                        acc[h][1].p = fma2(mul2(cc, cc), xp, acc[h][1].p);
                        acc[h][2].p = add2(acc[h][2].p, pk(l0 ? eb[u].x : 0.f, l1 ? eb[u].y : 0.f));
                        acc[h][3].p = add2(acc[h][3].p, cc);
                    }
                    continue;
                }
#pragma unroll
                for (int u = 0; u < UU; ++u) {
                    const f2 cc = pk(ea[u].z, ea[u].w);
                    if constexpr (SPREAD && is_float_px<P>()) {
                        if (!(isfinite(v0[u]) && isfinite(v1[u]))) {
                            const bool ok0 = isfinite(v0[u]), ok1 = isfinite(v1[u]);
                            const float x0 = ok0 ? v0[u] : 0.f, x1 = ok1 ? v1[u] : 0.f;
                            const f2 ce = pk(ok0 ? ea[u].z : 0.f, ok1 ? ea[u].w : 0.f);
                            const f2 x = pk(x0, x1), n = pk(eb[u].x, eb[u].y);
                            const f2 cre = pk(ok0 ? eb[u].z : 0.f, ok1 ? eb[u].w : 0.f);
                            acc[h][0].p = fma2(ce, x, acc[h][0].p);
                            acc[h][1].p = fma2(mul2(ce, ce), pk(fmaxf(x0, 0.f), fmaxf(x1, 0.f)),
                                               acc[h][1].p);
                            const f2 t = fma2(norg[h], ec[u], fma2(norg[h], n, x));
                            acc[h][2].p = fma2(mul2(cre, t), t, acc[h][2].p);
                            acc[h][kSpreadA].p = fma2(ce, t, acc[h][kSpreadA].p);
                            acc[h][NA - 2].p = add2(acc[h][NA - 2].p,
                                                    pk(ok0 ? 0.f : __fmul_rn(ea[u].z, eb[u].x),
                                                       ok1 ? 0.f : __fmul_rn(ea[u].w, eb[u].y)));
                            acc[h][NA - 1].p = add2(acc[h][NA - 1].p,
                                                    pk(!ok0 && ea[u].z > 0.f ? 1.f : 0.f,
                                                       !ok1 && ea[u].w > 0.f ? 1.f : 0.f));
                            continue;
                        }
                    }
                    const f2 x = pk(v0[u], v1[u]);
                    acc[h][0].p = fma2(cc, x, acc[h][0].p);
                    if constexpr (MODE != kIntensity) {
                        const f2 xp = is_unsigned_px<P>()
                                          ? x
                                          : pk(fmaxf(v0[u], 0.f), fmaxf(v1[u], 0.f));
                        acc[h][1].p = fma2(mul2(cc, cc), xp, acc[h][1].p);
                    }
                    if constexpr (SPREAD) {
                        const f2 n = pk(eb[u].x, eb[u].y), cr = pk(eb[u].z, eb[u].w);
                        const f2 t = fma2(norg[h], ec[u], fma2(norg[h], n, x));
                        acc[h][2].p = fma2(mul2(cr, t), t, acc[h][2].p);
                        acc[h][kSpreadA].p = fma2(cc, t, acc[h][kSpreadA].p);
                    }
                }
            }
        };
        auto fold = [&]() {
#pragma unroll
            for (int h = 0; h < F2; ++h)
#pragma unroll
                for (int a = 0; a < NA; ++a) acc[h][a].flush();
        };
        int p = p0;
        for (; p + U2 <= p1; p += U2) {
            body(p, std::integral_constant<int, U2>{});
            since += U2;
            if (since >= kBtFoldPairs) {
                since = 0;
                fold();
            }
        }
        for (; p < p1; ++p) {
            body(p, std::integral_constant<int, 1>{});
            if (++since >= kBtFoldPairs) {
                since = 0;
                fold();
            }
        }
        if (pending) stage_finish(j, pb);
        __syncwarp();
        if (lane == 0 && signal) mbar_arrive(empty + b);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    if (!ok) {
        // A wait gave up: this tile's sums are incomplete. The host finds the
        // flag (mapped host memory) and reports the call as failed.
        if (lane == 0) {
            *reinterpret_cast<volatile int *>(wait_err) = 1;
            __threadfence_system();
        }
        return;
    }
    if (r >= nrows) return;

    // Normalise (normalize_bin, prepared.rs:985-996; the spread's closing
    // formulas, azimuthal.rs:96-104), as k_finalize does from partial sums.
#pragma unroll
    for (int h = 0; h < F2; ++h) {
        const int fl = lane + 32 * h;
        if (fl >= nv) continue;
        const int row = row0 + r;
        double v[NA];
#pragma unroll
        for (int a = 0; a < NA; ++a) {
            acc[h][a].flush();
            v[a] = acc[h][a].value();
        }
        const int64_t oo = int64_t(f0 + fl) * n_rows + row;
        if constexpr (MODE == kRaw) {
            // Sums of this frame's mask: raw (integrate1d_raw*) or normalised
            // by the frame's own N (normalize_bin), as k_finalize_raw and
            // k_finalize<kRaw> do from partial sums.
            if (raw) {
                out_i[oo] = v[0];
                out_d[oo] = v[2];
                if (out_s) out_s[oo] = v[1];
                out_c[oo] = v[3];
            } else {
                const double n = v[2];
                out_i[oo] = n == 0.0 ? 0.0 : v[0] / n;
                if (out_s) {
                    const double q = n == 0.0 ? 0.0 : v[1] / (n * n);
                    out_s[oo] = sqrt(q > 0.0 ? q : 0.0);
                }
            }
            continue;
        }
        if (raw) {
            // Raw sums (integrate1d_raw*, integrate.rs:682-797): signal and
            // variance sums of the frame, the row's strict norm and weight sums.
            out_i[oo] = v[0];
            if (NA > 1 && out_s) out_s[oo] = v[NA > 1 ? 1 : 0];
            out_d[oo] = den[row];
            out_c[oo] = raw_cnt[row];
            continue;
        }
        if constexpr (!SPREAD) {
            const double n = den[row];
            out_i[oo] = n == 0.0 ? 0.0 : v[0] / n;
            if (MODE == kErrors) {
                const double q = n == 0.0 ? 0.0 : v[1] / (n * n);
                out_s[oo] = sqrt(q > 0.0 ? q : 0.0);
            }
        } else {
            int valid = valid_std[row];
            double sw = den_std[row];
            if (NA == 6) {
                valid -= int(v[NA - 1] + 0.5);
                sw -= v[NA - 2];
            }
            if (valid <= 0 || !(sw > 0.0)) {
                out_i[oo] = 0.0;
                if (out_s) out_s[oo] = 0.0;
                out_d[oo] = __longlong_as_double(0x7ff8000000000000ll);
                continue;
            }
            const double a1 = v[kSpreadA];
            out_i[oo] = v[0] / sw;
            if (out_s) out_s[oo] = sqrt(v[1] > 0.0 ? v[1] : 0.0) / sw;
            const double mean = a1 / sw;
            const double m2 = v[2] - mean * a1;
            const double q = m2 / sw;
            // one valid contribution: its deviation from itself is exactly 0
            out_d[oo] = valid == 1 ? 0.0 : sqrt(q > 0.0 ? q : 0.0);
        }
    }
}

// Bin-tile entry pairs from the plan-time layout: per pair {slot 0, slot 1,
// entry 0, entry 1} (entry -1: padding, slot = the zero column) to A {slot 0, slot 1,
// c0, c1} with the table's FP32 weights, AS the same with the spread's
// weights, B {n0, n1, c0/n0, c1/n1}.
__global__ void k_bt_fill(const int4 *__restrict__ desc, int64_t n_pairs,
                          const int2 *__restrict__ entry, const float4 *__restrict__ entry_std,
                          const float *__restrict__ entry_nlo, float4 *__restrict__ pair_a,
                          float4 *__restrict__ pair_as, float4 *__restrict__ pair_b,
                          float2 *__restrict__ pair_c) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n_pairs;
         i += int64_t(gridDim.x) * blockDim.x) {
        const int4 d = desc[i];
        float c[2] = {0.f, 0.f}, cs[2] = {0.f, 0.f}, n[2] = {1.f, 1.f}, cr[2] = {0.f, 0.f},
              nlo[2] = {0.f, 0.f};
        const int k[2] = {d.z, d.w};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (k[h] < 0) continue;
            c[h] = __int_as_float(entry[k[h]].y);
            const float4 es = entry_std[k[h]];
            cs[h] = es.y;
            n[h] = es.z;
            cr[h] = es.w;
            nlo[h] = entry_nlo[k[h]];
        }
        pair_a[i] = make_float4(__int_as_float(d.x), __int_as_float(d.y), c[0], c[1]);
        pair_as[i] = make_float4(__int_as_float(d.x), __int_as_float(d.y), cs[0], cs[1]);
        pair_b[i] = make_float4(n[0], n[1], cr[0], cr[1]);
        pair_c[i] = make_float2(nlo[0], nlo[1]);
    }
}

// Pairs of the per-frame-mask bin tiles from the same layout: A {slot 0,
// slot 1, w0, w1} and B {w0*norm, w1*norm, 0, 0} with the raw entries'
// FP32 weights (k_pack_raw); padding entries are zero.
__global__ void k_bt_fill_raw(const int4 *__restrict__ desc, int64_t n_pairs,
                              const float4 *__restrict__ entry_raw, float4 *__restrict__ pair_a,
                              float4 *__restrict__ pair_b) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n_pairs;
         i += int64_t(gridDim.x) * blockDim.x) {
        const int4 d = desc[i];
        float w[2] = {0.f, 0.f}, wn[2] = {0.f, 0.f};
        const int k[2] = {d.z, d.w};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (k[h] < 0) continue;
            const float4 e = entry_raw[k[h]];
            w[h] = e.y;
            wn[h] = e.z;
        }
        pair_a[i] = make_float4(__int_as_float(d.x), __int_as_float(d.y), w[0], w[1]);
        pair_b[i] = make_float4(wn[0], wn[1], 0.f, 0.f);
    }
}

// One thread per (frame, row): fold the row's segment partials in strip
// order in FP64 and normalise (normalize_bin, prepared.rs:985-996; the
// spread's closing formulas, azimuthal.rs:96-104).
constexpr int kFinRows = 8;  // rows per k_finalize CTA (x 32 frames)
// One tile of kFinRows rows from r0 and 32 frames from fb, by a CTA of 256
// threads: lanes run over frames while the partial sums are read
// (frame-contiguous), the results go through shared memory and are written
// row-contiguous for each frame. Ends with a CTA barrier, so the next tile
// may reuse the shared memory at once.
template <int MODE, typename P>
__device__ __forceinline__ void finalize_tile(
    int r0, int fb, const double *__restrict__ partial, const int32_t *__restrict__ row_seg,
    const int32_t *__restrict__ seg_ids, const double *__restrict__ den,
    const double *__restrict__ den_std, const int32_t *__restrict__ valid_std, int n_rows,
    int n_frames, double *__restrict__ out_i, double *__restrict__ out_s,
    double *__restrict__ out_d) {
    constexpr int NA = NAcc<MODE, P>::value;
    __shared__ double s_o[3][kFinRows][33];
    const int fl = threadIdx.x & 31, rl = threadIdx.x >> 5;
    const int r = r0 + rl, f = fb + fl;
    double ri = 0.0, rs = 0.0, rd = 0.0;
    if (r < n_rows && f < n_frames) {
        double v[NA];
        for (int a = 0; a < NA; ++a) v[a] = 0.0;
        const int k0 = row_seg[r], k1 = row_seg[r + 1];
        for (int k = k0; k < k1; ++k) {
            const double *p = partial + int64_t(seg_ids[k]) * NA * n_frames + f;
            for (int a = 0; a < NA; ++a) v[a] = __dadd_rn(v[a], p[int64_t(a) * n_frames]);
        }
        if (MODE == kRaw) {  // denominators of this frame's mask
            const double n = v[2];
            ri = n == 0.0 ? 0.0 : v[0] / n;
            const double q = n == 0.0 ? 0.0 : v[1] / (n * n);
            rs = sqrt(q > 0.0 ? q : 0.0);
        } else if (MODE != kSpread) {
            const double n = den[r];
            ri = n == 0.0 ? 0.0 : v[0] / n;
            if (MODE == kErrors) {
                const double q = n == 0.0 ? 0.0 : v[1] / (n * n);
                rs = sqrt(q > 0.0 ? q : 0.0);
            }
        } else {
            int valid = valid_std[r];
            double sw = den_std[r];
            if (NA == 6) {
                valid -= int(v[NA - 1] + 0.5);
                sw -= v[NA - 2];
            }
            if (valid <= 0 || !(sw > 0.0)) {
                rd = __longlong_as_double(0x7ff8000000000000ll);
            } else {
                const double a1 = v[kSpreadA];
                ri = v[0] / sw;
                rs = sqrt(v[1] > 0.0 ? v[1] : 0.0) / sw;
                const double mean = a1 / sw;
                const double m2 = v[2] - mean * a1;
                const double q = m2 / sw;
                // one valid contribution: its deviation from itself is exactly 0
                rd = valid == 1 ? 0.0 : sqrt(q > 0.0 ? q : 0.0);
            }
        }
    }
    s_o[0][rl][fl] = ri;
    s_o[1][rl][fl] = rs;
    s_o[2][rl][fl] = rd;
    __syncthreads();
    const int wr = threadIdx.x % kFinRows, wf = threadIdx.x / kFinRows;
    const int rr = r0 + wr, ff = fb + wf;
    if (rr < n_rows && ff < n_frames) {
        const int64_t o = int64_t(ff) * n_rows + rr;
        out_i[o] = s_o[0][wr][wf];
        if (MODE != kIntensity && out_s) out_s[o] = s_o[1][wr][wf];
        if (MODE == kSpread) out_d[o] = s_o[2][wr][wf];
    }
    __syncthreads();
}

template <int MODE, typename P>
__global__ void __launch_bounds__(256)
    k_finalize(const double *__restrict__ partial, const int32_t *__restrict__ row_seg,
               const int32_t *__restrict__ seg_ids, const double *__restrict__ den,
               const double *__restrict__ den_std, const int32_t *__restrict__ valid_std,
               int n_rows, int n_frames, double *__restrict__ out_i, double *__restrict__ out_s,
               double *__restrict__ out_d) {
    finalize_tile<MODE, P>(blockIdx.x * kFinRows, blockIdx.y * 32, partial, row_seg, seg_ids, den,
                           den_std, valid_std, n_rows, n_frames, out_i, out_s, out_d);
}

// Raw sums per (frame, row) (IntermediateResult1d, lut/integrate.rs:372-379):
// S and V from the partial sums; N and C from them too for the per-frame-mask
// gather, else the plan's strict FP64 denominator and weight sum.
template <int MODE>
__global__ void __launch_bounds__(256)
    k_finalize_raw(const double *__restrict__ partial, const int32_t *__restrict__ row_seg,
                   const int32_t *__restrict__ seg_ids, const double *__restrict__ den,
                   const double *__restrict__ cnt, int n_rows, int n_frames,
                   double *__restrict__ out_sig, double *__restrict__ out_norm,
                   double *__restrict__ out_var, double *__restrict__ out_cnt) {
    // Tiles of kFinRows rows x 32 frames, written row-contiguous per frame
    // through shared memory (as k_finalize).
    constexpr int NA = NAcc<MODE, float>::value;
    __shared__ double s_o[4][kFinRows][33];
    const int fl = threadIdx.x & 31, rl = threadIdx.x >> 5;
    const int r0 = blockIdx.x * kFinRows, fb = blockIdx.y * 32;
    const int r = r0 + rl, f = fb + fl;
    double v[NA];
    for (int a = 0; a < NA; ++a) v[a] = 0.0;
    if (r < n_rows && f < n_frames) {
        for (int k = row_seg[r]; k < row_seg[r + 1]; ++k) {
            const double *p = partial + int64_t(seg_ids[k]) * NA * n_frames + f;
            for (int a = 0; a < NA; ++a) v[a] = __dadd_rn(v[a], p[int64_t(a) * n_frames]);
        }
        s_o[0][rl][fl] = v[0];
        s_o[1][rl][fl] = NA > 1 ? v[1] : 0.0;
        s_o[2][rl][fl] = MODE == kRaw ? v[NA > 2 ? 2 : 0] : den[r];
        s_o[3][rl][fl] = MODE == kRaw ? v[NA > 3 ? 3 : 0] : cnt[r];
    }
    __syncthreads();
    const int wr = threadIdx.x % kFinRows, wf = threadIdx.x / kFinRows;
    const int rr = r0 + wr, ff = fb + wf;
    if (rr >= n_rows || ff >= n_frames) return;
    const int64_t o = int64_t(ff) * n_rows + rr;
    out_sig[o] = s_o[0][wr][wf];
    if (out_var) out_var[o] = s_o[1][wr][wf];
    out_norm[o] = s_o[2][wr][wf];
    out_cnt[o] = s_o[3][wr][wf];
}

// Entries for the per-frame-mask gather, {pixel, w, w*norm} in FP32 (the
// product formed in FP64), and the strict FP64 weight sum of every row.
__global__ void k_pack_raw(const int64_t *__restrict__ row_ptr, int n_rows,
                           const int32_t *__restrict__ col, const double *__restrict__ w,
                           const double *__restrict__ norm, float4 *__restrict__ entry_raw,
                           double *__restrict__ cnt, int flip_rows, int flip_cols) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    double sum = 0.0;
    for (int64_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
        const int32_t j = col[k];
        const double c = w[k];
        sum += c;
        // the frame's pixel (rows flipped for InputOrder::FlipVertical)
        int32_t jf = j;
        if (flip_rows) {
            const int32_t rr = j / flip_cols;
            jf = (flip_rows - 1 - rr) * flip_cols + (j - rr * flip_cols);
        }
        entry_raw[k] = make_float4(__int_as_float(jf), __double2float_rn(c),
                                   __double2float_rn(c * norm[j]), 0.f);
    }
    cnt[r] = sum;
}

// Packs the masked f64 table into the gather's entry formats and computes
// the spread's denominators over its valid entries (c > 0, n > 0, finite),
// its first valid entry and its origin entry (the heaviest valid, row_origin).
// The spread's n is stored as the pair (n_hi, n_lo): n_hi = FP32(n) in
// entry_std, n_lo = FP32(n - n_hi) in entry_nlo.
// Per-pixel norm as an FP32 pair for the row warps' spread, at frame
// storage index i: the detector pixel itself, or, for frames stored bottom row
// first (rows > 0), the pixel of the mirrored row.
__global__ void k_px_norm(const double *__restrict__ norm, int64_t n_px, int rows, int cols,
                          float2 *__restrict__ out) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n_px;
         i += int64_t(gridDim.x) * blockDim.x) {
        int64_t j = i;
        if (rows > 0) {
            const int64_t r = i / cols;
            j = (rows - 1 - r) * cols + (i - r * cols);
        }
        const double n = norm[j];
        const bool ok = isfinite(n) && n > 0.0;
        const float hi = ok ? __double2float_rn(n) : 0.f;
        out[i] = make_float2(hi, ok ? __double2float_rn(n - double(hi)) : 0.f);
    }
}

__global__ void k_pack(const int64_t *__restrict__ row_ptr, int n_rows,
                       const int32_t *__restrict__ col, const double *__restrict__ w,
                       const double *__restrict__ norm, int2 *__restrict__ entry,
                       float4 *__restrict__ entry_std, float *__restrict__ entry_nlo,
                       double *__restrict__ den_std, int32_t *__restrict__ valid_std,
                       int32_t *__restrict__ first_valid, int32_t *__restrict__ origin) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    double sw = 0.0, heaviest = 0.0;
    int valid = 0, first = -1, org = -1;
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
        entry_nlo[k] = ok ? __double2float_rn(n - double(nf)) : 0.f;
        if (ok) {
            sw += ww;
            ++valid;
            if (first < 0) first = int(k);
            if (ww > heaviest) {  // the first of equally heavy entries
                heaviest = ww;
                org = int(k);
            }
        }
    }
    den_std[r] = sw;
    valid_std[r] = valid;
    first_valid[r] = first;
    origin[r] = org;
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

template <int MODE, typename P, int U2, bool DB>
void launch_fl(const GatherTable &t, const P *fp, int64_t n_pixels, int nf, double *partial,
               cudaStream_t s) {
    if (t.fl_n_units <= 0)
        fail(DG_UNSUPPORTED, "the frame-lane gather is not available for this table");
    constexpr size_t smem = fl_smem_bytes<MODE, P, DB>();
    auto kern = k_gather_fl<MODE, P, U2, DB>;
    DG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const float4 *pa = MODE == kSpread ? t.fl_pair_as : t.fl_pair_a.ptr;
    kern<<<t.fl_n_units, kThreads, smem, s>>>(t.fl_unit.ptr, t.seg.ptr, t.fl_px.ptr, pa,
                                              t.fl_pair_b.ptr, t.fl_pair_c.ptr, t.entry_std.ptr,
                                              t.first_valid.ptr, t.origin.ptr, t.fl_seg_org.ptr,
                                              fp, n_pixels, nf, t.n_segments, partial);
}

// Launches lane-mapping variant `variant` of the gather (kVariantCount) with
// its partial sums in `partial`.
template <int MODE, typename P, class CFG>
void launch_bins(const GatherTable &t, const BinTiles &bt, const P *fp, int64_t n_pixels, int nf,
                 double *oi, double *os, double *od, cudaStream_t s, double *oc = nullptr,
                 int raw = 0, const uint8_t *masks = nullptr, int64_t mask_stride = 0) {
    constexpr size_t smem = CFG::template smem_bytes<MODE>();
    auto kern = k_gather_bins<MODE, P, CFG>;
    DG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const int groups = (nf + CFG::kFrames - 1) / CFG::kFrames;
    const int64_t grid = int64_t(bt.n_items) * groups;
    if (grid > INT32_MAX) fail(DG_UNSUPPORTED, "too many bin tiles for one launch");
    check_bin_tile_waits(t);
    const float4 *pa = MODE == kSpread ? bt.pair_as.ptr : MODE == kRaw ? bt.pair_ra.ptr : bt.pair_a.ptr;
    const float4 *pb = MODE == kRaw ? bt.pair_rb.ptr : bt.pair_b.ptr;
    const int paired = bt.paired ? 1 : 0;
    if (!paired) {
        kern<<<unsigned(grid), CFG::kThreads, smem, s>>>(
            bt.item.ptr, bt.meta.ptr, pa, pb, bt.pair_c.ptr, bt.org.ptr, t.entry_std.ptr,
            t.den.ptr, t.den_std.ptr, t.valid_std.ptr, fp, n_pixels, nf, t.n_rows, oi, os, od,
            bt.wait_err.dev, t.withhold_test, t.cnt.ptr, oc, raw, masks, mask_stride, paired);
        return;
    }
    // one 2-CTA cluster per (tile pair, frame group): both CTAs on one GPC
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(unsigned(grid), 1, 1);
    lc.blockDim = dim3(CFG::kThreads, 1, 1);
    lc.dynamicSmemBytes = smem;
    lc.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    DG_CUDA(cudaLaunchKernelEx(&lc, kern, static_cast<const int4 *>(bt.item.ptr),
                               static_cast<const int32_t *>(bt.meta.ptr), pa, pb,
                               static_cast<const float2 *>(bt.pair_c.ptr),
                               static_cast<const int4 *>(bt.org.ptr),
                               static_cast<const float4 *>(t.entry_std.ptr),
                               static_cast<const double *>(t.den.ptr),
                               static_cast<const double *>(t.den_std.ptr),
                               static_cast<const int32_t *>(t.valid_std.ptr), fp, n_pixels, nf,
                               int(t.n_rows), oi, os, od, bt.wait_err.dev, t.withhold_test,
                               static_cast<const double *>(t.cnt.ptr), oc, raw, masks,
                               mask_stride, paired));
}

// Row warps (mapping 10): F frames per pass over a row's entries, one CTA
// per (row item, block of F frames), so a launch of up to four frames reads
// every entry once and a larger one once per four frames.
template <int MODE, typename P>
void launch_rows(const GatherTable &t, const P *fp, int64_t n_pixels, int nf, double *oi,
                 double *os, double *od, cudaStream_t s) {
    const QueuePlan q = queue_plan(t, fp, n_pixels, nf, oi, os, od);
    const dim3 grid(unsigned(q.n_items), unsigned(q.frame_blocks));
    switch (rows_pass_frames(nf)) {
    case 1: k_rows<MODE, P, 1><<<grid, kRowsThreads, 0, s>>>(q); break;
    case 2: k_rows<MODE, P, 2><<<grid, kRowsThreads, 0, s>>>(q); break;
    default: k_rows<MODE, P, 4><<<grid, kRowsThreads, 0, s>>>(q); break;
    }
    DG_CUDA(cudaGetLastError());
}

// Launches lane mapping `variant`; returns true when the kernel wrote the
// normalised results to oi/os/od itself (mappings 7, 8, 10), false when it left
// partial sums for k_finalize. Those mappings need the outputs; callers without
// them (raw sums) get the frame-lane or an entry-lane mapping instead.
template <int MODE, typename P>
bool launch_gather(const GatherTable &t, int variant, const P *fp, int64_t n_pixels, int nf,
                   double *partial, cudaStream_t s, const uint8_t *masks = nullptr,
                   int64_t mask_stride = 0, double *oi = nullptr, double *os = nullptr,
                   double *od = nullptr) {
    if constexpr (MODE == kRaw) {
        if ((variant >= 5 && variant <= 8) || variant == 10) variant = 2;  // entry-lane mappings only
    } else {
        if (variant == 10) {
            if (oi && t.rw_n_items > 0) {
                launch_rows<MODE, P>(t, fp, n_pixels, nf, oi, os, od, s);
                return true;
            }
            variant = 2;
        }
        if (variant == 7 || variant == 8) {
            const BinTiles &bt = t.bt[variant - 7];
            if (oi && bt.n_items > 0) {
                if (variant == 7) launch_bins<MODE, P, Bt7>(t, bt, fp, n_pixels, nf, oi, os, od, s);
                else launch_bins<MODE, P, Bt8>(t, bt, fp, n_pixels, nf, oi, os, od, s);
                DG_CUDA(cudaGetLastError());
                return true;
            }
            variant = t.fl_n_units > 0 ? 5 : 2;
        }
        if (variant == 5 || variant == 6) {
            if (variant == 5) launch_fl<MODE, P, 4, false>(t, fp, n_pixels, nf, partial, s);
            else launch_fl<MODE, P, 4, true>(t, fp, n_pixels, nf, partial, s);
            DG_CUDA(cudaGetLastError());
            return false;
        }
    }
    const size_t smem = size_t(t.unit_cap) * (MODE == kSpread || MODE == kRaw ? 16 : 8);
    const float4 *wide = MODE == kRaw ? t.entry_raw.ptr : t.entry_std.ptr;
#define DG_GATHER_ARGS                                                                        \
    t.unit.ptr, t.seg.ptr, t.entry.ptr, wide, t.entry_nlo.ptr, t.first_valid.ptr, t.origin.ptr, fp, \
        n_pixels, nf, t.n_segments, partial, masks, mask_stride
    switch (variant) {
    case 0: k_gather<MODE, P, 32, 4, 4><<<t.n_units, kThreads, smem, s>>>(DG_GATHER_ARGS); break;
    case 1: k_gather<MODE, P, 32, 2, 8><<<t.n_units, kThreads, smem, s>>>(DG_GATHER_ARGS); break;
    case 2: k_gather<MODE, P, 8, 2, 4><<<t.n_units, kThreads, smem, s>>>(DG_GATHER_ARGS); break;
    case 3: k_gather<MODE, P, 4, 1, 8><<<t.n_units, kThreads, smem, s>>>(DG_GATHER_ARGS); break;
    case 9: k_gather<MODE, P, 32, 1, 8><<<t.n_units, kThreads, smem, s>>>(DG_GATHER_ARGS); break;
    default: k_gather<MODE, P, 16, 4, 2><<<t.n_units, kThreads, smem, s>>>(DG_GATHER_ARGS); break;
    }
#undef DG_GATHER_ARGS
    DG_CUDA(cudaGetLastError());
    return false;
}

template <typename P>
bool launch_typed(const GatherTable &t, int variant, const void *frames, int64_t n_pixels,
                  int n_frames, int mode, double *partial, double *oi, double *os, double *od,
                  cudaStream_t s) {
    const P *fp = static_cast<const P *>(frames);
    if (mode == kSpread)
        return launch_gather<kSpread, P>(t, variant, fp, n_pixels, n_frames, partial, s, nullptr,
                                         0, oi, os, od);
    if (mode == kErrors)
        return launch_gather<kErrors, P>(t, variant, fp, n_pixels, n_frames, partial, s, nullptr,
                                         0, oi, os, od);
    return launch_gather<kIntensity, P>(t, variant, fp, n_pixels, n_frames, partial, s, nullptr,
                                        0, oi, os, od);
}

template <int MODE, typename P>
void launch_finalize(const GatherTable &t, const double *partial, int nf, double *oi, double *os,
                     double *od, cudaStream_t s) {
    const dim3 grid(unsigned((t.n_rows + kFinRows - 1) / kFinRows), unsigned((nf + 31) / 32));
    k_finalize<MODE, P><<<grid, 32 * kFinRows, 0, s>>>(partial, t.row_seg.ptr, t.seg_ids.ptr,
                                                        t.den.ptr, t.den_std.ptr, t.valid_std.ptr,
                                                        t.n_rows, nf, oi, os, od);
    DG_CUDA(cudaGetLastError());
}

template <typename P>
void finalize_typed(const GatherTable &t, int mode, const double *partial, int nf, double *oi,
                    double *os, double *od, cudaStream_t s) {
    if (mode == kSpread) launch_finalize<kSpread, P>(t, partial, nf, oi, os, od, s);
    else if (mode == kErrors) launch_finalize<kErrors, P>(t, partial, nf, oi, os, od, s);
    else launch_finalize<kIntensity, P>(t, partial, nf, oi, os, od, s);
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

// Frame-lane units (k_gather_fl): runs of at most kFlSegs segments and
// kFlECap entries of one strip, split in halves by entries until each holds
// at most kFlDCap distinct pixels; then their pixel lists and entry pairs.
template <class Group>
void build_fl_units(GatherTable &out, const DeviceCsr &table, const std::vector<int4> &segs,
                    Group &&group, cudaStream_t s) {
    out.fl_n_units = 0;
    out.fl_pair_as = nullptr;
    if (segs.empty() || table.nnz > INT32_MAX) return;
    std::vector<int4> fl;
    group(kFlECap, kFlSegs, fl);
    DeviceArray<int4> d_units;
    DeviceArray<int32_t> d_count;
    std::vector<int32_t> count;
    auto seg_len = [&](int i) { return segs[size_t(i)].z - segs[size_t(i)].y; };
    for (int pass = 0;; ++pass) {
        d_units.alloc(fl.size());
        d_count.alloc(fl.size());
        DG_CUDA(cudaMemcpyAsync(d_units.ptr, fl.data(), fl.size() * sizeof(int4),
                                cudaMemcpyHostToDevice, s));
        k_fl_units<<<unsigned(fl.size()), 256, 0, s>>>(
            d_units.ptr, out.seg.ptr, table.col.ptr, out.origin.ptr, 0, d_count.ptr, nullptr,
            nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
        DG_CUDA(cudaGetLastError());
        count.resize(fl.size());
        DG_CUDA(cudaMemcpyAsync(count.data(), d_count.ptr, count.size() * 4,
                                cudaMemcpyDeviceToHost, s));
        DG_CUDA(cudaStreamSynchronize(s));
        std::vector<int4> next;
        bool split = false;
        for (size_t u = 0; u < fl.size(); ++u) {
            const int4 un = fl[u];
            if (count[u] <= kFlDCap || un.y < 2) {
                next.push_back(make_int4(un.x, un.y, 0, count[u]));
                continue;
            }
            // Split where the first part's entries reach half the unit's.
            int total = 0;
            for (int i = 0; i < un.y; ++i) total += seg_len(un.x + i);
            int acc = 0, cut = 1;
            for (int i = 0; i < un.y - 1; ++i) {
                acc += seg_len(un.x + i);
                cut = i + 1;
                if (2 * acc >= total) break;
            }
            next.push_back(make_int4(un.x, cut, 0, 0));
            next.push_back(make_int4(un.x + cut, un.y - cut, 0, 0));
            split = true;
        }
        fl.swap(next);
        if (!split) break;
        if (pass > 8) fail(DG_DEVICE, "frame-lane units did not converge");
    }
    int64_t pairs = 0;
    for (auto &un : fl) {
        if (un.w > kFlDCap) fail(DG_DEVICE, "frame-lane unit exceeds its pixel cap");
        un.z = int(pairs);
        for (int i = 0; i < un.y; ++i) pairs += (seg_len(un.x + i) + 1) / 2;
    }
    // The spread needs its own weights only if it excludes some entry.
    std::vector<int32_t> valid(size_t(out.n_rows));
    if (!valid.empty())
        DG_CUDA(cudaMemcpyAsync(valid.data(), out.valid_std.ptr, valid.size() * 4,
                                cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    int64_t n_valid = 0;
    for (int32_t v : valid) n_valid += v;
    const bool own_spread = n_valid != table.nnz;
    out.fl_unit.alloc(fl.size());
    out.fl_px.alloc(fl.size() * size_t(kFlDCap));
    out.fl_pair_a.alloc(size_t(std::max<int64_t>(pairs, 1)));
    out.fl_pair_b.alloc(size_t(std::max<int64_t>(pairs, 1)));
    out.fl_pair_c.alloc(size_t(std::max<int64_t>(pairs, 1)));
    if (own_spread) out.fl_pair_s.alloc(size_t(std::max<int64_t>(pairs, 1)));
    else out.fl_pair_s.release();
    DG_CUDA(cudaMemcpyAsync(out.fl_unit.ptr, fl.data(), fl.size() * sizeof(int4),
                            cudaMemcpyHostToDevice, s));
    out.fl_seg_org.alloc(segs.size());
    k_fl_units<<<unsigned(fl.size()), 256, 0, s>>>(
        out.fl_unit.ptr, out.seg.ptr, table.col.ptr, out.origin.ptr, 1, d_count.ptr,
        out.fl_px.ptr, out.entry.ptr, out.entry_std.ptr, out.entry_nlo.ptr, out.fl_pair_a.ptr,
        out.fl_pair_b.ptr, out.fl_pair_c.ptr, own_spread ? out.fl_pair_s.ptr : nullptr,
        out.fl_seg_org.ptr);
    DG_CUDA(cudaGetLastError());
    DG_CUDA(cudaStreamSynchronize(s));
    out.fl_pair_as = own_spread ? out.fl_pair_s.ptr : out.fl_pair_a.ptr;
    out.fl_n_units = int32_t(fl.size());
}

// Bin tiles (k_gather_bins) at plan time, on the host: for every run of
// CFG::kRows rows, the rows' entries merged in pixel order and cut into chunks of
// at most kBtDCap distinct pixels and kBtPCap pairs (a new pixel that would
// exceed either opens the next chunk, so a chunk is a pixel-index interval
// and each row's entries in it are a contiguous run of its CSR row). Tiles
// are ordered largest first. Each row keeps {origin entry, first valid entry,
// row end} for the spread's origin (row_origin), read before the first chunk.
template <class CFG>
void build_bin_tiles(GatherTable &gt, BinTiles &out, const DeviceCsr &table, cudaStream_t s) {
    constexpr int kBtDCap = CFG::kDCap, kBtPCap = CFG::kPCap, kBtRows = CFG::kRows;
    constexpr int kBtMetaHead = CFG::kMetaHead, kBtMetaWords = CFG::kMetaWords;
    const int64_t nb = table.n_rows;
    out.n_items = 0;
    if (nb == 0 || table.nnz == 0) return;
    out.wait_err.alloc();
    std::vector<int64_t> rp(static_cast<size_t>(nb) + 1);
    DG_CUDA(cudaMemcpyAsync(rp.data(), table.row_ptr.ptr, rp.size() * 8, cudaMemcpyDeviceToHost, s));
    std::vector<int32_t> col(static_cast<size_t>(table.nnz)), fv(static_cast<size_t>(nb)),
        oe(static_cast<size_t>(nb));
    DG_CUDA(cudaMemcpyAsync(col.data(), table.col.ptr, col.size() * 4, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaMemcpyAsync(fv.data(), gt.first_valid.ptr, fv.size() * 4, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaMemcpyAsync(oe.data(), gt.origin.ptr, oe.size() * 4, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    const int64_t n_items = (nb + kBtRows - 1) / kBtRows;
    struct Tile {
        std::vector<int4> chunks;      // {px offset, D, pair offset, pairs} (tile-relative)
        std::vector<int32_t> cpair;    // per chunk kBtRows + 1
        std::vector<int32_t> px;
        std::vector<int4> pairs;       // {slot0, slot1, entry0, entry1}
        int64_t entries = 0;
    };
    std::vector<Tile> tiles(static_cast<size_t>(n_items));
    auto build = [&](int64_t ti) {
        Tile &T = tiles[size_t(ti)];
        const int64_t r0 = ti * kBtRows, r1 = std::min<int64_t>(nb, r0 + kBtRows);
        const int nr = int(r1 - r0);
        // Entries merged in pixel order, rows ascending within a pixel: keys
        // pixel << 32 | row << 27 | position in row; each row is sorted
        // already, so four rounds of pairwise merges order the tile.
        const int64_t n_e = rp[size_t(r1)] - rp[size_t(r0)];
        std::vector<uint64_t> ka(static_cast<size_t>(n_e)), kb(static_cast<size_t>(n_e));
        std::vector<int64_t> bounds(static_cast<size_t>(kBtRows) + 1, 0);
        for (int j = 0; j < nr; ++j) {
            const int64_t b = rp[size_t(r0 + j)], e = rp[size_t(r0 + j) + 1];
            if (e - b >= (int64_t(1) << 27)) fail(DG_UNSUPPORTED, "a bin too large for bin tiles");
            uint64_t *o = ka.data() + (b - rp[size_t(r0)]);
            for (int64_t k = b; k < e; ++k)
                o[k - b] = (uint64_t(uint32_t(col[size_t(k)])) << 32) | (uint64_t(j) << 27) |
                           uint64_t(k - b);
            bounds[size_t(j) + 1] = e - rp[size_t(r0)];
        }
        for (int j = nr; j < kBtRows; ++j) bounds[size_t(j) + 1] = n_e;
        for (int width = 1; width < kBtRows; width *= 2) {
            for (int j = 0; j < kBtRows; j += 2 * width) {
                const int64_t a0 = bounds[size_t(j)], a1 = bounds[size_t(std::min(j + width, kBtRows))],
                              a2 = bounds[size_t(std::min(j + 2 * width, kBtRows))];
                std::merge(ka.begin() + a0, ka.begin() + a1, ka.begin() + a1, ka.begin() + a2,
                           kb.begin() + a0);
            }
            ka.swap(kb);
        }
        struct Ent {
            int32_t px, row, k;
        };
        std::vector<Ent> m(static_cast<size_t>(n_e));
        for (int64_t i = 0; i < n_e; ++i) {
            const uint64_t key = ka[size_t(i)];
            const int j = int((key >> 27) & 31u);
            m[size_t(i)] = {int32_t(key >> 32), j, int32_t(rp[size_t(r0 + j)] + int64_t(key & ((1u << 27) - 1)))};
        }
        T.entries = n_e;
        T.pairs.reserve(size_t(n_e / 2 + 64));
        T.px.reserve(size_t(n_e / 2 + 64));
        std::vector<std::vector<std::pair<int32_t, int32_t>>> run(static_cast<size_t>(nr));  // (slot, entry)
        std::vector<int32_t> chunk_px;
        auto close = [&]() {
            if (chunk_px.empty()) return;
            int4 ch = make_int4(int(T.px.size()), int(chunk_px.size()), int(T.pairs.size()), 0);
            T.px.insert(T.px.end(), chunk_px.begin(), chunk_px.end());
            int po = 0;
            for (int j = 0; j < kBtRows; ++j) {
                T.cpair.push_back(po);
                if (j >= nr) continue;
                const auto &rv = run[size_t(j)];
                for (size_t e = 0; e < rv.size(); e += 2) {
                    const bool two = e + 1 < rv.size();
                    T.pairs.push_back(make_int4(rv[e].first, two ? rv[e + 1].first : kBtDCap,
                                                rv[e].second, two ? rv[e + 1].second : -1));
                    ++po;
                }
            }
            T.cpair.push_back(po);
            ch.w = po;
            T.chunks.push_back(ch);
            chunk_px.clear();
            for (auto &rv : run) rv.clear();
        };
        int pairs = 0;
        for (size_t i = 0; i < m.size();) {
            size_t e = i;
            while (e < m.size() && m[e].px == m[i].px) ++e;
            // pairs after adding this pixel's entries
            int add = 0;
            for (size_t q = i; q < e; ++q) add += (run[size_t(m[q].row)].size() % 2 == 0) ? 1 : 0;
            if (!chunk_px.empty() &&
                (int(chunk_px.size()) + 1 > kBtDCap || pairs + add > kBtPCap)) {
                close();
                pairs = 0;
                add = int(e - i);
            }
            const int slot = int(chunk_px.size());
            chunk_px.push_back(m[i].px);
            for (size_t q = i; q < e; ++q) run[size_t(m[q].row)].push_back({slot, m[q].k});
            pairs += add;
            i = e;
        }
        close();
    };
    const int nt = int(std::min<int64_t>(
        n_items, std::max(1u, std::min(16u, std::thread::hardware_concurrency()))));
    auto parallel = [&](auto &&fn, int64_t count) {
        std::vector<std::thread> pool;
        std::atomic<int64_t> next{0};
        for (int t = 0; t < nt; ++t)
            pool.emplace_back([&]() {
                for (int64_t i; (i = next.fetch_add(1)) < count;) fn(i);
            });
        for (auto &th : pool) th.join();
    };
    parallel(build, n_items);
    // Tile order, then flatten.
    std::vector<int64_t> order(static_cast<size_t>(n_items));
    for (int64_t i = 0; i < n_items; ++i) order[size_t(i)] = i;
#if DG_BT_LARGEST_FIRST
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
        return tiles[size_t(a)].entries > tiles[size_t(b)].entries;
    });
#endif
    // Mapping 8: neighbouring tiles 2m, 2m + 1 side by side (pairs largest
    // first), launched as 2-CTA clusters so both run on one GPC and read the
    // pixel runs they share through the same L2; -1 marks the empty partner
    // of an odd last tile.
    out.paired = false;
    if (kBtClusterPairs && std::is_same<CFG, Bt8>::value && n_items > 1) {
        const int64_t np = (n_items + 1) / 2;
        std::vector<int64_t> pairs_order(static_cast<size_t>(np));
        auto pair_size = [&](int64_t m) {
            int64_t e = tiles[size_t(2 * m)].entries;
            if (2 * m + 1 < n_items) e = std::max<int64_t>(e, tiles[size_t(2 * m + 1)].entries);
            return e;
        };
        for (int64_t m = 0; m < np; ++m) pairs_order[size_t(m)] = m;
        std::stable_sort(pairs_order.begin(), pairs_order.end(),
                         [&](int64_t a, int64_t b) { return pair_size(a) > pair_size(b); });
        order.clear();
        for (int64_t m : pairs_order) {
            order.push_back(2 * m);
            order.push_back(2 * m + 1 < n_items ? 2 * m + 1 : -1);
        }
        out.paired = true;
    }
    const int64_t n_slots = int64_t(order.size());
    // Output offsets of every tile, then the tiles copied in parallel.
    std::vector<int64_t> o_ch(size_t(n_slots) + 1, 0), o_px(size_t(n_slots) + 1, 0),
        o_pr(size_t(n_slots) + 1, 0);
    const Tile empty_tile;
    auto tile_at = [&](int64_t i) -> const Tile & {
        return order[size_t(i)] < 0 ? empty_tile : tiles[size_t(order[size_t(i)])];
    };
    for (int64_t i = 0; i < n_slots; ++i) {
        const Tile &T = tile_at(i);
        o_ch[size_t(i) + 1] = o_ch[size_t(i)] + int64_t(T.chunks.size());
        o_px[size_t(i) + 1] = o_px[size_t(i)] + int64_t(T.px.size());
        o_pr[size_t(i) + 1] = o_pr[size_t(i)] + int64_t(T.pairs.size());
    }
    if (o_pr[size_t(n_slots)] > INT32_MAX || o_px[size_t(n_slots)] > INT32_MAX)
        fail(DG_UNSUPPORTED, "table too large for bin tiles");
    // default-initialised (not zeroed): every element is written below
    const size_t n_chunks = size_t(o_ch[size_t(n_slots)]), n_pairs = size_t(o_pr[size_t(n_slots)]);
    std::vector<int4> items(static_cast<size_t>(n_slots)), org(static_cast<size_t>(nb));
    // per row {origin entry, first valid entry, row end, 0} (row_origin)
    for (int64_t r = 0; r < nb; ++r)
        org[size_t(r)] = make_int4(oe[size_t(r)], fv[size_t(r)], int(rp[size_t(r) + 1]), 0);
    std::unique_ptr<int32_t[]> meta(new int32_t[std::max<size_t>(n_chunks * kBtMetaWords, 1)]);
    std::unique_ptr<int4[]> pairs(new int4[std::max<size_t>(n_pairs, 1)]);
    auto flatten = [&](int64_t i) {
        const int64_t ti = order[size_t(i)];
        if (ti < 0) {  // the empty partner: no rows, no chunks
            items[size_t(i)] = make_int4(0, 0, int(o_ch[size_t(i)]), 0);
            return;
        }
        Tile &T = tiles[size_t(ti)];
        const int64_t c0 = o_ch[size_t(i)], pr0 = o_pr[size_t(i)];
        for (size_t c = 0; c < T.chunks.size(); ++c) {
            const int4 ch = T.chunks[c];
            int32_t *rec = meta.get() + (size_t(c0) + c) * kBtMetaWords;
            rec[0] = ch.y;
            rec[1] = ch.w;
            rec[2] = int32_t(ch.z + pr0);
            rec[3] = 0;
            for (int j = 0; j < kBtMetaHead - 4; ++j)
                rec[4 + j] = j <= kBtRows ? T.cpair[c * (kBtRows + 1) + size_t(j)] : 0;
            std::copy(T.px.begin() + ch.x, T.px.begin() + ch.x + ch.y, rec + kBtMetaHead);
            std::fill(rec + kBtMetaHead + ch.y, rec + kBtMetaWords, 0);
        }
        std::copy(T.pairs.begin(), T.pairs.end(), pairs.get() + pr0);
        const int64_t r0 = ti * kBtRows;
        const int nr = int(std::min<int64_t>(nb, r0 + kBtRows) - r0);
        items[size_t(i)] = make_int4(int(r0), nr, int(c0), int(T.chunks.size()));
        T = Tile();
    };
    parallel(flatten, n_slots);
    out.n_items = int32_t(items.size());
    out.item.alloc(items.size());
    out.meta.alloc(std::max<size_t>(n_chunks * kBtMetaWords, 1));
    out.org.alloc(org.size());
    out.pair_a.alloc(std::max<size_t>(n_pairs, 1));
    out.pair_as.alloc(std::max<size_t>(n_pairs, 1));
    out.pair_b.alloc(std::max<size_t>(n_pairs, 1));
    out.pair_c.alloc(std::max<size_t>(n_pairs, 1));
    DeviceArray<int4> &desc = out.desc;  // kept for the per-frame-mask pairs
    desc.alloc(std::max<size_t>(n_pairs, 1));
    out.pair_ra.release();
    out.pair_rb.release();
    out.raw_built = false;
    DG_CUDA(cudaMemcpyAsync(out.item.ptr, items.data(), items.size() * sizeof(int4),
                            cudaMemcpyHostToDevice, s));
    if (n_chunks)
        DG_CUDA(cudaMemcpyAsync(out.meta.ptr, meta.get(), n_chunks * kBtMetaWords * 4,
                                cudaMemcpyHostToDevice, s));
    DG_CUDA(cudaMemcpyAsync(out.org.ptr, org.data(), org.size() * sizeof(int4),
                            cudaMemcpyHostToDevice, s));
    if (n_pairs) {
        DG_CUDA(cudaMemcpyAsync(desc.ptr, pairs.get(), n_pairs * sizeof(int4),
                                cudaMemcpyHostToDevice, s));
        k_bt_fill<<<148 * 8, 256, 0, s>>>(desc.ptr, int64_t(n_pairs), gt.entry.ptr,
                                         gt.entry_std.ptr, gt.entry_nlo.ptr, out.pair_a.ptr,
                                         out.pair_as.ptr, out.pair_b.ptr, out.pair_c.ptr);
        DG_CUDA(cudaGetLastError());
    }
    DG_CUDA(cudaStreamSynchronize(s));
    // Only mapping 8's tiles carry per-frame masks (BtR); the others drop the
    // descriptor once their pairs are filled.
    if (!std::is_same<CFG, Bt8>::value) desc.release();
}

namespace {
__global__ void k_flip_meta(int32_t *__restrict__ meta, int64_t n_rec, int words, int head,
                            int rows, int cols);
}  // namespace

bool bin_tile_wait_failed(const GatherTable &t) {
    bool failed = false;
    for (const BinTiles &bt : t.bt)
        if (bt.wait_err.host && *static_cast<volatile int *>(bt.wait_err.host)) {
            *bt.wait_err.host = 0;
            failed = true;
        }
    return failed;
}

void check_bin_tile_waits(const GatherTable &t) {
    if (bin_tile_wait_failed(t))
        fail(DG_TIMEOUT, "bin-tile gather: a chunk-pipeline wait gave up after 1 s; the "
                          "results of a launch on this plan since the last check are invalid");
}

void ensure_bin_tiles(GatherTable &t, const DeviceCsr &table, int variant, cudaStream_t s) {
    if (variant != 7 && variant != 8) return;
    BinTiles &bt = t.bt[variant - 7];
    if (bt.built) return;
    int words = 0, head = 0;
    if (variant == 7) {
        build_bin_tiles<Bt7>(t, bt, table, s);
        words = Bt7::kMetaWords;
        head = Bt7::kMetaHead;
    } else {
        build_bin_tiles<Bt8>(t, bt, table, s);
        words = Bt8::kMetaWords;
        head = Bt8::kMetaHead;
    }
    if (t.flip_rows && bt.n_items > 0) {
        k_flip_meta<<<148 * 4, 256, 0, s>>>(bt.meta.ptr, int64_t(bt.meta.count) / words, words,
                                            head, t.flip_rows, t.flip_cols);
        DG_CUDA(cudaGetLastError());
        DG_CUDA(cudaStreamSynchronize(s));
    }
    bt.built = true;
}

bool gather_variant_needs_tiles(int variant) { return variant == 7 || variant == 8; }

bool bin_tiles_fill_gpu(const GatherTable &t, int variant, int64_t n_frames) {
    if (!gather_variant_needs_tiles(variant)) return false;
    const int64_t rows = variant == 7 ? Bt7::kRows : Bt8::kRows;
    const int64_t per = variant == 7 ? Bt7::kFrames : Bt8::kFrames;
    const int64_t nf = std::min<int64_t>(n_frames, 256);
    const int64_t ctas = (int64_t(t.n_rows) + rows - 1) / rows * ((nf + per - 1) / per);
    return 2 * nf >= per && ctas >= 2 * 148;
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
    out.entry_nlo.alloc(size_t(table.nnz));
    out.valid_std.alloc(size_t(table.n_rows));
    out.first_valid.alloc(size_t(table.n_rows));
    out.origin.alloc(size_t(table.n_rows));
    denominators(table, d_norm, s, out.den.ptr);
    const int64_t n_px = int64_t(dim1) * dim2;
    out.px_norm.alloc(size_t(std::max<int64_t>(n_px, 1)));
    if (n_px > 0)
        k_px_norm<<<unsigned(std::min<int64_t>((n_px + 255) / 256, 148 * 16)), 256, 0, s>>>(
            d_norm, n_px, 0, 0, out.px_norm.ptr);
    const unsigned rb = unsigned((table.n_rows + 127) / 128);
    if (table.n_rows > 0)
        k_pack<<<rb, 128, 0, s>>>(table.row_ptr.ptr, int(table.n_rows), table.col.ptr, table.w.ptr,
                                  d_norm, out.entry.ptr, out.entry_std.ptr, out.entry_nlo.ptr,
                                  out.den_std.ptr, out.valid_std.ptr, out.first_valid.ptr,
                                  out.origin.ptr);
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
    std::vector<int32_t> strip_first(size_t(n_strips) + 1, 0);
    for (int st = 0; st < n_strips; ++st) {
        strip_first[size_t(st)] = int32_t(segs.size());
        for (int64_t r = 0; r < nb; ++r) {
            const int32_t *b = hb.data() + r * (n_strips + 1);
            for (int32_t lo = b[st]; lo < b[st + 1]; lo += kSegMax) {
                int32_t hi = std::min<int32_t>(lo + kSegMax, b[st + 1]);
                segs.push_back(make_int4(int(r), lo, hi, int(rp[size_t(r) + 1])));
                seg_count[size_t(r)]++;
            }
        }
    }
    strip_first[size_t(n_strips)] = int32_t(segs.size());
    // Units: runs of consecutive segments of one strip, at most max_segs
    // segments and `cap` entries each.
    auto group = [&](int cap, int max_segs, auto &&emit) {
        for (int st = 0; st < n_strips; ++st) {
            int first = strip_first[size_t(st)], entries = 0;
            for (int i = first; i < strip_first[size_t(st) + 1]; ++i) {
                const int len = segs[size_t(i)].z - segs[size_t(i)].y;
                if (i - first == max_segs || entries + len > cap) {
                    emit(first, i - first);
                    first = i;
                    entries = 0;
                }
                entries += len;
            }
            if (strip_first[size_t(st) + 1] > first) emit(first, strip_first[size_t(st) + 1] - first);
        }
    };
    group(kUnitCap, kWarps, [&](int first, int n) { units.push_back(make_int2(first, n)); });
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
    // Row warps (mapping 10): long rows one per CTA, longest first; the
    // others eight per CTA in row order.
    std::vector<int32_t> rw_ptr, rw_rows;
    std::vector<int4> rw_items;
    if (table.nnz <= INT32_MAX && nb > 0) {
        rw_ptr.assign(rp.begin(), rp.end());
        for (int64_t r = 0; r < nb; ++r)
            if (rp[size_t(r) + 1] - rp[size_t(r)] > kRowsLong) rw_rows.push_back(int32_t(r));
        std::stable_sort(rw_rows.begin(), rw_rows.end(), [&](int32_t a, int32_t b) {
            return rp[size_t(a) + 1] - rp[size_t(a)] > rp[size_t(b) + 1] - rp[size_t(b)];
        });
        for (size_t i = 0; i < rw_rows.size(); ++i) {  // long rows carry their range
            const int32_t r = rw_rows[i];
            rw_items.push_back(make_int4(r, 0, int(rp[size_t(r)]), int(rp[size_t(r) + 1])));
        }
        auto len = [&](int64_t r) { return rp[size_t(r) + 1] - rp[size_t(r)]; };
        const size_t first_mid = rw_rows.size();
        for (int64_t r = 0; r < nb; ++r)
            if (len(r) <= kRowsLong && len(r) > kRowsTiny) rw_rows.push_back(int32_t(r));
        for (size_t i = first_mid; i < rw_rows.size(); i += kRowsWarps)
            rw_items.push_back(make_int4(int(i), int(std::min<size_t>(kRowsWarps,
                                                                      rw_rows.size() - i)), 0, 0));
        const size_t first_tiny = rw_rows.size();
        for (int64_t r = 0; r < nb; ++r)
            if (len(r) <= kRowsTiny) rw_rows.push_back(int32_t(r));
        for (size_t i = first_tiny; i < rw_rows.size(); i += 4 * kRowsWarps)
            rw_items.push_back(make_int4(int(i), -int(std::min<size_t>(4 * kRowsWarps,
                                                                       rw_rows.size() - i)), 0, 0));
        out.rw_row_ptr.alloc(rw_ptr.size());
        out.rw_rows.alloc(rw_rows.size());
        out.rw_item.alloc(rw_items.size());
        DG_CUDA(cudaMemcpyAsync(out.rw_row_ptr.ptr, rw_ptr.data(), rw_ptr.size() * 4,
                                cudaMemcpyHostToDevice, s));
        DG_CUDA(cudaMemcpyAsync(out.rw_rows.ptr, rw_rows.data(), rw_rows.size() * 4,
                                cudaMemcpyHostToDevice, s));
        DG_CUDA(cudaMemcpyAsync(out.rw_item.ptr, rw_items.data(), rw_items.size() * sizeof(int4),
                                cudaMemcpyHostToDevice, s));
        out.rw_n_items = int32_t(rw_items.size());
    }
    DG_CUDA(cudaStreamSynchronize(s));
    build_fl_units(out, table, segs, [&](int cap, int max_segs, std::vector<int4> &fl) {
        group(cap, max_segs, [&](int first, int n) { fl.push_back(make_int4(first, n, 0, 0)); });
    }, s);
}

bool gather_writes_results(const GatherTable &t) {
    if (t.variant == 10) return t.rw_n_items > 0;
    return (t.variant == 7 || t.variant == 8) && t.bt[t.variant - 7].n_items > 0;
}

void reserve_partials(GatherTable &t, int64_t n_frames, uint32_t flags, int dtype,
                      bool any_mapping) {
    if ((!any_mapping && gather_writes_results(t)) || n_frames <= 0) return;
    const int mode = (flags & DG_AZIMUTHAL_STD) ? kSpread : (flags & DG_ERRORS) ? kErrors
                                                                                : kIntensity;
    const int64_t need = std::max<int64_t>(1, t.n_segments) *
                         n_accumulators(mode, dtype == DG_F32 || dtype == DG_F64) *
                         std::min<int64_t>(256, (n_frames + 31) / 32 * 32);
    if (t.partial.count < size_t(need)) t.partial.alloc(size_t(need));
}

QueuePlan queue_plan(const GatherTable &t, const void *d_frames, int64_t n_pixels, int n_frames,
                     double *oi, double *os, double *od) {
    QueuePlan q{};
    q.item = t.rw_item.ptr;
    q.rows = t.rw_rows.ptr;
    q.row_ptr = t.rw_row_ptr.ptr;
    q.entry = t.entry.ptr;
    q.entry_std = t.entry_std.ptr;
    q.entry_nlo = t.entry_nlo.ptr;
    q.px_norm = t.px_norm.ptr;
    q.first_valid = t.first_valid.ptr;
    q.origin = t.origin.ptr;
    q.den = t.den.ptr;
    q.den_std = t.den_std.ptr;
    q.valid_std = t.valid_std.ptr;
    q.frames = d_frames;
    q.out_i = oi;
    q.out_s = os;
    q.out_d = od;
    q.n_pixels = n_pixels;
    q.n_frames = n_frames;
    q.n_rows = t.n_rows;
    q.n_items = n_frames > 0 ? t.rw_n_items : 0;
    q.frame_blocks = std::max(1, (n_frames + rows_pass_frames(n_frames) - 1) /
                                     rows_pass_frames(n_frames));
    return q;
}

namespace {

// Resident capacity of the work-queue gather: the CTAs the SMs hold at
// once, the grid of a call of more than kQueueDirectTiles tiles, whose CTAs
// stay resident and claim tiles until the queue is empty. Smaller calls run
// one CTA per tile (queue_grid).
template <int MODE, typename P>
int queue_capacity() {
    static int cap = 0;
    if (cap == 0) {
        int per_sm = 0, dev = 0, sms = 0;
        DG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rows_queue<MODE, P>,
                                                              kRowsThreads, 0));
        DG_CUDA(cudaGetDevice(&dev));
        DG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        cap = std::max(1, per_sm) * std::max(1, sms);
    }
    return cap;
}

template <int MODE, typename P>
void queue_launch_typed(QueueHeader *hdr, const QueuePlan *plans, cudaStream_t s) {
    k_rows_queue<MODE, P><<<queue_capacity<MODE, P>(), kRowsThreads, 0, s>>>(hdr, plans);
    DG_CUDA(cudaGetLastError());
}

template <typename P>
int queue_capacity_mode(int mode) {
    if (mode == kSpread) return queue_capacity<kSpread, P>();
    if (mode == kErrors) return queue_capacity<kErrors, P>();
    return queue_capacity<kIntensity, P>();
}

template <typename P>
void queue_launch_mode(int mode, QueueHeader *hdr, const QueuePlan *plans, cudaStream_t s) {
    if (mode == kSpread) queue_launch_typed<kSpread, P>(hdr, plans, s);
    else if (mode == kErrors) queue_launch_typed<kErrors, P>(hdr, plans, s);
    else queue_launch_typed<kIntensity, P>(hdr, plans, s);
}

}  // namespace

int queue_grid(int dtype, uint32_t flags, int64_t total_tiles, bool resident) {
    // one CTA per tile (the hardware schedules them as CTAs retire, beside
    // other streams' kernels); a batch of more tiles than kQueueDirectTiles
    // runs the resident grid that claims them
    if (!resident && total_tiles <= kQueueDirectTiles)
        return int(std::max<int64_t>(1, total_tiles));
    const int mode = (flags & DG_AZIMUTHAL_STD) ? kSpread : (flags & DG_ERRORS) ? kErrors
                                                                                : kIntensity;
    int cap = 1;
    switch (dtype) {
    case DG_U16: cap = queue_capacity_mode<uint16_t>(mode); break;
    case DG_U32: cap = queue_capacity_mode<uint32_t>(mode); break;
    case DG_I32: cap = queue_capacity_mode<int32_t>(mode); break;
    case DG_F32: cap = queue_capacity_mode<float>(mode); break;
    case DG_F64: cap = queue_capacity_mode<double>(mode); break;
    default: fail(DG_INVALID_INPUT, "unknown pixel dtype");
    }
    const int64_t claims = (total_tiles + kQueueClaim - 1) / kQueueClaim;
    return int(std::max<int64_t>(1, std::min<int64_t>(claims, cap)));
}

void queue_launch(int dtype, uint32_t flags, QueueHeader *hdr, const QueuePlan *plans,
                  cudaStream_t s) {
    const int mode = (flags & DG_AZIMUTHAL_STD) ? kSpread : (flags & DG_ERRORS) ? kErrors
                                                                                : kIntensity;
    switch (dtype) {
    case DG_U16: queue_launch_mode<uint16_t>(mode, hdr, plans, s); break;
    case DG_U32: queue_launch_mode<uint32_t>(mode, hdr, plans, s); break;
    case DG_I32: queue_launch_mode<int32_t>(mode, hdr, plans, s); break;
    case DG_F32: queue_launch_mode<float>(mode, hdr, plans, s); break;
    case DG_F64: queue_launch_mode<double>(mode, hdr, plans, s); break;
    default: fail(DG_INVALID_INPUT, "unknown pixel dtype");
    }
}

void run_gather(GatherTable &t, const void *d_frames, int dtype, int64_t n_pixels,
                int64_t n_frames, uint32_t flags, int precision, double *d_i, double *d_sigma,
                double *d_std, cudaStream_t s, double *scratch, size_t scratch_doubles) {
    (void)precision;
    if (n_frames <= 0) return;
    if (dtype < DG_U16 || dtype > DG_F64) fail(DG_INVALID_INPUT, "unknown pixel dtype");
    const int mode = (flags & DG_AZIMUTHAL_STD) ? kSpread : (flags & DG_ERRORS) ? kErrors
                                                                                : kIntensity;
    // Frames per launch: 256, or fewer where the caller's fixed scratch holds
    // the partial sums of fewer frames (the bin tiles write no partial sums).
    int64_t chunk = 256;
    double *partial = nullptr;
    if (scratch) {
        const bool fpx = dtype == DG_F32 || dtype == DG_F64;
        const int64_t per_frame =
            gather_writes_results(t) || t.n_units == 0
                ? 0
                : std::max<int64_t>(1, t.n_segments) * n_accumulators(mode, fpx);
        if (per_frame > 0) chunk = std::min<int64_t>(chunk, int64_t(scratch_doubles) / per_frame);
        if (chunk < 1)
            fail(DG_UNSUPPORTED, "this plan needs " + std::to_string(per_frame * 8) +
                                     " bytes of partial sums per frame; the fixed scratch holds " +
                                     std::to_string(scratch_doubles * 8) + " bytes");
        partial = scratch;
    } else {
        // [segment][accumulator][frame] for the largest launch of this call,
        // frames rounded up to 32 so that growing batches reallocate rarely
        reserve_partials(t, std::min<int64_t>(chunk, n_frames), flags, dtype, true);
        t.scratch.wait(s);
        partial = t.partial.ptr;
    }
    const size_t esize = dtype == DG_U16 ? 2 : dtype == DG_F64 ? 8 : 4;
    for (int64_t f0 = 0; f0 < n_frames; f0 += chunk) {
        const int nf = int(std::min<int64_t>(chunk, n_frames - f0));
        const void *fp = static_cast<const unsigned char *>(d_frames) + f0 * n_pixels * esize;
        double *oi = d_i + f0 * t.n_rows;
        double *os = d_sigma ? d_sigma + f0 * t.n_rows : nullptr;
        double *od = d_std ? d_std + f0 * t.n_rows : nullptr;
        bool done = false;  // results written by the gather itself (bin tiles)
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
            case DG_U16: done = launch_typed<uint16_t>(t, t.variant, fp, n_pixels, nf, mode, partial, oi, os, od, s); break;
            case DG_U32: done = launch_typed<uint32_t>(t, t.variant, fp, n_pixels, nf, mode, partial, oi, os, od, s); break;
            case DG_I32: done = launch_typed<int32_t>(t, t.variant, fp, n_pixels, nf, mode, partial, oi, os, od, s); break;
            case DG_F32: done = launch_typed<float>(t, t.variant, fp, n_pixels, nf, mode, partial, oi, os, od, s); break;
            case DG_F64: done = launch_typed<double>(t, t.variant, fp, n_pixels, nf, mode, partial, oi, os, od, s); break;
            }
            if (ev) DG_CUDA(cudaEventRecord(ev->second, s));
        }
        if (t.n_rows > 0 && !done) {
            ++t.launches;
            switch (dtype) {
            case DG_U16: finalize_typed<uint16_t>(t, mode, partial, nf, oi, os, od, s); break;
            case DG_U32: finalize_typed<uint32_t>(t, mode, partial, nf, oi, os, od, s); break;
            case DG_I32: finalize_typed<int32_t>(t, mode, partial, nf, oi, os, od, s); break;
            case DG_F32: finalize_typed<float>(t, mode, partial, nf, oi, os, od, s); break;
            case DG_F64: finalize_typed<double>(t, mode, partial, nf, oi, os, od, s); break;
            }
        }
    }
    if (!scratch) t.scratch.mark(s);
}

namespace {

// Swaps detector rows r and rows - 1 - r of a per-pixel array.
__global__ void k_flip_px_norm(float2 *__restrict__ a, int rows, int cols) {
    const int64_t half = int64_t(rows / 2) * cols;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < half;
         i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t r = i / cols, c = i - r * cols;
        const int64_t j = (rows - 1 - r) * cols + c;
        const float2 t = a[i];
        a[i] = a[j];
        a[j] = t;
    }
}

// Row flip of a pixel index for frames stored bottom row first.
__device__ __forceinline__ int32_t flip_px(int32_t j, int rows, int cols) {
    const int32_t r = j / cols, c = j - r * cols;
    return (rows - 1 - r) * cols + c;
}

// InputOrder::FlipVertical: every pixel index the gathers load through,
// remapped in place (entry order, and so every sum, unchanged). Pixel-list
// slots past a unit's pixel count hold no index and may hold anything; values
// outside the frame are left alone.
__global__ void k_flip_rows(int2 *__restrict__ entry, float4 *__restrict__ entry_std, int64_t nnz,
                            int32_t *__restrict__ px, int64_t n_px, int rows, int cols) {
    const int64_t npix = int64_t(rows) * cols;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nnz + n_px;
         i += int64_t(gridDim.x) * blockDim.x) {
        if (i < nnz) {
            entry[i].x = flip_px(entry[i].x, rows, cols);
            entry_std[i].x = __int_as_float(flip_px(__float_as_int(entry_std[i].x), rows, cols));
        } else {
            const int32_t v = px[i - nnz];
            if (v >= 0 && v < npix) px[i - nnz] = flip_px(v, rows, cols);
        }
    }
}

// The same for the pixel indices of bin-tile chunk records (D of them each).
__global__ void k_flip_meta(int32_t *__restrict__ meta, int64_t n_rec, int words, int head,
                            int rows, int cols) {
    for (int64_t r = blockIdx.x; r < n_rec; r += gridDim.x) {
        int32_t *rec = meta + r * words;
        const int d = rec[0];
        for (int k = threadIdx.x; k < d; k += blockDim.x)
            rec[head + k] = flip_px(rec[head + k], rows, cols);
    }
}

}  // namespace

void flip_gather_rows(GatherTable &t, int32_t dim1, int32_t dim2, cudaStream_t s) {
    t.flip_rows = dim1;
    t.flip_cols = dim2;
    // per-pixel norms to frame storage order: rows r and dim1 - 1 - r swapped
    const int64_t half = int64_t(dim1 / 2) * dim2;
    if (t.px_norm.ptr && half > 0)
        k_flip_px_norm<<<unsigned(std::min<int64_t>((half + 255) / 256, 148 * 16)), 256, 0, s>>>(
            t.px_norm.ptr, dim1, dim2);
    const int64_t n_px = t.fl_px.ptr ? int64_t(t.fl_px.count) : 0;
    if (t.nnz + n_px > 0)
        k_flip_rows<<<148 * 8, 256, 0, s>>>(t.entry.ptr, t.entry_std.ptr, t.nnz, t.fl_px.ptr,
                                            n_px, dim1, dim2);
    DG_CUDA(cudaGetLastError());
    // bin tiles are built later (ensure_bin_tiles) and flipped then
}

void prepare_raw(GatherTable &t, const DeviceCsr &table, const double *d_norm, cudaStream_t s) {
    if (t.cnt.ptr) return;
    t.entry_raw.alloc(std::max<size_t>(size_t(table.nnz), 1));
    t.cnt.alloc(std::max<size_t>(size_t(table.n_rows), 1));
    if (table.n_rows > 0)
        k_pack_raw<<<unsigned((table.n_rows + 127) / 128), 128, 0, s>>>(
            table.row_ptr.ptr, int(table.n_rows), table.col.ptr, table.w.ptr, d_norm,
            t.entry_raw.ptr, t.cnt.ptr, t.flip_rows, t.flip_cols);
    DG_CUDA(cudaGetLastError());
}

namespace {

template <typename P>
bool launch_raw(GatherTable &t, const void *frames, int64_t n_pixels, int nf, int mode,
                const uint8_t *masks, int64_t mask_stride, cudaStream_t s, bool raw, double *o0,
                double *o1, double *o2, double *o3) {
    const P *fp = static_cast<const P *>(frames);
    // Per-frame masks on a mapping-8 plan: the masked tiles write the raw
    // sums (S, N, V, C in o0..o3) or the normalised results (o0, o1).
    if (mode == kRaw && t.variant == 8 && t.bt[1].n_items > 0 && t.entry_raw.ptr) {
        BinTiles &bt = t.bt[1];
        if (!bt.raw_built) {
            bt.pair_ra.alloc(bt.desc.count);
            bt.pair_rb.alloc(bt.desc.count);
            k_bt_fill_raw<<<148 * 8, 256, 0, s>>>(bt.desc.ptr, int64_t(bt.desc.count),
                                                 t.entry_raw.ptr, bt.pair_ra.ptr, bt.pair_rb.ptr);
            DG_CUDA(cudaGetLastError());
            bt.raw_built = true;
        }
        if (raw) launch_bins<kRaw, P, BtR<P>>(t, bt, fp, n_pixels, nf, o0, o2, o1, s, o3, 1, masks, mask_stride);
        else launch_bins<kRaw, P, BtR<P>>(t, bt, fp, n_pixels, nf, o0, o1, nullptr, s, nullptr, 0, masks, mask_stride);
        DG_CUDA(cudaGetLastError());
        return true;
    }
    // Raw sums over the plan mask on a bin-tile plan: the tiles write them.
    if (raw && mode != kRaw && gather_variant_needs_tiles(t.variant) &&
        t.bt[t.variant - 7].n_items > 0) {
        const BinTiles &bt = t.bt[t.variant - 7];
        if (mode == kErrors) {
            if (t.variant == 7) launch_bins<kErrors, P, Bt7>(t, bt, fp, n_pixels, nf, o0, o2, o1, s, o3, 1);
            else launch_bins<kErrors, P, Bt8>(t, bt, fp, n_pixels, nf, o0, o2, o1, s, o3, 1);
        } else {
            if (t.variant == 7) launch_bins<kIntensity, P, Bt7>(t, bt, fp, n_pixels, nf, o0, nullptr, o1, s, o3, 1);
            else launch_bins<kIntensity, P, Bt8>(t, bt, fp, n_pixels, nf, o0, nullptr, o1, s, o3, 1);
        }
        DG_CUDA(cudaGetLastError());
        return true;
    }
    if (mode == kRaw)
        launch_gather<kRaw, P>(t, t.variant, fp, n_pixels, nf, t.partial.ptr, s, masks, mask_stride);
    else if (mode == kErrors)
        launch_gather<kErrors, P>(t, t.variant, fp, n_pixels, nf, t.partial.ptr, s);
    else
        launch_gather<kIntensity, P>(t, t.variant, fp, n_pixels, nf, t.partial.ptr, s);
    return false;
}

}  // namespace

void run_gather_raw(GatherTable &t, const void *d_frames, int dtype, int64_t n_pixels,
                    int64_t n_frames, const uint8_t *d_masks, int64_t mask_stride, uint32_t flags,
                    bool raw, double *o0, double *o1, double *o2, double *o3, cudaStream_t s) {
    if (n_frames <= 0) return;
    if (dtype < DG_U16 || dtype > DG_F64) fail(DG_INVALID_INPUT, "unknown pixel dtype");
    if (!t.cnt.ptr) fail(DG_DEVICE, "raw-sum entries were not prepared");
    const bool errors = (flags & DG_ERRORS) != 0;
    const int mode = d_masks ? kRaw : errors ? kErrors : kIntensity;
    const int64_t chunk = 256;
    const int64_t need = std::max<int64_t>(1, t.n_segments) *
                         n_accumulators(mode, dtype == DG_F32 || dtype == DG_F64) *
                         std::min<int64_t>(chunk, (n_frames + 31) / 32 * 32);
    if (t.partial.count < size_t(need)) t.partial.alloc(size_t(need));
    t.scratch.wait(s);
    const size_t esize = dtype == DG_U16 ? 2 : dtype == DG_F64 ? 8 : 4;
    for (int64_t f0 = 0; f0 < n_frames; f0 += chunk) {
        const int nf = int(std::min<int64_t>(chunk, n_frames - f0));
        const void *fp = static_cast<const unsigned char *>(d_frames) + f0 * n_pixels * esize;
        const uint8_t *mp = d_masks ? d_masks + f0 * mask_stride : nullptr;
        const int64_t off = f0 * t.n_rows;
        auto at = [&](double *o) { return o ? o + off : nullptr; };
        bool done = false;  // raw sums written by the bin tiles themselves
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
            // raw: S, N, V, C; normalised (per-frame masks only): I, sigma
            double *r0 = at(o0), *r1 = at(o1), *r2 = raw && errors ? at(o2) : nullptr,
                   *r3 = raw ? at(o3) : nullptr;
            if (!raw && !errors) r1 = nullptr;
#define DG_RAW_CALL(T) \
    done = launch_raw<T>(t, fp, n_pixels, nf, mode, mp, mask_stride, s, raw, r0, r1, r2, r3)
            switch (dtype) {
            case DG_U16: DG_RAW_CALL(uint16_t); break;
            case DG_U32: DG_RAW_CALL(uint32_t); break;
            case DG_I32: DG_RAW_CALL(int32_t); break;
            case DG_F32: DG_RAW_CALL(float); break;
            case DG_F64: DG_RAW_CALL(double); break;
            }
#undef DG_RAW_CALL
            if (ev) DG_CUDA(cudaEventRecord(ev->second, s));
        }
        if (t.n_rows == 0 || done) continue;
        ++t.launches;
        const dim3 grid(unsigned((t.n_rows + kFinRows - 1) / kFinRows), unsigned((nf + 31) / 32));
        if (raw) {
#define DG_RAW_ARGS                                                                          \
    t.partial.ptr, t.row_seg.ptr, t.seg_ids.ptr, t.den.ptr, t.cnt.ptr, t.n_rows, nf, at(o0), \
        at(o1), errors ? at(o2) : nullptr, at(o3)
            if (mode == kRaw) k_finalize_raw<kRaw><<<grid, 32 * kFinRows, 0, s>>>(DG_RAW_ARGS);
            else if (mode == kErrors) k_finalize_raw<kErrors><<<grid, 32 * kFinRows, 0, s>>>(DG_RAW_ARGS);
            else k_finalize_raw<kIntensity><<<grid, 32 * kFinRows, 0, s>>>(DG_RAW_ARGS);
#undef DG_RAW_ARGS
            DG_CUDA(cudaGetLastError());
        } else {
            if (mode != kRaw) fail(DG_INVALID_INPUT, "normalised results need per-frame masks");
            double *oi = at(o0), *os = errors ? at(o1) : nullptr;
            launch_finalize<kRaw, float>(t, t.partial.ptr, nf, oi, os, nullptr, s);
        }
    }
    t.scratch.mark(s);
}

namespace {

// One integration with mapping `variant`: the gather and, unless it wrote the
// results itself, the finalize (the autotuner compares whole integrations).
template <typename P>
void launch_mode(GatherTable &t, int variant, int mode, const void *frames, int64_t n_pixels,
                 int nf, double *oi, double *os, double *od, cudaStream_t s) {
    if (!launch_typed<P>(t, variant, frames, n_pixels, nf, mode, t.partial.ptr, oi, os, od, s) &&
        t.n_rows > 0)
        finalize_typed<P>(t, mode, t.partial.ptr, nf, oi, os, od, s);
}

}  // namespace

int gather_variant_count() { return kVariantCount; }

bool gather_variant_available(const GatherTable &t, int variant) {
    if (variant < 0 || variant >= kVariantCount) return false;
    if (variant == 5 || variant == 6) return t.fl_n_units > 0;
    if (variant == 7 || variant == 8) return t.bt[variant - 7].n_items > 0;
    if (variant == 10) return t.rw_n_items > 0;
    return true;
}

int autotune_gather(GatherTable &t, const void *d_frames, int dtype, int64_t n_pixels,
                    int64_t n_frames, uint32_t flags, cudaStream_t s,
                    std::vector<double> *each) {
    if (dtype < DG_U16 || dtype > DG_F64) fail(DG_INVALID_INPUT, "unknown pixel dtype");
    if (n_frames <= 0) fail(DG_INVALID_INPUT, "autotuning needs at least one frame");
    const int mode = (flags & DG_AZIMUTHAL_STD) ? kSpread : (flags & DG_ERRORS) ? kErrors
                                                                                : kIntensity;
    const int nf = int(std::min<int64_t>(n_frames, 256));
    reserve_partials(t, nf, flags, dtype, true);
    t.scratch.wait(s);
    if (each) each->assign(size_t(kVariantCount), 0.0);
    if (t.n_units == 0) return t.variant;
    DeviceArray<double> outs;
    outs.alloc(size_t(std::max<int64_t>(1, int64_t(t.n_rows) * nf * 3)));
    double *oi = outs.ptr, *os = oi + int64_t(t.n_rows) * nf, *od = os + int64_t(t.n_rows) * nf;
    if (!(flags & DG_ERRORS)) os = nullptr;
    if (!(flags & DG_AZIMUTHAL_STD)) od = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    DG_CUDA(cudaEventCreate(&a));
    DG_CUDA(cudaEventCreate(&b));
    int best = t.variant;
    float best_t = 3.4e38f;
    try {
        for (int v = 0; v < kVariantCount; ++v) {
            if (!gather_variant_available(t, v) ||
                (gather_variant_needs_tiles(v) && !bin_tiles_fill_gpu(t, v, n_frames))) {
                if (each) (*each)[size_t(v)] = -1.0;
                continue;
            }
            float vt = 3.4e38f;
            for (int rep = 0; rep < 4; ++rep) {
                DG_CUDA(cudaEventRecord(a, s));
                switch (dtype) {
                case DG_U16: launch_mode<uint16_t>(t, v, mode, d_frames, n_pixels, nf, oi, os, od, s); break;
                case DG_U32: launch_mode<uint32_t>(t, v, mode, d_frames, n_pixels, nf, oi, os, od, s); break;
                case DG_I32: launch_mode<int32_t>(t, v, mode, d_frames, n_pixels, nf, oi, os, od, s); break;
                case DG_F32: launch_mode<float>(t, v, mode, d_frames, n_pixels, nf, oi, os, od, s); break;
                case DG_F64: launch_mode<double>(t, v, mode, d_frames, n_pixels, nf, oi, os, od, s); break;
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
    t.scratch.mark(s);
    t.variant = best;
    return best;
}

}  // namespace dg

// ---------------------------------------------------------------------------
// Fixed scratch of the allocation-free entry point (dg_integrate_device_noalloc
// in dg_api.cu).
//
// Some callers may not allocate device memory while they integrate: a
// real-time acquisition loop with a fixed memory budget, a host thread that
// must not enter the CUDA allocator, code running where cudaMalloc is not
// permitted. dg_integrate_device allocates its per-segment partial sums on
// first use; the allocation-free entry point keeps them in this one fixed
// array instead. It is a file-scope __device__ variable of
// kNoAllocScratchBytes, which every GPU that loads the library holds until
// the process exits. Host code cannot use its name as a device address (a
// kernel given the host-side name would fault or read the wrong memory), so
// its address is looked up with cudaGetSymbolAddress, with the device
// current, on every call: the lookup allocates nothing once the module is
// loaded, the first call on a device loads it (make that call before any
// stream capture), and an address never outlives a context that was reset.
namespace dg {
namespace {
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB per device
static __device__ __align__(256) double g_noalloc_partial[kNoAllocScratchBytes / sizeof(double)];
}  // namespace

double *noalloc_scratch(size_t *n_doubles) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partial);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        fail(DG_DEVICE, std::string("cudaGetSymbolAddress of the fixed scratch array failed: ") +
                            cudaGetErrorString(e));
    }
    *n_doubles = kNoAllocScratchBytes / sizeof(double);
    return static_cast<double *>(p);
}

}  // namespace dg
