// Device construction of the integration lookup tables.
//
// Compiled with -fmad=false: every a*b+c below is a separate multiply and
// add, in C's left-to-right order, which is the order the reference's Rust
// evaluates (Rust never contracts to FMA unless mul_add is written). Double
// division and sqrt are IEEE round-to-nearest on the device, and atan2 and sin
// are the correctly rounded double-double versions of dg_ddmath.cuh, so a
// corner's 2-theta and chi are the bits the C library gives the reference
// (cos, used only for the polarisation factor, is CUDA's). Table indices
// depend on corners through floor((r - min)/step) and through clip areas,
// whose shoelace sums amplify a last-bit change of a corner ~1e5-fold; the
// build also counts the corners that lie within a guard band of a bin edge
// (guard_corners), where any remaining difference could show.
//
// Every builder is count -> exclusive scan -> fill, first into a pixel-major
// list of (pixel, bin, weight) contributions, then transposed into CSR rows by
// a stable, sort-free placement: pixels are split into chunks, per-(chunk, bin)
// counts are scanned down the chunks, and one warp per chunk walks its
// contributions in pixel order, ranking equal bins inside the warp with
// __match_any_sync. Rows therefore list pixels in ascending order, exactly the
// order the reference's serial fills produce.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "dg_ddmath.cuh"
#include "dg_internal.h"

namespace dg {

GeomParams make_geom_params(const dg_geometry &g, const dg_method &m) {
    GeomParams p{};
    p.pixel1 = g.pixel1;
    p.pixel2 = g.pixel2;
    p.distance = g.distance;
    p.poni1 = g.poni1;
    p.poni2 = g.poni2;
    // TrigonometricConstants::new (geometry.rs:648-659), glibc on the host.
    p.s1 = std::sin(g.rot1);
    p.c1 = std::cos(g.rot1);
    p.s2 = std::sin(g.rot2);
    p.c2 = std::cos(g.rot2);
    p.s3 = std::sin(g.rot3);
    p.c3 = std::cos(g.rot3);
    p.wavelength = g.wavelength;
    p.unit = m.unit;
    // RadialConverter::new (integration.rs:147-158).
    const double pi = 3.14159265358979323846;
    if (m.unit == DG_UNIT_Q_A) p.q_scale = 4.0 * pi / (g.wavelength * 1e10);
    else if (m.unit == DG_UNIT_Q_NM) p.q_scale = 4.0 * pi / (g.wavelength * 1e9);
    else p.q_scale = 0.0;
    p.has_pol = m.has_polarization;
    p.pol_factor = m.polarization_factor;
    return p;
}

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTau = 6.28318530717958647692;
constexpr double kEps = DBL_EPSILON;
constexpr int kClipCap = 16;

// ------------------------------------------------------------ geometry

// f_x1/f_x2/f_x3 (geometry.rs:663-680) in Rust's evaluation order.
__device__ __forceinline__ void sample_xyz(const GeomParams &g, double p1, double p2, double &x,
                                           double &y, double &z) {
    const double p3 = g.distance;
    x = p1 * g.c2 * g.c3 + p2 * (g.c3 * g.s1 * g.s2 - g.c1 * g.s3) -
        p3 * (g.c1 * g.c3 * g.s2 + g.s1 * g.s3);
    y = p1 * g.c2 * g.s3 + p2 * (g.c1 * g.c3 + g.s1 * g.s2 * g.s3) -
        p3 * (-(g.c3 * g.s1) + g.c1 * g.s2 * g.s3);
    z = p1 * g.s2 - p2 * g.c2 * g.s1 + p3 * g.c1 * g.c2;
}

// RadialConverter::convert (integration.rs:160-172).
__device__ __forceinline__ double to_unit(const GeomParams &g, double tth) {
    switch (g.unit) {
    case DG_UNIT_TTH_DEG: return tth * (180.0 / kPi);
    case DG_UNIT_Q_A:
    case DG_UNIT_Q_NM: return g.q_scale * ddm::cr_sin(tth * 0.5);
    default: return tth;
    }
}

// (radial, chi) at detector coordinates d1, d2 in pixels (geometry.rs:519-549,
// f_tth :684, f_azimuth :690).
__device__ __forceinline__ void radial_chi(const GeomParams &g, double d1, double d2, double &r,
                                           double &chi) {
    double x, y, z;
    sample_xyz(g, d1 * g.pixel1 - g.poni1, d2 * g.pixel2 - g.poni2, x, y, z);
    r = to_unit(g, ddm::cr_atan2(sqrt(y * y + x * x), z));
    chi = ddm::cr_atan2(x, y);
}

// Corner grid (geometry.rs:229-278): corner (i, j) at i * pixel - poni.
__global__ void k_corners(GeomParams g, int dim1, int dim2, double *__restrict__ rc,
                          double *__restrict__ ac) {
    int64_t n = int64_t(dim1 + 1) * (dim2 + 1);
    for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n;
         k += int64_t(gridDim.x) * blockDim.x) {
        int64_t i = k / (dim2 + 1), j = k % (dim2 + 1);
        double x, y, z;
        sample_xyz(g, double(i) * g.pixel1 - g.poni1, double(j) * g.pixel2 - g.poni2, x, y, z);
        rc[k] = to_unit(g, ddm::cr_atan2(sqrt(y * y + x * x), z));
        ac[k] = ddm::cr_atan2(x, y);
    }
}

// compute_geometry (corrections.rs:57-85): centre radial, chi and the
// normalisation pol * sa with sa = cos^3 (geometry.rs:697-707) and
// pol = 0.5*(1 + c2 - f*cos(2 chi)*(1 - c2)) (geometry.rs:625-636, :715-717).
__global__ void k_centres(GeomParams g, int dim1, int dim2, double *__restrict__ radial,
                          double *__restrict__ chi, double *__restrict__ norm) {
    int64_t n = int64_t(dim1) * dim2;
    for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n;
         k += int64_t(gridDim.x) * blockDim.x) {
        int64_t i = k / dim2, j = k % dim2;
        double d1 = (double(i) + 0.5) * g.pixel1 - g.poni1;
        double d2 = (double(j) + 0.5) * g.pixel2 - g.poni2;
        double x, y, z;
        sample_xyz(g, d1, d2, x, y, z);
        double tth = ddm::cr_atan2(sqrt(y * y + x * x), z);
        double az = ddm::cr_atan2(x, y);
        double cosa = g.distance / sqrt(d1 * d1 + d2 * d2 + g.distance * g.distance);
        double sa = cosa * (cosa * cosa);
        double pol = 1.0;
        if (g.has_pol) {
            double c = cos(tth);
            double c2 = c * c;
            pol = 0.5 * (1.0 + c2 - g.pol_factor * cos(2.0 * az) * (1.0 - c2));
        }
        radial[k] = to_unit(g, tth);
        chi[k] = az;
        norm[k] = pol * sa;
    }
}

// Monotone unsigned key of a double, for atomicMin/atomicMax.
__device__ __forceinline__ unsigned long long dkey(double v) {
    unsigned long long b = __double_as_longlong(v);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

double key_to_double(unsigned long long k) {
    unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    double v;
    std::memcpy(&v, &b, sizeof v);
    return v;
}

__global__ void k_minmax(const double *__restrict__ v, int64_t n, unsigned long long *out) {
    unsigned long long lo = ~0ull, hi = 0ull;
    for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n;
         k += int64_t(gridDim.x) * blockDim.x) {
        unsigned long long key = dkey(v[k]);
        lo = key < lo ? key : lo;
        hi = key > hi ? key : hi;
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long a = __shfl_down_sync(0xffffffffu, lo, o);
        unsigned long long b = __shfl_down_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&out[0], lo);
        atomicMax(&out[1], hi);
    }
}

// hull_grid (lut/common.rs:33-65) point k: radial extremes into out and,
// when out_az is given, azimuthal extremes into out_az.
__global__ void k_hull_minmax(GeomParams g, int dim1, int dim2, int n_ss,
                              unsigned long long *out, unsigned long long *out_az) {
    int64_t a = int64_t(dim1) * n_ss, b = int64_t(dim2) * n_ss - 1;
    int64_t n = 2 * a + 2 * b;
    double off = 0.5 / double(n_ss), st = 1.0 / double(n_ss);
    unsigned long long lo = ~0ull, hi = 0ull, alo = ~0ull, ahi = 0ull;
    for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n;
         k += int64_t(gridDim.x) * blockDim.x) {
        double d1, d2;
        if (k < a) { d1 = off + double(k) * st; d2 = off; }
        else if (k < 2 * a) { d1 = off + double(k - a) * st; d2 = double(dim2) - off; }
        else if (k < 2 * a + b) { d1 = off; d2 = off + double(k - 2 * a + 1) * st; }
        else { d1 = double(dim1) - off; d2 = off + double(k - 2 * a - b + 1) * st; }
        double r, chi;
        radial_chi(g, d1, d2, r, chi);
        unsigned long long key = dkey(r);
        lo = key < lo ? key : lo;
        hi = key > hi ? key : hi;
        key = dkey(chi);
        alo = key < alo ? key : alo;
        ahi = key > ahi ? key : ahi;
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long x = __shfl_down_sync(0xffffffffu, lo, o);
        unsigned long long y = __shfl_down_sync(0xffffffffu, hi, o);
        lo = x < lo ? x : lo;
        hi = y > hi ? y : hi;
        x = __shfl_down_sync(0xffffffffu, alo, o);
        y = __shfl_down_sync(0xffffffffu, ahi, o);
        alo = x < alo ? x : alo;
        ahi = y > ahi ? y : ahi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&out[0], lo);
        atomicMax(&out[1], hi);
        if (out_az) {
            atomicMin(&out_az[0], alo);
            atomicMax(&out_az[1], ahi);
        }
    }
}

// ------------------------------------------------------- bin helpers

// `f as usize` / `f as isize` in Rust: truncating, saturating, NaN -> 0; the
// PTX conversions cvt.rzi.{u64,s64}.f64 have exactly those semantics.
__device__ __forceinline__ unsigned long long as_usize(double v) { return __double2ull_rz(v); }
__device__ __forceinline__ long long as_isize(double v) { return __double2ll_rz(v); }

__device__ __forceinline__ double rem_euclid_tau(double x) {
    double r = fmod(x, kTau);
    return r < 0.0 ? r + kTau : r;
}
// wrap_tau (pyfai_1d.rs:170-177).
__device__ __forceinline__ double wrap_tau(double x) {
    return (x >= 0.0 && x < kTau) ? x : rem_euclid_tau(x);
}

struct Pt {
    double x, y;
};

// polygon_area (pixel_split.rs:14-25).
__device__ double polygon_area(const Pt *p, int n) {
    if (n < 3) return 0.0;
    double area = 0.0;
    for (int i = 0; i < n; ++i) {
        Pt a = p[i], b = p[i + 1 == n ? 0 : i + 1];
        area += a.x * b.y - b.x * a.y;
    }
    return 0.5 * area;
}

// intersect_with_x / intersect_with_y (pixel_split.rs:28-45).
__device__ __forceinline__ Pt isect(Pt p0, Pt p1, double e, bool vertical) {
    if (vertical) {
        double dx = p1.x - p0.x;
        if (fabs(dx) < kEps) return Pt{e, p0.y};
        double t = (e - p0.x) / dx;
        return Pt{e, p0.y + t * (p1.y - p0.y)};
    }
    double dy = p1.y - p0.y;
    if (fabs(dy) < kEps) return Pt{p0.x, e};
    double t = (e - p0.y) / dy;
    return Pt{p0.x + t * (p1.x - p0.x), e};
}

// One Sutherland-Hodgman pass (pixel_split.rs:48-145); side 0: x >= e,
// 1: x <= e, 2: y >= e, 3: y <= e. Sets *overflow instead of writing past cap.
__device__ int clip_pass(const Pt *in, int n, double e, int side, Pt *out, int *overflow) {
    if (n == 0) return 0;
    int m = 0;
    auto inside = [&](Pt p) {
        return side == 0 ? p.x >= e : side == 1 ? p.x <= e : side == 2 ? p.y >= e : p.y <= e;
    };
    const bool vertical = side < 2;
    Pt prev = in[n - 1];
    bool prev_in = inside(prev);
    for (int i = 0; i < n; ++i) {
        Pt cur = in[i];
        bool cur_in = inside(cur);
        if (cur_in) {
            if (!prev_in) {
                if (m < kClipCap) out[m] = isect(prev, cur, e, vertical);
                ++m;
            }
            if (m < kClipCap) out[m] = cur;
            ++m;
        } else if (prev_in) {
            if (m < kClipCap) out[m] = isect(prev, cur, e, vertical);
            ++m;
        }
        prev = cur;
        prev_in = cur_in;
    }
    if (m > kClipCap) {
        *overflow = 1;
        m = kClipCap;
    }
    return m;
}

// clip_polygon_rect_scratch (pixel_split.rs:148-163) followed by |area|.
__device__ double clipped_area(const Pt *poly, double x0, double x1, double y0, double y1,
                               int *overflow) {
    Pt b1[kClipCap], b2[kClipCap];
    int m = clip_pass(poly, 4, x0, 0, b1, overflow);
    if (!m) return 0.0;
    m = clip_pass(b1, m, x1, 1, b2, overflow);
    if (!m) return 0.0;
    m = clip_pass(b2, m, y0, 2, b1, overflow);
    if (!m) return 0.0;
    m = clip_pass(b1, m, y1, 3, b2, overflow);
    return fabs(polygon_area(b2, m));
}

// unwrap_angle (pixel_split.rs:166-175).
__device__ __forceinline__ double unwrap_angle(double a, double ref) {
    double d = a - ref;
    if (d > kPi) a -= 2.0 * kPi;
    else if (d < -kPi) a += 2.0 * kPi;
    return a;
}

// singular (pyfai_1d.rs:188-201).
__device__ bool singular(const Pt *p) {
    double winding = 0.0;
    for (int i = 0; i < 4; ++i) {
        if (p[i].x == 0.0) return true;
        double delta = wrap_tau(p[(i + 1) & 3].y - p[i].y + kPi) - kPi;
        if (fabs(delta) >= kPi - 64.0 * kEps) return true;
        winding += delta;
    }
    return fabs(winding) > kPi;
}

// ----------------------------------------------------- pixel split 1D

struct Ps1d {
    GeomParams g;
    int dim1, dim2;
    int n;
    double min, step, r1;
    int have_grid, clamp_low;
    const double *rc, *ac, *cr, *cc;
};

// One pixel of lut1d_ps_fractions (pixel_split.rs:214-310). Returns the
// number of entries; with FILL, writes them. Returns -1 for a singular pixel
// (detector-plane sampling, done by k_sample).
template <bool FILL>
__device__ int ps1d_pixel(const Ps1d &a, int64_t idx, int *bins, double *ws, int *overflow) {
    const int64_t w = a.dim2 + 1;
    int64_t b0 = idx / a.dim2 * w + idx % a.dim2;
    int64_t i00 = b0, i01 = b0 + 1, i11 = b0 + w + 1, i10 = b0 + w;
    double r00 = a.rc[i00], r01 = a.rc[i01], r10 = a.rc[i10], r11 = a.rc[i11];
    if (a.have_grid) {
        Pt raw[4] = {{r00, a.ac[i00]}, {r01, a.ac[i01]}, {r11, a.ac[i11]}, {r10, a.ac[i10]}};
        if (singular(raw)) return -1;
    }
    double cchi = a.cc[idx];
    double a00 = unwrap_angle(a.ac[i00], cchi);
    double a01 = unwrap_angle(a.ac[i01], cchi);
    double a10 = unwrap_angle(a.ac[i10], cchi);
    double a11 = unwrap_angle(a.ac[i11], cchi);
    Pt poly[4] = {{r00, a00}, {r01, a01}, {r11, a11}, {r10, a10}};
    double area_total = fabs(polygon_area(poly, 4));
    if (area_total <= 0.0) {
        double pos = (a.cr[idx] - a.min) / a.step;
        if (pos < 0.0) return 0;
        long long bin = as_isize(floor(pos));
        if (bin >= 0 && bin < a.n) {
            if (FILL) {
                bins[0] = int(bin);
                ws[0] = 1.0;
            }
            return 1;
        }
        return 0;
    }
    double rmin = r00, rmax = r00;
    double rv[3] = {r01, r10, r11};
    for (int k = 0; k < 3; ++k) {
        if (rv[k] < rmin) rmin = rv[k];
        if (rv[k] > rmax) rmax = rv[k];
    }
    long long start = as_isize(floor((rmin - a.min) / a.step));
    long long end = as_isize(floor((rmax - a.min) / a.step));
    if (end < 0 || start >= a.n) return 0;
    if (start < 0) start = 0;
    if (end >= a.n) end = a.n - 1;
    double amin = a00, amax = a00;
    double av[3] = {a01, a10, a11};
    for (int k = 0; k < 3; ++k) {
        if (av[k] < amin) amin = av[k];
        if (av[k] > amax) amax = av[k];
    }
    int m = 0;
    for (long long b = start; b <= end; ++b) {
        double bin_min = a.min + double(b) * a.step;
        double bin_max = bin_min + a.step;
        double area = clipped_area(poly, bin_min, bin_max, amin, amax, overflow);
        if (area > 0.0) {
            if (FILL) {
                bins[m] = int(b);
                ws[m] = area / area_total;
            }
            ++m;
        }
    }
    return m;
}

__global__ void k_ps1d_count(Ps1d a, int32_t *__restrict__ count, int32_t *__restrict__ sing,
                             int32_t sing_cap, int32_t *__restrict__ n_sing, int *overflow) {
    int64_t n = int64_t(a.dim1) * a.dim2;
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n;
         p += int64_t(gridDim.x) * blockDim.x) {
        int c = ps1d_pixel<false>(a, p, nullptr, nullptr, overflow);
        if (c < 0) {
            int slot = atomicAdd(n_sing, 1);
            if (slot < sing_cap) sing[slot] = int32_t(p);
            c = 0;
        }
        count[p] = c;
    }
}

// pyfai_1d::sample (pyfai_1d.rs:208-252) for singular pixel blockIdx.x: 128 x
// 128 x 4 detector-plane samples counted per radial bin of [r0, r1).
__global__ void k_sample(GeomParams g, int dim2, const int32_t *__restrict__ sing, int n,
                         double r0, double r1, int clamp_low, int32_t *__restrict__ hits) {
    const int N = 128;
    const double off[4][2] = {{0.25, 0.5}, {0.5, 0.25}, {0.75, 0.5}, {0.5, 0.75}};
    int32_t pixel = sing[blockIdx.x];
    int32_t *h = hits + int64_t(blockIdx.x) * n;
    double prow = double(pixel / dim2), pcol = double(pixel % dim2);
    const double a0 = -kPi, a1 = kPi;
    for (int s = threadIdx.x; s < N * N * 4; s += blockDim.x) {
        int row = s / (N * 4), col = (s / 4) % N, o = s & 3;
        double d1 = prow + (double(row) + off[o][0]) / double(N);
        double d2 = pcol + (double(col) + off[o][1]) / double(N);
        double r, az;
        radial_chi(g, d1, d2, r, az);
        az = a0 + rem_euclid_tau(az - a0);
        if ((r < r0 && !clamp_low) || r >= r1 || az >= a1) continue;
        unsigned long long ir = r < r0 ? 0ull : as_usize((r - r0) / (r1 - r0) * double(n));
        unsigned long long ia = as_usize((az - a0) / (a1 - a0) * 1.0);
        if (ir < (unsigned long long)n && ia < 1ull) atomicAdd(&h[ir], 1);
    }
}

__global__ void k_sample_count(const int32_t *__restrict__ sing, int n,
                               const int32_t *__restrict__ hits, int32_t *__restrict__ count) {
    const int32_t *h = hits + int64_t(blockIdx.x) * n;
    int c = 0;
    for (int b = threadIdx.x; b < n; b += blockDim.x) c += h[b] != 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    __shared__ int ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int i = 0; i < int(blockDim.x + 31) / 32; ++i) t += ws[i];
        count[sing[blockIdx.x]] = t;
    }
}

// Fill of the pixel-major contribution list; singular pixels copy their
// sampled hits (bins ascending, weight hits / 65536).
__global__ void k_ps1d_fill(Ps1d a, const int64_t *__restrict__ off,
                            const int32_t *__restrict__ sing_slot,
                            const int32_t *__restrict__ hits, int32_t *__restrict__ cbin,
                            double *__restrict__ cw, int32_t *__restrict__ cpix, int *overflow) {
    int64_t n = int64_t(a.dim1) * a.dim2;
    int bins[kClipCap * 4];
    double ws[kClipCap * 4];
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n;
         p += int64_t(gridDim.x) * blockDim.x) {
        int64_t o = off[p];
        int32_t s = sing_slot ? sing_slot[p] : -1;
        if (s >= 0) {
            const int32_t *h = hits + int64_t(s) * a.n;
            for (int b = 0; b < a.n; ++b)
                if (h[b]) {
                    cbin[o] = b;
                    cw[o] = double(h[b]) / 65536.0;
                    cpix[o] = int32_t(p);
                    ++o;
                }
            continue;
        }
        // Entries of one pixel are produced in bin order; the local buffer
        // holds a chunk at a time so very wide pixels need no large array.
        int total = int(off[p + 1] - off[p]);
        if (total <= kClipCap * 4) {
            int m = ps1d_pixel<true>(a, p, bins, ws, overflow);
            for (int k = 0; k < m; ++k) {
                cbin[o + k] = bins[k];
                cw[o + k] = ws[k];
                cpix[o + k] = int32_t(p);
            }
        } else {
            // Rare: a pixel spanning more bins than the local buffer. Redo the
            // walk bin by bin (same arithmetic as ps1d_pixel).
            const int64_t w = a.dim2 + 1;
            int64_t b0 = p / a.dim2 * w + p % a.dim2;
            int64_t i00 = b0, i01 = b0 + 1, i11 = b0 + w + 1, i10 = b0 + w;
            double cchi = a.cc[p];
            double a00 = unwrap_angle(a.ac[i00], cchi), a01 = unwrap_angle(a.ac[i01], cchi);
            double a10 = unwrap_angle(a.ac[i10], cchi), a11 = unwrap_angle(a.ac[i11], cchi);
            double r00 = a.rc[i00], r01 = a.rc[i01], r10 = a.rc[i10], r11 = a.rc[i11];
            Pt poly[4] = {{r00, a00}, {r01, a01}, {r11, a11}, {r10, a10}};
            double area_total = fabs(polygon_area(poly, 4));
            double rmin = r00, rmax = r00;
            double rv[3] = {r01, r10, r11};
            for (int k = 0; k < 3; ++k) {
                if (rv[k] < rmin) rmin = rv[k];
                if (rv[k] > rmax) rmax = rv[k];
            }
            long long start = as_isize(floor((rmin - a.min) / a.step));
            long long end = as_isize(floor((rmax - a.min) / a.step));
            if (start < 0) start = 0;
            if (end >= a.n) end = a.n - 1;
            double amin = a00, amax = a00;
            double av[3] = {a01, a10, a11};
            for (int k = 0; k < 3; ++k) {
                if (av[k] < amin) amin = av[k];
                if (av[k] > amax) amax = av[k];
            }
            for (long long b = start; b <= end; ++b) {
                double bin_min = a.min + double(b) * a.step;
                double area = clipped_area(poly, bin_min, bin_min + a.step, amin, amax, overflow);
                if (area > 0.0) {
                    cbin[o] = int(b);
                    cw[o] = area / area_total;
                    cpix[o] = int32_t(p);
                    ++o;
                }
            }
        }
    }
}

// ----------------------------------------------- pyFAI full split 1D

struct Pf1d {
    int dim1, dim2, n;
    double r0, r1;
    const double *rc, *ac;
};
constexpr int kPfCap = 64;  // radial bins one pixel may span

// split1d (pyfai_1d.rs:259-354) on n radial bins over [r0, r1), azimuthal
// edges (-pi, pi), no sector, corner sign +1 (a geometry without a detector
// object, pyfai_1d.rs:131-137). poly in pyFAI order A, D, C, B. Returns the
// number of weights kept; with FILL writes them. Sets *overflow when the
// pixel spans more than kPfCap bins.
template <bool FILL>
__device__ int pf_split1d(Pt poly[4], int n, double r0, double r1, int *bins, double *ws,
                          int *overflow) {
    for (int i = 0; i < 4; ++i) poly[i].y = wrap_tau(poly[i].y - 0.0 + kPi) - kPi;
    const Pt a = poly[0], b = poly[1], c = poly[2], d = poly[3];
    const double area = 1.0 * (0.5 * (c.x - a.x) * (d.y - b.y) - (c.y - a.y) * (d.x - b.x));
    if (area > 0.0) {
        for (int i = 0; i < 4; ++i)
            if (poly[i].y < 0.0) poly[i].y += kTau;
        double sum = -0.0;
        for (int i = 0; i < 4; ++i) sum += poly[i].y;
        if (sum * 0.25 > kPi)
            for (int i = 0; i < 4; ++i) poly[i].y -= kTau;
    }
    for (int i = 0; i < 4; ++i) poly[i].y += 0.0;
    const double dr = (r1 - r0) / double(n);
    for (int i = 0; i < 4; ++i) poly[i].x = (poly[i].x - r0) / dr;
    double lo = INFINITY, hi = -INFINITY;
    for (int i = 0; i < 4; ++i) {
        lo = fmin(lo, poly[i].x);
        hi = fmax(hi, poly[i].x);
    }
    if (hi < 0.0 || lo >= double(n)) return 0;
    const double flo = floor(lo), fhi = floor(hi);
    const long long first = (long long)as_usize(fmax(flo, 0.0));
    long long end = as_isize(fhi) + 1;
    if (end < 0) end = 0;
    if (end > n) end = n;
    if (flo == fhi) {
        if (FILL) {
            bins[0] = int(first);
            ws[0] = 1.0;
        }
        return 1;
    }
    const int span = int(end - first);
    if (span > kPfCap) {
        atomicExch(overflow + 1, 1);
        return 0;
    }
    float buffer[kPfCap];
    for (int j = 0; j < span; ++j) buffer[j] = 0.0f;
    for (int i = 0; i < 4; ++i) {
        const double x0 = poly[i].x, y0 = poly[i].y;
        const double x1 = poly[(i + 1) & 3].x, y1 = poly[(i + 1) & 3].y;
        if (x0 == x1) continue;
        const double slope = (y1 - y0) / (x1 - x0);
        const double intercept = y0 - slope * x0;
        const double sg = x1 > x0 ? 1.0 : -1.0;
        for (int j = 0; j < span; ++j) {
            const double left = fmax(fmin(x0, x1), double(first + j));
            const double right = fmin(fmax(x0, x1), double(first + j + 1));
            if (right > left)
                buffer[j] = __fadd_rn(buffer[j], __double2float_rn(
                    sg * (right - left) * (0.5 * slope * (right + left) + intercept)));
        }
    }
    double sum = -0.0;
    for (int j = 0; j < span; ++j) sum += double(buffer[j]);
    if (!isfinite(sum) || sum == 0.0) return 0;
    int m = 0;
    double total = -0.0;
    for (int j = 0; j < span; ++j) {
        const double w = double(buffer[j]) / sum;
        if (isfinite(w) && w > 0.0) {
            total += w;
            if (FILL) {
                bins[m] = int(first + j);
                ws[m] = w;
            }
            ++m;
        }
    }
    if (FILL)
        for (int k = 0; k < m; ++k) ws[k] /= total;
    return m;
}

// One pixel of build_lut1d_pyfai_csr (pyfai_1d.rs:77-93); -1 for a singular
// pixel (detector-plane sampling, done by k_sample).
template <bool FILL>
__device__ int pf1d_pixel(const Pf1d &a, int64_t idx, int *bins, double *ws, int *overflow) {
    const int64_t w = a.dim2 + 1;
    const int64_t b0 = idx / a.dim2 * w + idx % a.dim2;
    const int64_t ia = b0, ib = b0 + 1, ic = b0 + w + 1, id = b0 + w;
    // corner_indices A, B, C, D taken as [a, d, c, b] (pyfai_1d.rs:73-76)
    Pt poly[4] = {{a.rc[ia], a.ac[ia]}, {a.rc[id], a.ac[id]}, {a.rc[ic], a.ac[ic]},
                  {a.rc[ib], a.ac[ib]}};
    if (singular(poly)) return -1;
    return pf_split1d<FILL>(poly, a.n, a.r0, a.r1, bins, ws, overflow);
}

__global__ void k_pf1d_count(Pf1d a, int32_t *__restrict__ count, int32_t *__restrict__ sing,
                             int32_t sing_cap, int32_t *__restrict__ n_sing, int *overflow) {
    const int64_t n = int64_t(a.dim1) * a.dim2;
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n;
         p += int64_t(gridDim.x) * blockDim.x) {
        int c = pf1d_pixel<false>(a, p, nullptr, nullptr, overflow);
        if (c < 0) {
            const int slot = atomicAdd(n_sing, 1);
            if (slot < sing_cap) sing[slot] = int32_t(p);
            c = 0;
        }
        count[p] = c;
    }
}

__global__ void k_pf1d_fill(Pf1d a, const int64_t *__restrict__ off,
                            const int32_t *__restrict__ sing_slot,
                            const int32_t *__restrict__ hits, int32_t *__restrict__ cbin,
                            double *__restrict__ cw, int32_t *__restrict__ cpix, int *overflow) {
    const int64_t n = int64_t(a.dim1) * a.dim2;
    int bins[kPfCap];
    double ws[kPfCap];
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n;
         p += int64_t(gridDim.x) * blockDim.x) {
        int64_t o = off[p];
        const int32_t s = sing_slot ? sing_slot[p] : -1;
        if (s >= 0) {
            const int32_t *h = hits + int64_t(s) * a.n;
            for (int b = 0; b < a.n; ++b)
                if (h[b]) {
                    cbin[o] = b;
                    cw[o] = double(h[b]) / 65536.0;
                    cpix[o] = int32_t(p);
                    ++o;
                }
            continue;
        }
        const int m = pf1d_pixel<true>(a, p, bins, ws, overflow);
        for (int k = 0; k < m; ++k) {
            cbin[o + k] = bins[k];
            cw[o + k] = ws[k];
            cpix[o + k] = int32_t(p);
        }
    }
}

// Corners whose scaled position lies within a guard band of a bin edge: the
// only corners where a last-bit difference between CUDA's and glibc's atan2
// could move an index.
__global__ void k_guard(const double *__restrict__ rc, int64_t n, double min, double step,
                        unsigned long long *count) {
    unsigned long long c = 0;
    for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n;
         k += int64_t(gridDim.x) * blockDim.x) {
        double r = rc[k];
        double pos = (r - min) / step;
        double band = 64.0 * kEps * (fabs(r) + fabs(min)) / step + 4.0 * kEps * fabs(pos);
        c += fabs(pos - rint(pos)) <= band;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// ------------------------------------------------------- counting 1D

// build_lut1d_csr / _with_range (counting_csr.rs:54-134): one contribution of
// weight 1 per pixel in range.
__global__ void k_count1d(const double *__restrict__ radial, int64_t n, double min, double max,
                          double step, int nb, int has_range, int32_t *__restrict__ count,
                          int32_t *__restrict__ bin_of) {
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n;
         p += int64_t(gridDim.x) * blockDim.x) {
        double v = radial[p];
        int b = -1;
        if (!has_range || (v >= min && v <= max)) {
            unsigned long long q = as_usize((v - min) / step);
            b = q < (unsigned long long)(nb - 1) ? int(q) : nb - 1;
        }
        count[p] = b >= 0;
        bin_of[p] = b;
    }
}

__global__ void k_count1d_fill(const int32_t *__restrict__ bin_of, int64_t n,
                               const int64_t *__restrict__ off, int32_t *__restrict__ cbin,
                               double *__restrict__ cw, int32_t *__restrict__ cpix) {
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n;
         p += int64_t(gridDim.x) * blockDim.x) {
        int b = bin_of[p];
        if (b >= 0) {
            int64_t o = off[p];
            cbin[o] = b;
            cw[o] = 1.0;
            cpix[o] = int32_t(p);
        }
    }
}

// --------------------------------------------------- supersampled 1D

struct Ss1d {
    GeomParams g;
    int dim1, dim2, n_ss, nb, has_range;
    double min, max, step;
};

// build_counted_csr (supersampled.rs:21-104) for one pixel: samples
// d1 = row + (i + .5)/n, d2 = ((col*n + j) + .5)/n, distinct bins counted in
// first-seen order; weight count / n^2 (1D, normalize_bins = false).
template <bool FILL>
__device__ int ss1d_pixel(const Ss1d &a, int64_t p, int *bins, int *counts) {
    int64_t row = p / a.dim2, col = p % a.dim2;
    int nc = 0;
    for (int i = 0; i < a.n_ss; ++i) {
        double d1 = double(row) + (double(i) + 0.5) / double(a.n_ss);
        for (int j = 0; j < a.n_ss; ++j) {
            double d2 = (double(col * a.n_ss + j) + 0.5) / double(a.n_ss);
            double r, chi;
            radial_chi(a.g, d1, d2, r, chi);
            if (a.has_range && !(r >= a.min && r <= a.max)) continue;
            unsigned long long q = as_usize((r - a.min) / a.step);
            int b = q < (unsigned long long)(a.nb - 1) ? int(q) : a.nb - 1;
            int f = -1;
            for (int k = 0; k < nc; ++k)
                if (bins[k] == b) { f = k; break; }
            if (f < 0) { bins[nc] = b; counts[nc] = 1; ++nc; }
            else counts[f] += 1;
        }
    }
    return nc;
}

constexpr int kMaxSs = 8;

__global__ void k_ss1d(Ss1d a, const int64_t *__restrict__ off, int32_t *__restrict__ count,
                       int32_t *__restrict__ cbin, double *__restrict__ cw,
                       int32_t *__restrict__ cpix) {
    int64_t n = int64_t(a.dim1) * a.dim2;
    int bins[kMaxSs * kMaxSs], counts[kMaxSs * kMaxSs];
    double denom = double(a.n_ss * a.n_ss);
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n;
         p += int64_t(gridDim.x) * blockDim.x) {
        int nc = ss1d_pixel<true>(a, p, bins, counts);
        if (!off) {
            count[p] = nc;
            continue;
        }
        int64_t o = off[p];
        for (int k = 0; k < nc; ++k) {
            cbin[o + k] = bins[k];
            cw[o + k] = double(counts[k]) / denom;
            cpix[o + k] = int32_t(p);
        }
    }
}

// ------------------------------------------------------------ 2D tables

// IntegrationGrid2d (grid.rs:26-222) with its steps precomputed on the host
// as (hi - lo) / n, the reference's radial_step/azimuthal_step.
struct Grid2 {
    int nr, na;
    double r0, r1, a0, a1, dr, da;
    int clamp_radial_end, clamp_index_rounding, clamp_radial_outside, clamp_azimuthal_outside;
    int pyfai;
};

// IntegrationGrid2d::bin (grid.rs:176-222); -1 for no bin.
__device__ long long bin2d(const Grid2 &g, double radial, double azimuthal) {
    if (!isfinite(radial) || !isfinite(azimuthal)) return -1;
    if (!g.clamp_radial_outside &&
        (radial < g.r0 || radial > g.r1 || (radial == g.r1 && !g.clamp_radial_end)))
        return -1;
    double offset;
    if (g.clamp_azimuthal_outside) {
        offset = azimuthal - g.a0;
        const double span = g.a1 - g.a0;
        if (offset < 0.0) offset = 0.0;
        if (offset > span) offset = span;
    } else if (g.clamp_index_rounding) {
        const double wrapped = (azimuthal >= g.a0 && azimuthal < g.a1)
                                   ? azimuthal
                                   : g.a0 + rem_euclid_tau(azimuthal - g.a0);
        if (wrapped >= g.a1 && g.a1 - g.a0 < kTau) return -1;
        offset = wrapped - g.a0;
    } else {
        const double az = g.a0 + rem_euclid_tau(azimuthal - g.a0);
        if (az >= g.a1) return -1;
        offset = az - g.a0;
    }
    unsigned long long r = as_usize((radial - g.r0) / g.dr);
    unsigned long long a = as_usize(offset / g.da);
    if (g.clamp_radial_end || g.clamp_index_rounding || g.clamp_radial_outside)
        if (r > (unsigned long long)(g.nr - 1)) r = (unsigned long long)(g.nr - 1);
    if (g.clamp_index_rounding || g.clamp_azimuthal_outside)
        if (a > (unsigned long long)(g.na - 1)) a = (unsigned long long)(g.na - 1);
    if (r < (unsigned long long)g.nr && a < (unsigned long long)g.na)
        return (long long)(a * (unsigned long long)g.nr + r);
    return -1;
}

// Counting 2D (shared_grid.rs:57-61): the pixel centre's bin, weight 1.
__global__ void k_count2d(Grid2 g, const double *__restrict__ cr, const double *__restrict__ cc,
                          int64_t n, int32_t *__restrict__ count, int32_t *__restrict__ bin_of) {
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n;
         p += int64_t(gridDim.x) * blockDim.x) {
        const long long b = bin2d(g, cr[p], cc[p]);
        bin_of[p] = int32_t(b);
        count[p] = b >= 0;
    }
}

constexpr int kEnt2Cap = 128;   // entries of one pixel (fractional / pyFAI split)
constexpr int kRaster2Cap = 512; // cells of one pixel's pyFAI raster

struct Split2 {
    Grid2 g;
    int dim1, dim2;
    const double *rc, *ac, *cr, *cc;
};

// Adds w to bin in the pixel's list (repeated bins add up, shared_grid.rs).
__device__ __forceinline__ void ent_add(int *bins, double *ws, int &m, int bin, double w,
                                        int *overflow) {
    for (int k = 0; k < m; ++k)
        if (bins[k] == bin) {
            ws[k] += w;
            return;
        }
    if (m == kEnt2Cap) {
        atomicExch(overflow + 1, 1);
        return;
    }
    bins[m] = bin;
    ws[m] = w;
    ++m;
}

// line (pyfai_split.rs:146-168).
__device__ void pyfai_line(float *buffer, int stride, Pt start, Pt stop) {
    if (start.x == stop.x) return;
    const float slope = __double2float_rn((stop.y - start.y) / (stop.x - start.x));
    const float intercept = __double2float_rn(stop.y - double(slope) * stop.x);
    const double lo = fmin(start.x, stop.x), hi = fmax(start.x, stop.x);
    const double sign = stop.x > start.x ? 1.0 : -1.0;
    const unsigned long long rb = as_usize(floor(lo)), re = as_usize(ceil(hi));
    for (unsigned long long r = rb; r < re; ++r) {
        const double left = fmax(lo, double(r)), right = fmin(hi, double(r + 1));
        const float area = __double2float_rn(
            sign * (right - left) * (0.5 * double(slope) * (right + left) + double(intercept)));
        const float width = __double2float_rn(right - left);
        float remaining = fabsf(area);
        for (int a = 0; a < stride; ++a) {
            if (remaining <= 0.0f) break;
            const float increment = fminf(width, remaining);
            float *cell = buffer + int64_t(r) * stride + a;
            *cell = __fadd_rn(*cell, copysignf(increment, area));
            remaining = __fsub_rn(remaining, increment);
        }
    }
}

// pyfai_split::split (pyfai_split.rs:35-144) with corner sign +1. Returns the
// number of entries, -1 for None (fractional fallback).
__device__ int pyfai_split2(const Grid2 &g, Pt poly[4], int *bins, double *ws, float *buffer,
                            int *overflow) {
    const double canonical = (g.a0 >= -kPi && g.a1 <= kPi) ? -kPi
                             : (g.a0 >= 0.0 && g.a1 <= kTau) ? 0.0
                                                            : g.a0;
    const double offset = canonical + kPi;
    for (int i = 0; i < 4; ++i) poly[i].y = wrap_tau(poly[i].y - offset + kPi) - kPi;
    const Pt a = poly[0], b = poly[1], c = poly[2], d = poly[3];
    const double area = 1.0 * (0.5 * (c.x - a.x) * (d.y - b.y) - (c.y - a.y) * (d.x - b.x));
    if (area > 0.0) {
        for (int i = 0; i < 4; ++i)
            if (poly[i].y < 0.0) poly[i].y += kTau;
        double s = -0.0;
        for (int i = 0; i < 4; ++i) s += poly[i].y;
        if (s * 0.25 > kPi)
            for (int i = 0; i < 4; ++i) poly[i].y -= kTau;
    }
    for (int i = 0; i < 4; ++i) poly[i].y += offset;
    bool lr = true, hr = true, la = true, ha = true;
    for (int i = 0; i < 4; ++i) {
        lr &= poly[i].x < g.r0;
        hr &= poly[i].x > g.r1;
        la &= poly[i].y < g.a0;
        ha &= poly[i].y > g.a1;
    }
    if (lr || hr || la || ha) return 0;
    for (int i = 0; i < 4; ++i) {
        double x = poly[i].x, y = poly[i].y;
        x = x < g.r0 ? g.r0 : x;
        x = x > g.r1 ? g.r1 : x;
        y = y < g.a0 ? g.a0 : y;
        y = y > g.a1 ? g.a1 : y;
        poly[i].x = (x - g.r0) / g.dr;
        poly[i].y = (y - g.a0) / g.da;
    }
    double mr = INFINITY, ma = INFINITY;
    for (int i = 0; i < 4; ++i) {
        mr = fmin(mr, poly[i].x);
        ma = fmin(ma, poly[i].y);
    }
    const unsigned long long ir = as_usize(floor(mr)), ia = as_usize(floor(ma));
    for (int i = 0; i < 4; ++i) {
        poly[i].x -= double(ir);
        poly[i].y -= double(ia);
    }
    double xr = 0.0, xa = 0.0;
    for (int i = 0; i < 4; ++i) {
        xr = fmax(xr, poly[i].x);
        xa = fmax(xa, poly[i].y);
    }
    const unsigned long long nr = as_usize(ceil(xr)), na = as_usize(ceil(xa));
    if (nr == 0 || na == 0) return -1;
    if ((nr + 1) * (na + 1) > (unsigned long long)kRaster2Cap) {
        atomicExch(overflow + 1, 1);
        return 0;
    }
    const int stride = int(na + 1);
    for (int k = 0; k < int((nr + 1) * (na + 1)); ++k) buffer[k] = 0.0f;
    for (int i = 0; i < 4; ++i) pyfai_line(buffer, stride, poly[i], poly[(i + 1) & 3]);
    int m = 0;
    double total = 0.0;
    for (unsigned long long r = 0; r < nr; ++r)
        for (unsigned long long q = 0; q < na; ++q) {
            const double value = 1.0 * double(buffer[r * stride + q]);
            if (!isfinite(value)) return -1;
            if (value > 0.0 && ir + r < (unsigned long long)g.nr &&
                ia + q < (unsigned long long)g.na) {
                if (m == kEnt2Cap) {
                    atomicExch(overflow + 1, 1);
                    return 0;
                }
                bins[m] = int((ia + q) * (unsigned long long)g.nr + ir + r);
                ws[m] = value;
                total += value;
                ++m;
            }
        }
    if (total <= 0.0) return -1;
    for (int k = 0; k < m; ++k) ws[k] /= total;
    return m;
}

// split_polygon (shared_grid.rs:152-200).
__device__ int split_polygon2(const Grid2 &g, const Pt poly[4], double area, int *bins,
                              double *ws, int *overflow) {
    double rmn = INFINITY, rmx = -INFINITY;
    for (int i = 0; i < 4; ++i) {
        rmn = fmin(rmn, poly[i].x);
        rmx = fmax(rmx, poly[i].x);
    }
    long long rs = as_isize(floor((rmn - g.r0) / g.dr));
    if (rs < 0) rs = 0;
    long long re = as_isize(floor((rmx - g.r0) / g.dr));
    if (re > g.nr - 1) re = g.nr - 1;
    int m = 0;
    const double shifts[3] = {-kTau, 0.0, kTau};
    for (int sh = 0; sh < 3; ++sh) {
        Pt q[4];
        double amn = INFINITY, amx = -INFINITY;
        for (int i = 0; i < 4; ++i) {
            q[i].x = poly[i].x;
            q[i].y = poly[i].y + shifts[sh];
            amn = fmin(amn, q[i].y);
            amx = fmax(amx, q[i].y);
        }
        long long as_ = as_isize(floor((amn - g.a0) / g.da));
        if (as_ < 0) as_ = 0;
        long long ae = as_isize(floor((amx - g.a0) / g.da));
        if (ae > g.na - 1) ae = g.na - 1;
        for (long long ar = as_; ar <= ae; ++ar)
            for (long long rr = rs; rr <= re; ++rr) {
                const double r = g.r0 + double(rr) * g.dr;
                const double a = g.a0 + double(ar) * g.da;
                const double w = clipped_area(q, r, r + g.dr, a, a + g.da, overflow) / area;
                if (w > 0.0) ent_add(bins, ws, m, int(ar * g.nr + rr), w, overflow);
            }
    }
    return m;
}

// One pixel of shared_grid::build for pixel splitting (shared_grid.rs:62-117):
// -1 for a pixel sampled on the detector plane.
__device__ int split2_pixel(const Split2 &s, int64_t pixel, int *bins, double *ws, float *raster,
                            int *overflow) {
    const Grid2 &g = s.g;
    const int64_t w = s.dim2 + 1;
    const int64_t b0 = pixel / s.dim2 * w + pixel % s.dim2;
    const int64_t idx[4] = {b0, b0 + 1, b0 + w + 1, b0 + w};
    bool axis_on_edge = false, has_zero = false;
    double winding = 0.0;
    for (int i = 0; i < 4; ++i) {
        double delta = s.ac[idx[(i + 1) & 3]] - s.ac[idx[i]];
        delta = rem_euclid_tau(delta + kPi) - kPi;
        axis_on_edge |= fabs(delta) >= kPi - 64.0 * kEps;
        winding += delta;
        has_zero |= s.rc[idx[i]] == 0.0;
    }
    if (fabs(winding) > kPi || axis_on_edge || has_zero) return -1;
    if (g.pyfai) {
        Pt poly[4] = {{s.rc[idx[0]], s.ac[idx[0]]}, {s.rc[idx[3]], s.ac[idx[3]]},
                      {s.rc[idx[2]], s.ac[idx[2]]}, {s.rc[idx[1]], s.ac[idx[1]]}};
        const int m = pyfai_split2(g, poly, bins, ws, raster, overflow);
        if (m >= 0) return m;
    }
    const double center = g.a0 + rem_euclid_tau(s.cc[pixel] - g.a0);
    Pt poly[4];
    for (int i = 0; i < 4; ++i) {
        poly[i].x = s.rc[idx[i]];
        poly[i].y = center + rem_euclid_tau(s.ac[idx[i]] - center + kPi) - kPi;
    }
    const double area = fabs(polygon_area(poly, 4));
    if (area > 0.0) return split_polygon2(g, poly, area, bins, ws, overflow);
    const long long b = bin2d(g, s.cr[pixel], s.cc[pixel]);
    if (b < 0) return 0;
    bins[0] = int(b);
    ws[0] = 1.0;
    return 1;
}

// FILL = false: counts and lists the sampled pixels; true: writes entries.
template <bool FILL>
__global__ void __launch_bounds__(128)
    k_split2(Split2 s, const int64_t *__restrict__ off, int32_t *__restrict__ count,
             int32_t *__restrict__ sing, int32_t sing_cap, int32_t *__restrict__ n_sing,
             int32_t *__restrict__ cbin, double *__restrict__ cw, int32_t *__restrict__ cpix,
             int *overflow) {
    const int64_t n = int64_t(s.dim1) * s.dim2;
    int bins[kEnt2Cap];
    double ws[kEnt2Cap];
    float raster[kRaster2Cap];
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n;
         p += int64_t(gridDim.x) * blockDim.x) {
        const int m = split2_pixel(s, p, bins, ws, raster, overflow);
        if (FILL && m < 0) continue;  // sampled pixel, filled by k_sample2d_fill
        if (!FILL) {
            if (m < 0) {
                const int slot = atomicAdd(n_sing, 1);
                if (slot < sing_cap) sing[slot] = int32_t(p);
            }
            count[p] = m;  // -1 marks a sampled pixel until its count is known
            continue;
        }
        const int64_t o = off[p];
        for (int k = 0; k < m; ++k) {
            cbin[o + k] = bins[k];
            cw[o + k] = ws[k];
            cpix[o + k] = int32_t(p);
        }
    }
}

// sample_pixel (shared_grid.rs:202-232) for sampled pixel blockIdx.x of a
// batch: 128 x 128 x 4 detector-plane samples counted per grid bin.
__global__ void k_sample2d(GeomParams gp, Grid2 g, int dim2, const int32_t *__restrict__ sing,
                           int32_t *__restrict__ hits) {
    const int N = 128;
    const double off[4][2] = {{0.25, 0.5}, {0.5, 0.25}, {0.75, 0.5}, {0.5, 0.75}};
    const int32_t pixel = sing[blockIdx.x];
    int32_t *h = hits + int64_t(blockIdx.x) * g.nr * g.na;
    const int64_t row = pixel / dim2, col = pixel % dim2;
    for (int sm = threadIdx.x; sm < N * N * 4; sm += blockDim.x) {
        const int i = sm / (N * 4), j = (sm / 4) % N, o = sm & 3;
        const double d1 = double(row) + (double(i) + off[o][0]) / double(N);
        const double d2 = (double(col * N + j) + off[o][1]) / double(N);
        double r, az;
        radial_chi(gp, d1, d2, r, az);
        const long long b = bin2d(g, r, az);
        if (b >= 0) atomicAdd(&h[b], 1);
    }
}

// Entry count of each sampled pixel of a batch (bins with hits).
__global__ void k_sample2d_count(const int32_t *__restrict__ sing, int64_t nb,
                                 const int32_t *__restrict__ hits, int32_t *__restrict__ count) {
    const int32_t *h = hits + int64_t(blockIdx.x) * nb;
    int c = 0;
    for (int64_t b = threadIdx.x; b < nb; b += blockDim.x) c += h[b] != 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    __shared__ int wsum[32];
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int i = 0; i < int(blockDim.x + 31) / 32; ++i) t += wsum[i];
        count[sing[blockIdx.x]] = t;
    }
}

// Entries of each sampled pixel of a batch, bins ascending, weight hits/65536
// (the sum of hits samples of weight 2^-16, exact).
__global__ void k_sample2d_fill(const int32_t *__restrict__ sing, int64_t nb,
                                const int32_t *__restrict__ hits, const int64_t *__restrict__ off,
                                int32_t *__restrict__ cbin, double *__restrict__ cw,
                                int32_t *__restrict__ cpix) {
    if (threadIdx.x != 0) return;
    const int32_t pixel = sing[blockIdx.x];
    const int32_t *h = hits + int64_t(blockIdx.x) * nb;
    int64_t o = off[pixel];
    for (int64_t b = 0; b < nb; ++b)
        if (h[b]) {
            cbin[o] = int32_t(b);
            cw[o] = double(h[b]) / 65536.0;
            cpix[o] = pixel;
            ++o;
        }
}

// build_shared_grid_ss_csr through the exact counted path (supersampled.rs
// :1437-1477, :21-104, normalize_bins false): samples d1 = row + (i+.5)/n,
// d2 = ((col*n + j) + .5)/n, distinct grid bins in first-seen order, weight
// count / n^2.
__global__ void k_ss2d(GeomParams gp, Grid2 g, int dim1, int dim2, int n_ss,
                       const int64_t *__restrict__ off, int32_t *__restrict__ count,
                       int32_t *__restrict__ cbin, double *__restrict__ cw,
                       int32_t *__restrict__ cpix) {
    const int64_t n = int64_t(dim1) * dim2;
    int bins[kMaxSs * kMaxSs], cnt[kMaxSs * kMaxSs];
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < n;
         p += int64_t(gridDim.x) * blockDim.x) {
        const int64_t row = p / dim2, col = p % dim2;
        int nc = 0;
        for (int i = 0; i < n_ss; ++i) {
            const double d1 = double(row) + (double(i) + 0.5) / double(n_ss);
            for (int j = 0; j < n_ss; ++j) {
                const double d2 = (double(col * n_ss + j) + 0.5) / double(n_ss);
                double r, az;
                radial_chi(gp, d1, d2, r, az);
                const long long b = bin2d(g, r, az);
                if (b < 0) continue;
                int f = -1;
                for (int q = 0; q < nc; ++q)
                    if (bins[q] == int(b)) {
                        f = q;
                        break;
                    }
                if (f < 0) {
                    bins[nc] = int(b);
                    cnt[nc++] = 1;
                } else {
                    cnt[f]++;
                }
            }
        }
        if (!off) {
            count[p] = nc;
            continue;
        }
        const int64_t o = off[p];
        const double denom = double(n_ss * n_ss);
        for (int q = 0; q < nc; ++q) {
            cbin[o + q] = bins[q];
            cw[o + q] = double(cnt[q]) / denom;
            cpix[o + q] = int32_t(p);
        }
    }
}

// ------------------------------------------------ ordered transpose

__global__ void k_chunk_count(const int32_t *__restrict__ cbin, const int32_t *__restrict__ cpix,
                              int64_t ncoo, int chunk, int nb, int32_t *__restrict__ m) {
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < ncoo;
         e += int64_t(gridDim.x) * blockDim.x) {
        int c = cpix[e] / chunk;
        atomicAdd(&m[int64_t(c) * nb + cbin[e]], 1);
    }
}

// Exclusive scan of every bin's column down the chunks; totals per bin.
__global__ void k_column_scan(int32_t *__restrict__ m, int n_chunks, int nb,
                              int64_t *__restrict__ totals) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    int32_t run = 0;
    for (int c = 0; c < n_chunks; ++c) {
        int64_t k = int64_t(c) * nb + b;
        int32_t v = m[k];
        m[k] = run;
        run += v;
    }
    totals[b] = run;
}

// One warp per chunk: walk the chunk's contributions in pixel order and place
// each at row_ptr[bin] + cursor(chunk, bin) + rank among equal bins of lower
// lanes. Cursors of a chunk are touched by its warp only.
__global__ void k_place(const int32_t *__restrict__ cbin, const double *__restrict__ cw,
                        const int32_t *__restrict__ cpix, const int64_t *__restrict__ pix_off,
                        int64_t n_pixels, int chunk, int n_chunks, int nb,
                        int32_t *__restrict__ m, const int64_t *__restrict__ row_ptr,
                        int32_t *__restrict__ col, double *__restrict__ w) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= n_chunks) return;
    int64_t p0 = int64_t(warp) * chunk;
    int64_t p1 = p0 + chunk < n_pixels ? p0 + chunk : n_pixels;
    int64_t e0 = pix_off[p0], e1 = pix_off[p1];
    int32_t *cur = m + int64_t(warp) * nb;
    unsigned lt = (1u << lane) - 1u;
    for (int64_t base = e0; base < e1; base += 32) {
        int64_t e = base + lane;
        bool act = e < e1;
        unsigned active = __ballot_sync(0xffffffffu, act);
        if (!act) continue;
        int b = cbin[e];
        unsigned peers = __match_any_sync(active, b);
        int rank = __popc(peers & lt);
        int leader = __ffs(peers) - 1;
        int32_t c0 = cur[b];
        __syncwarp(active);
        int64_t slot = row_ptr[b] + c0 + rank;
        col[slot] = cpix[e];
        w[slot] = cw[e];
        if (lane == leader) cur[b] = c0 + __popc(peers);
        __syncwarp(active);
    }
}

// ------------------------------------------------------ compaction

__global__ void k_keep(const int32_t *__restrict__ col, int64_t nnz, const uint8_t *__restrict__ mask,
                       int32_t *__restrict__ keep) {
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < nnz;
         e += int64_t(gridDim.x) * blockDim.x)
        keep[e] = mask[col[e]] == 0;
}

__global__ void k_compact(const int32_t *__restrict__ col, const double *__restrict__ w,
                          int64_t nnz, const int32_t *__restrict__ keep,
                          const int64_t *__restrict__ pos, int32_t *__restrict__ ocol,
                          double *__restrict__ ow) {
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < nnz;
         e += int64_t(gridDim.x) * blockDim.x)
        if (keep[e]) {
            ocol[pos[e]] = col[e];
            ow[pos[e]] = w[e];
        }
}

__global__ void k_compact_rows(const int64_t *__restrict__ row_ptr, int64_t n_rows,
                               const int64_t *__restrict__ pos, int64_t nnz,
                               int64_t total, int64_t *__restrict__ out) {
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r <= n_rows;
         r += int64_t(gridDim.x) * blockDim.x) {
        int64_t k = row_ptr[r];
        out[r] = k < nnz ? pos[k] : total;
    }
}

// normalization::<false> (prepared.rs:229-262) via row() (prepared.rs:1011):
// n = n + w*x, strictly sequential per row.
__global__ void k_denominators(const int64_t *__restrict__ row_ptr, int64_t n_rows,
                               const int32_t *__restrict__ col, const double *__restrict__ w,
                               const double *__restrict__ norm, double *__restrict__ den) {
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n_rows;
         r += int64_t(gridDim.x) * blockDim.x) {
        double n = 0.0;
        for (int64_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) n = n + w[k] * norm[col[k]];
        den[r] = n;
    }
}

unsigned grid_for(int64_t n, int threads = 256) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 64) b = 148 * 64;
    return unsigned(b);
}

template <typename T>
std::vector<T> to_host(const T *d, size_t n, cudaStream_t s) {
    std::vector<T> h(n);
    if (n) DG_CUDA(cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    return h;
}

// IntegrationGrid2d::new radial validity (grid.rs:49-105), as used for the
// 1D sampling grid of singular pixels.
bool grid_ok(double lo, double hi, int64_t n) {
    double step = (hi - lo) / double(n);
    if (!std::isfinite(lo) || !std::isfinite(hi) || !std::isfinite(step) || step <= 0.0 ||
        lo + step == lo || hi - step == hi)
        return false;
    return lo >= 0.0;
}

// Pixel-major contributions -> CSR rows, sort-free and stable.
void transpose(const int32_t *cbin, const double *cw, const int32_t *cpix,
               const int64_t *pix_off, int64_t n_pixels, int64_t ncoo, int nb,
               cudaStream_t s, DeviceCsr &out) {
    // Chunk size: keep the (chunk x bin) cursor matrix under 64 Mi entries.
    int64_t chunk = 1024;
    while ((n_pixels + chunk - 1) / chunk * int64_t(nb) > (int64_t(1) << 26)) chunk *= 2;
    int n_chunks = int((n_pixels + chunk - 1) / chunk);
    DeviceArray<int32_t> m;
    m.alloc(size_t(n_chunks) * nb);
    DG_CUDA(cudaMemsetAsync(m.ptr, 0, m.bytes(), s));
    k_chunk_count<<<grid_for(ncoo), 256, 0, s>>>(cbin, cpix, ncoo, int(chunk), nb, m.ptr);
    DG_CUDA(cudaGetLastError());
    DeviceArray<int64_t> totals;
    totals.alloc(size_t(nb) + 1);
    k_column_scan<<<(nb + 255) / 256, 256, 0, s>>>(m.ptr, n_chunks, nb, totals.ptr);
    DG_CUDA(cudaGetLastError());
    out.n_rows = nb;
    out.nnz = ncoo;
    out.row_ptr.alloc(size_t(nb) + 1);
    DeviceArray<unsigned char> tmp;
    tmp.alloc(scan_temp_bytes(nb + 1));
    DG_CUDA(cudaMemsetAsync(totals.ptr + nb, 0, sizeof(int64_t), s));
    exclusive_scan_i64(totals.ptr, out.row_ptr.ptr, nb + 1, tmp.ptr, s);
    out.col.alloc(size_t(ncoo));
    out.w.alloc(size_t(ncoo));
    unsigned blocks = unsigned((int64_t(n_chunks) * 32 + 255) / 256);
    k_place<<<blocks, 256, 0, s>>>(cbin, cw, cpix, pix_off, n_pixels, int(chunk), n_chunks, nb,
                                   m.ptr, out.row_ptr.ptr, out.col.ptr, out.w.ptr);
    DG_CUDA(cudaGetLastError());
    DG_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

namespace {

// IntegrationGrid2d::new (grid.rs:49-105) on host values; the azimuthal start
// is corrected into [-pi, pi) when it lies outside +-2pi.
void grid2_new(int nr, int na, double r0, double r1, double a0, double a1, Grid2 &g) {
    const double lo[2] = {r0, a0}, hi[2] = {r1, a1};
    const int cnt[2] = {nr, na};
    const char *name[2] = {"radial", "azimuthal"};
    for (int k = 0; k < 2; ++k) {
        const double step = (hi[k] - lo[k]) / double(cnt[k]);
        if (!std::isfinite(lo[k]) || !std::isfinite(hi[k]) || !std::isfinite(step) ||
            step <= 0.0 || lo[k] + step == lo[k] || hi[k] - step == hi[k])
            fail(DG_INVALID_INPUT, std::string(name[k]) +
                                       " range must have finite, increasing, resolvable bin edges");
    }
    if (r0 < 0.0) fail(DG_INVALID_INPUT, "radial range must be nonnegative");
    if (a1 - a0 > kTau + 1e-12)
        fail(DG_INVALID_INPUT, "azimuthal span must be at most 2pi (one full turn)");
    if (!(a0 >= -kTau && a0 <= kTau)) {
        double start = std::fmod(a0, kTau);
        if (start < 0.0) start += kTau;
        if (start >= kPi) start -= kTau;
        const double span = a1 - a0;
        a0 = start;
        a1 = start + span;
    }
    g = Grid2{};
    g.nr = nr;
    g.na = na;
    g.r0 = r0;
    g.r1 = r1;
    g.a0 = a0;
    g.a1 = a1;
    g.dr = (r1 - r0) / double(nr);
    g.da = (a1 - a0) / double(na);
}

// 2D tables: the grid of prepare_cuda2d (cuda.rs:1111-1157; edges and clamps
// of methods.rs:365-388 and grid.rs:579-624, :700-755, :975-1028), then
// shared_grid::build (shared_grid.rs:13-150) or the supersampled counted
// table, transposed into rows a * n_radial + r.
void build_table_2d(const dg_geometry &geom, const dg_method &m, int32_t dim1, int32_t dim2,
                    int32_t nr, int32_t na, const double *azimuthal_range, cudaStream_t s,
                    BuildResult &out) {
    GeomParams gp = make_geom_params(geom, m);
    const int64_t npix = int64_t(dim1) * dim2;
    const int64_t ncorner = int64_t(dim1 + 1) * (dim2 + 1);
    const int64_t nb = int64_t(nr) * na;
    if (nb > INT32_MAX) fail(DG_INVALID_INPUT, "2D bin count must be in 1..=2147483647");
    const double eps = DBL_EPSILON;
    if (azimuthal_range) {
        Grid2 probe;
        grid2_new(nr, na, 0.0, 1.0, azimuthal_range[0], azimuthal_range[1], probe);
    }
    if (m.kind == DG_METHOD_SUPERSAMPLED && (m.n_ss < 1 || m.n_ss > kMaxSs))
        fail(DG_UNSUPPORTED, "supersampling factor must be between 1 and 8");

    DeviceArray<double> cr, cc, rc, ac;
    cr.alloc(npix);
    cc.alloc(npix);
    rc.alloc(ncorner);
    ac.alloc(ncorner);
    out.norm.alloc(npix);
    k_centres<<<grid_for(npix), 256, 0, s>>>(gp, dim1, dim2, cr.ptr, cc.ptr, out.norm.ptr);
    k_corners<<<grid_for(ncorner), 256, 0, s>>>(gp, dim1, dim2, rc.ptr, ac.ptr);
    DG_CUDA(cudaGetLastError());
    DeviceArray<unsigned long long> mm;
    mm.alloc(12);
    unsigned long long init[12];
    for (int i = 0; i < 12; i += 2) {
        init[i] = ~0ull;
        init[i + 1] = 0ull;
    }
    DG_CUDA(cudaMemcpyAsync(mm.ptr, init, sizeof init, cudaMemcpyHostToDevice, s));
    k_minmax<<<grid_for(npix), 256, 0, s>>>(cr.ptr, npix, mm.ptr);
    k_minmax<<<grid_for(npix), 256, 0, s>>>(cc.ptr, npix, mm.ptr + 2);
    k_minmax<<<grid_for(ncorner), 256, 0, s>>>(rc.ptr, ncorner, mm.ptr + 4);
    k_minmax<<<grid_for(ncorner), 256, 0, s>>>(ac.ptr, ncorner, mm.ptr + 6);
    if (m.kind == DG_METHOD_SUPERSAMPLED)
        k_hull_minmax<<<grid_for(2 * (int64_t(dim1) + dim2) * m.n_ss), 256, 0, s>>>(
            gp, dim1, dim2, m.n_ss, mm.ptr + 8, mm.ptr + 10);
    DG_CUDA(cudaGetLastError());
    auto k = to_host(mm.ptr, 12, s);
    double ext[12];
    for (int i = 0; i < 12; ++i) ext[i] = key_to_double(k[size_t(i)]);
    // ext: centre radial lo/hi, centre chi lo/hi, corner radial lo/hi, corner
    // chi lo/hi, hull radial lo/hi, hull chi lo/hi.
    double r0, r1, a0, a1;
    if (m.has_radial_range) {
        r0 = m.radial_min;
        r1 = m.radial_max;
    } else if (m.kind == DG_METHOD_COUNTING) {
        r0 = ext[0];
        r1 = ext[1] + 10.0 * eps;
    } else if (m.kind == DG_METHOD_PIXEL_SPLIT) {
        r0 = ext[4];
        r1 = ext[5] + 10.0 * eps;
    } else if (m.kind == DG_METHOD_PYFAI_FULL) {
        r0 = std::fmax(ext[4], 0.0);
        r1 = ext[5] * (1.0 + double(FLT_EPSILON));
    } else {
        r0 = std::fmin(ext[0], ext[8]);
        r1 = std::fmax(ext[1], ext[9]) + 3.0 * eps;
    }
    if (azimuthal_range) {
        a0 = azimuthal_range[0];
        a1 = azimuthal_range[1];
    } else if (m.kind == DG_METHOD_PYFAI_FULL) {
        a0 = -kPi;
        a1 = kPi;
    } else {
        if (m.kind == DG_METHOD_COUNTING) {
            a0 = ext[2];
            a1 = ext[3] + 10.0 * eps;
        } else if (m.kind == DG_METHOD_SUPERSAMPLED) {
            a0 = std::fmin(ext[2], ext[10]);
            a1 = std::fmax(ext[3], ext[11]) + 3.0 * eps;
        } else {
            a0 = ext[6];
            a1 = ext[7] + 10.0 * eps;
        }
        if (!(a1 - a0 > 1e-12)) {
            a0 = -kPi;
            a1 = kPi;
        }
    }
    Grid2 g;
    grid2_new(nr, na, r0, r1, a0, a1, g);
    g.clamp_index_rounding = 1;
    if (m.kind == DG_METHOD_PYFAI_FULL) g.pyfai = 1;
    else if (!m.has_radial_range && m.kind == DG_METHOD_COUNTING) g.clamp_radial_end = 1;
    else if (!m.has_radial_range && m.kind == DG_METHOD_SUPERSAMPLED) g.clamp_radial_outside = 1;
    if (m.kind == DG_METHOD_SUPERSAMPLED && !azimuthal_range) g.clamp_azimuthal_outside = 1;
    out.hist_min = g.r0;
    out.hist_step = g.dr;
    out.radial_centres.resize(size_t(nr));
    for (int i = 0; i < nr; ++i) out.radial_centres[size_t(i)] = g.r0 + (double(i) + 0.5) * g.dr;
    out.azimuthal_centres.resize(size_t(na));
    for (int i = 0; i < na; ++i)
        out.azimuthal_centres[size_t(i)] = g.a0 + (double(i) + 0.5) * g.da;

    DeviceArray<int32_t> count;
    count.alloc(npix + 1);
    DG_CUDA(cudaMemsetAsync(count.ptr, 0, count.bytes(), s));
    DeviceArray<int64_t> off;
    off.alloc(npix + 1);
    DeviceArray<unsigned char> scan_tmp;
    scan_tmp.alloc(scan_temp_bytes(npix + 1));
    DeviceArray<int32_t> cbin, cpix;
    DeviceArray<double> cw;
    DeviceArray<int> flags;
    flags.alloc(2);
    DG_CUDA(cudaMemsetAsync(flags.ptr, 0, flags.bytes(), s));
    auto scan_counts = [&]() -> int64_t {
        exclusive_scan_i32_to_i64(count.ptr, off.ptr, npix + 1, scan_tmp.ptr, s);
        int64_t total = 0;
        DG_CUDA(cudaMemcpyAsync(&total, off.ptr + npix, sizeof total, cudaMemcpyDeviceToHost, s));
        DG_CUDA(cudaStreamSynchronize(s));
        if (total > int64_t(INT32_MAX) - 128)
            fail(DG_UNSUPPORTED, "lookup table of " + std::to_string(total) +
                                     " entries exceeds 32-bit indexing");
        cbin.alloc(size_t(total));
        cpix.alloc(size_t(total));
        cw.alloc(size_t(total));
        return total;
    };
    int64_t ncoo = 0;
    if (m.kind == DG_METHOD_COUNTING) {
        DeviceArray<int32_t> bin_of;
        bin_of.alloc(npix);
        k_count2d<<<grid_for(npix), 256, 0, s>>>(g, cr.ptr, cc.ptr, npix, count.ptr, bin_of.ptr);
        DG_CUDA(cudaGetLastError());
        ncoo = scan_counts();
        k_count1d_fill<<<grid_for(npix), 256, 0, s>>>(bin_of.ptr, npix, off.ptr, cbin.ptr,
                                                      cw.ptr, cpix.ptr);
        DG_CUDA(cudaGetLastError());
    } else if (m.kind == DG_METHOD_SUPERSAMPLED) {
        k_ss2d<<<grid_for(npix, 128), 128, 0, s>>>(gp, g, dim1, dim2, m.n_ss, nullptr, count.ptr,
                                                   nullptr, nullptr, nullptr);
        DG_CUDA(cudaGetLastError());
        ncoo = scan_counts();
        k_ss2d<<<grid_for(npix, 128), 128, 0, s>>>(gp, g, dim1, dim2, m.n_ss, off.ptr, count.ptr,
                                                   cbin.ptr, cw.ptr, cpix.ptr);
        DG_CUDA(cudaGetLastError());
    } else {
        Split2 sp{};
        sp.g = g;
        sp.dim1 = dim1;
        sp.dim2 = dim2;
        sp.rc = rc.ptr;
        sp.ac = ac.ptr;
        sp.cr = cr.ptr;
        sp.cc = cc.ptr;
        const int32_t sing_cap = 1 << 16;
        DeviceArray<int32_t> sing, n_sing;
        sing.alloc(sing_cap);
        n_sing.alloc(1);
        DG_CUDA(cudaMemsetAsync(n_sing.ptr, 0, sizeof(int32_t), s));
        k_split2<false><<<grid_for(npix, 128), 128, 0, s>>>(sp, nullptr, count.ptr, sing.ptr,
                                                             sing_cap, n_sing.ptr, nullptr,
                                                             nullptr, nullptr, flags.ptr);
        DG_CUDA(cudaGetLastError());
        const int32_t ns = to_host(n_sing.ptr, 1, s)[0];
        if (ns > sing_cap) fail(DG_UNSUPPORTED, "too many singular pixels for sampling");
        out.singular_pixels = ns;
        // Sampled pixels in batches, each with a hit count per grid bin; the
        // fill below samples them again (integer counts, order-independent).
        const int64_t batch = std::max<int64_t>(1, std::min<int64_t>(64, (int64_t(1) << 28) / nb));
        DeviceArray<int32_t> hits;
        if (ns > 0) {
            std::vector<int32_t> hs = to_host(sing.ptr, size_t(ns), s);
            std::sort(hs.begin(), hs.end());
            DG_CUDA(cudaMemcpyAsync(sing.ptr, hs.data(), hs.size() * 4, cudaMemcpyHostToDevice, s));
            hits.alloc(size_t(std::min<int64_t>(batch, ns) * nb));
            for (int64_t b0 = 0; b0 < ns; b0 += batch) {
                const int nbat = int(std::min<int64_t>(batch, ns - b0));
                DG_CUDA(cudaMemsetAsync(hits.ptr, 0, size_t(nbat) * nb * 4, s));
                k_sample2d<<<nbat, 256, 0, s>>>(gp, g, dim2, sing.ptr + b0, hits.ptr);
                k_sample2d_count<<<nbat, 256, 0, s>>>(sing.ptr + b0, nb, hits.ptr, count.ptr);
                DG_CUDA(cudaGetLastError());
            }
        }
        ncoo = scan_counts();
        k_split2<true><<<grid_for(npix, 128), 128, 0, s>>>(sp, off.ptr, count.ptr, nullptr, 0,
                                                            nullptr, cbin.ptr, cw.ptr, cpix.ptr,
                                                            flags.ptr);
        DG_CUDA(cudaGetLastError());
        for (int64_t b0 = 0; b0 < ns; b0 += batch) {
            const int nbat = int(std::min<int64_t>(batch, ns - b0));
            DG_CUDA(cudaMemsetAsync(hits.ptr, 0, size_t(nbat) * nb * 4, s));
            k_sample2d<<<nbat, 256, 0, s>>>(gp, g, dim2, sing.ptr + b0, hits.ptr);
            k_sample2d_fill<<<nbat, 32, 0, s>>>(sing.ptr + b0, nb, hits.ptr, off.ptr, cbin.ptr,
                                                cw.ptr, cpix.ptr);
            DG_CUDA(cudaGetLastError());
        }
    }
    int hflags[2] = {0, 0};
    DG_CUDA(cudaMemcpyAsync(hflags, flags.ptr, sizeof hflags, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    if (hflags[0]) fail(DG_UNSUPPORTED, "polygon clipping exceeded its vertex capacity");
    if (hflags[1])
        fail(DG_UNSUPPORTED, "a pixel covers more 2D bins than the builder's per-pixel capacity");
    transpose(cbin.ptr, cw.ptr, cpix.ptr, off.ptr, npix, ncoo, int(nb), s, out.full);
}

}  // namespace

void build_table(const dg_geometry &geom, const dg_method &m, int32_t dim1, int32_t dim2,
                 int32_t n_radial, int32_t n_azimuthal, const double *azimuthal_range,
                 cudaStream_t s, BuildResult &out) {
    if (n_azimuthal != 0) {
        build_table_2d(geom, m, dim1, dim2, n_radial, n_azimuthal, azimuthal_range, s, out);
        return;
    }
    GeomParams g = make_geom_params(geom, m);
    const int64_t npix = int64_t(dim1) * dim2;
    const int64_t ncorner = int64_t(dim1 + 1) * (dim2 + 1);
    const int nb = n_radial;

    DeviceArray<double> cr, cc;
    cr.alloc(npix);
    cc.alloc(npix);
    out.norm.alloc(npix);
    k_centres<<<grid_for(npix), 256, 0, s>>>(g, dim1, dim2, cr.ptr, cc.ptr, out.norm.ptr);
    DG_CUDA(cudaGetLastError());

    DeviceArray<int32_t> count;
    count.alloc(npix + 1);
    DG_CUDA(cudaMemsetAsync(count.ptr, 0, count.bytes(), s));
    DeviceArray<int64_t> off;
    off.alloc(npix + 1);
    DeviceArray<unsigned char> scan_tmp;
    scan_tmp.alloc(scan_temp_bytes(npix + 1));
    DeviceArray<int32_t> cbin, cpix;
    DeviceArray<double> cw;
    DeviceArray<unsigned long long> mm;
    mm.alloc(4);
    const unsigned long long init[4] = {~0ull, 0ull, ~0ull, 0ull};
    DG_CUDA(cudaMemcpyAsync(mm.ptr, init, sizeof init, cudaMemcpyHostToDevice, s));
    DeviceArray<int> flags;
    flags.alloc(2);
    DG_CUDA(cudaMemsetAsync(flags.ptr, 0, flags.bytes(), s));

    auto scan_counts = [&]() -> int64_t {
        exclusive_scan_i32_to_i64(count.ptr, off.ptr, npix + 1, scan_tmp.ptr, s);
        int64_t total = 0;
        DG_CUDA(cudaMemcpyAsync(&total, off.ptr + npix, sizeof total, cudaMemcpyDeviceToHost, s));
        DG_CUDA(cudaStreamSynchronize(s));
        if (total > int64_t(INT32_MAX) - 128)
            fail(DG_UNSUPPORTED, "lookup table of " + std::to_string(total) +
                                     " entries exceeds 32-bit indexing");
        cbin.alloc(size_t(total));
        cpix.alloc(size_t(total));
        cw.alloc(size_t(total));
        return total;
    };

    int64_t ncoo = 0;
    const double eps = DBL_EPSILON;
    if (m.kind == DG_METHOD_PIXEL_SPLIT) {
        DeviceArray<double> rc, ac;
        rc.alloc(ncorner);
        ac.alloc(ncorner);
        k_corners<<<grid_for(ncorner), 256, 0, s>>>(g, dim1, dim2, rc.ptr, ac.ptr);
        DG_CUDA(cudaGetLastError());
        double mn, step;
        int clamp_low;
        if (m.has_radial_range) {
            // min_max_step_from_range (histogram.rs:184-188).
            double mx = m.radial_max + 10.0 * eps;
            mn = m.radial_min;
            step = (mx - mn) / double(nb);
            clamp_low = 0;
        } else {
            // build_lut1d_ps_csr (pixel_split.rs:402-405): corner min/max.
            k_minmax<<<grid_for(ncorner), 256, 0, s>>>(rc.ptr, ncorner, mm.ptr);
            DG_CUDA(cudaGetLastError());
            auto k = to_host(mm.ptr, 2, s);
            mn = key_to_double(k[0]);
            double mx = key_to_double(k[1]);
            mx += 10.0 * eps;
            step = (mx - mn) / double(nb);
            clamp_low = 1;
        }
        out.hist_min = mn;
        out.hist_step = step;
        Ps1d a{};
        a.g = g;
        a.dim1 = dim1;
        a.dim2 = dim2;
        a.n = nb;
        a.min = mn;
        a.step = step;
        a.r1 = mn + double(nb) * step;
        a.have_grid = grid_ok(mn, a.r1, nb);
        a.clamp_low = clamp_low;
        a.rc = rc.ptr;
        a.ac = ac.ptr;
        a.cr = cr.ptr;
        a.cc = cc.ptr;
        const int32_t sing_cap = 1 << 16;
        DeviceArray<int32_t> sing, n_sing;
        sing.alloc(sing_cap);
        n_sing.alloc(1);
        DG_CUDA(cudaMemsetAsync(n_sing.ptr, 0, sizeof(int32_t), s));
        k_ps1d_count<<<grid_for(npix, 128), 128, 0, s>>>(a, count.ptr, sing.ptr, sing_cap,
                                                         n_sing.ptr, flags.ptr);
        DG_CUDA(cudaGetLastError());
        DeviceArray<unsigned long long> guard;
        guard.alloc(1);
        DG_CUDA(cudaMemsetAsync(guard.ptr, 0, sizeof(unsigned long long), s));
        k_guard<<<grid_for(ncorner), 256, 0, s>>>(rc.ptr, ncorner, mn, step, guard.ptr);
        DG_CUDA(cudaGetLastError());
        int32_t ns = to_host(n_sing.ptr, 1, s)[0];
        out.guard_corners = int64_t(to_host(guard.ptr, 1, s)[0]);
        if (ns > sing_cap) fail(DG_UNSUPPORTED, "too many singular pixels for sampling");
        out.singular_pixels = ns;
        DeviceArray<int32_t> hits, slot;
        if (ns > 0) {
            // Sort the singular list so slots are deterministic.
            std::vector<int32_t> hs = to_host(sing.ptr, size_t(ns), s);
            std::sort(hs.begin(), hs.end());
            DG_CUDA(cudaMemcpyAsync(sing.ptr, hs.data(), hs.size() * 4, cudaMemcpyHostToDevice, s));
            hits.alloc(size_t(ns) * nb);
            DG_CUDA(cudaMemsetAsync(hits.ptr, 0, hits.bytes(), s));
            k_sample<<<ns, 256, 0, s>>>(g, dim2, sing.ptr, nb, mn, a.r1, clamp_low, hits.ptr);
            DG_CUDA(cudaGetLastError());
            k_sample_count<<<ns, 256, 0, s>>>(sing.ptr, nb, hits.ptr, count.ptr);
            DG_CUDA(cudaGetLastError());
            std::vector<int32_t> hslot(size_t(npix), -1);
            for (int32_t i = 0; i < ns; ++i) hslot[size_t(hs[size_t(i)])] = i;
            slot.alloc(size_t(npix));
            DG_CUDA(cudaMemcpyAsync(slot.ptr, hslot.data(), size_t(npix) * 4,
                                    cudaMemcpyHostToDevice, s));
            DG_CUDA(cudaStreamSynchronize(s));
        }
        ncoo = scan_counts();
        k_ps1d_fill<<<grid_for(npix, 128), 128, 0, s>>>(a, off.ptr, ns ? slot.ptr : nullptr,
                                                        hits.ptr, cbin.ptr, cw.ptr, cpix.ptr,
                                                        flags.ptr);
        DG_CUDA(cudaGetLastError());
    } else if (m.kind == DG_METHOD_COUNTING) {
        double mn, mx, step;
        if (m.has_radial_range) {
            mx = m.radial_max + 10.0 * eps;
            mn = m.radial_min;
            step = (mx - mn) / double(nb);
        } else {
            // min_max_step (histogram.rs:191-196) over pixel centres.
            k_minmax<<<grid_for(npix), 256, 0, s>>>(cr.ptr, npix, mm.ptr);
            DG_CUDA(cudaGetLastError());
            auto k = to_host(mm.ptr, 2, s);
            mn = key_to_double(k[0]);
            mx = key_to_double(k[1]) + 10.0 * eps;
            step = (mx - mn) / double(nb);
        }
        out.hist_min = mn;
        out.hist_step = step;
        DeviceArray<int32_t> bin_of;
        bin_of.alloc(npix);
        k_count1d<<<grid_for(npix), 256, 0, s>>>(cr.ptr, npix, mn, mx, step, nb,
                                                 m.has_radial_range, count.ptr, bin_of.ptr);
        DG_CUDA(cudaGetLastError());
        ncoo = scan_counts();
        k_count1d_fill<<<grid_for(npix), 256, 0, s>>>(bin_of.ptr, npix, off.ptr, cbin.ptr,
                                                      cw.ptr, cpix.ptr);
        DG_CUDA(cudaGetLastError());
    } else if (m.kind == DG_METHOD_SUPERSAMPLED) {
        if (m.n_ss < 1 || m.n_ss > kMaxSs)
            fail(DG_UNSUPPORTED, "supersampling factor must be between 1 and 8");
        Ss1d a{};
        a.g = g;
        a.dim1 = dim1;
        a.dim2 = dim2;
        a.n_ss = m.n_ss;
        a.nb = nb;
        a.has_range = m.has_radial_range;
        if (m.has_radial_range) {
            a.max = m.radial_max + 10.0 * eps;
            a.min = m.radial_min;
            a.step = (a.max - a.min) / double(nb);
        } else {
            // ss_tth_min_max_step (histogram.rs:151-166): centres and hull.
            k_minmax<<<grid_for(npix), 256, 0, s>>>(cr.ptr, npix, mm.ptr);
            k_hull_minmax<<<grid_for(2 * (int64_t(dim1) + dim2) * m.n_ss), 256, 0, s>>>(
                g, dim1, dim2, m.n_ss, mm.ptr + 2, nullptr);
            DG_CUDA(cudaGetLastError());
            auto k = to_host(mm.ptr, 4, s);
            double c_lo = key_to_double(k[0]), c_hi = key_to_double(k[1]);
            double h_lo = key_to_double(k[2]), h_hi = key_to_double(k[3]);
            a.min = h_lo < c_lo ? h_lo : c_lo;
            a.max = (h_hi > c_hi ? h_hi : c_hi) + 3.0 * eps;
            a.step = (a.max - a.min) / double(nb);
        }
        out.hist_min = a.min;
        out.hist_step = a.step;
        k_ss1d<<<grid_for(npix, 128), 128, 0, s>>>(a, nullptr, count.ptr, nullptr, nullptr,
                                                   nullptr);
        DG_CUDA(cudaGetLastError());
        ncoo = scan_counts();
        k_ss1d<<<grid_for(npix, 128), 128, 0, s>>>(a, off.ptr, count.ptr, cbin.ptr, cw.ptr,
                                                   cpix.ptr);
        DG_CUDA(cudaGetLastError());
    } else if (m.kind == DG_METHOD_PYFAI_FULL) {
        DeviceArray<double> rc, ac;
        rc.alloc(ncorner);
        ac.alloc(ncorner);
        k_corners<<<grid_for(ncorner), 256, 0, s>>>(g, dim1, dim2, rc.ptr, ac.ptr);
        DG_CUDA(cudaGetLastError());
        Pf1d a{};
        a.dim1 = dim1;
        a.dim2 = dim2;
        a.n = nb;
        if (m.has_radial_range) {
            // build_lut1d_pyfai_csr takes an explicit range as the edges.
            a.r0 = m.radial_min;
            a.r1 = m.radial_max;
        } else {
            // pyfai_radial_range (pyfai_1d.rs:36-46).
            k_minmax<<<grid_for(ncorner), 256, 0, s>>>(rc.ptr, ncorner, mm.ptr);
            DG_CUDA(cudaGetLastError());
            auto k = to_host(mm.ptr, 2, s);
            a.r0 = std::fmax(key_to_double(k[0]), 0.0);
            a.r1 = key_to_double(k[1]) * (1.0 + double(FLT_EPSILON));
        }
        if (!grid_ok(a.r0, a.r1, nb))
            fail(DG_INVALID_INPUT, "radial range must have finite, increasing, resolvable, "
                                   "nonnegative bin edges for pyfai_full");
        out.hist_min = a.r0;
        out.hist_step = (a.r1 - a.r0) / double(nb);
        a.rc = rc.ptr;
        a.ac = ac.ptr;
        const int32_t sing_cap = 1 << 16;
        DeviceArray<int32_t> sing, n_sing;
        sing.alloc(sing_cap);
        n_sing.alloc(1);
        DG_CUDA(cudaMemsetAsync(n_sing.ptr, 0, sizeof(int32_t), s));
        k_pf1d_count<<<grid_for(npix, 128), 128, 0, s>>>(a, count.ptr, sing.ptr, sing_cap,
                                                         n_sing.ptr, flags.ptr);
        DG_CUDA(cudaGetLastError());
        const int32_t ns = to_host(n_sing.ptr, 1, s)[0];
        if (ns > sing_cap) fail(DG_UNSUPPORTED, "too many singular pixels for sampling");
        out.singular_pixels = ns;
        DeviceArray<int32_t> hits, slot;
        if (ns > 0) {
            std::vector<int32_t> hs = to_host(sing.ptr, size_t(ns), s);
            std::sort(hs.begin(), hs.end());
            DG_CUDA(cudaMemcpyAsync(sing.ptr, hs.data(), hs.size() * 4, cudaMemcpyHostToDevice, s));
            hits.alloc(size_t(ns) * nb);
            DG_CUDA(cudaMemsetAsync(hits.ptr, 0, hits.bytes(), s));
            k_sample<<<ns, 256, 0, s>>>(g, dim2, sing.ptr, nb, a.r0, a.r1,
                                        m.has_radial_range ? 0 : 1, hits.ptr);
            DG_CUDA(cudaGetLastError());
            k_sample_count<<<ns, 256, 0, s>>>(sing.ptr, nb, hits.ptr, count.ptr);
            DG_CUDA(cudaGetLastError());
            std::vector<int32_t> hslot(size_t(npix), -1);
            for (int32_t i = 0; i < ns; ++i) hslot[size_t(hs[size_t(i)])] = i;
            slot.alloc(size_t(npix));
            DG_CUDA(cudaMemcpyAsync(slot.ptr, hslot.data(), size_t(npix) * 4,
                                    cudaMemcpyHostToDevice, s));
            DG_CUDA(cudaStreamSynchronize(s));
        }
        ncoo = scan_counts();
        if (ncoo > 64ll * 1024 * 1024)
            fail(DG_UNSUPPORTED, "pyFAI-compatible splitting exceeds the 64-million-entry memory "
                                 "bound; reduce binning.");
        k_pf1d_fill<<<grid_for(npix, 128), 128, 0, s>>>(a, off.ptr, ns ? slot.ptr : nullptr,
                                                        hits.ptr, cbin.ptr, cw.ptr, cpix.ptr,
                                                        flags.ptr);
        DG_CUDA(cudaGetLastError());
    } else {
        fail(DG_UNSUPPORTED, "unknown integration method");
    }

    int hflags[2] = {0, 0};
    DG_CUDA(cudaMemcpyAsync(hflags, flags.ptr, sizeof hflags, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    if (hflags[0]) fail(DG_UNSUPPORTED, "polygon clipping exceeded its vertex capacity");
    if (hflags[1]) fail(DG_UNSUPPORTED, "a pixel spans more than 64 radial bins");

    transpose(cbin.ptr, cw.ptr, cpix.ptr, off.ptr, npix, ncoo, nb, s, out.full);

    out.radial_centres.resize(size_t(nb));
    for (int i = 0; i < nb; ++i)
        out.radial_centres[size_t(i)] = out.hist_min + (double(i) + 0.5) * out.hist_step;
}

void compact_table(const DeviceCsr &full, const uint8_t *d_mask, int32_t n_pixels,
                   cudaStream_t s, DeviceCsr &out) {
    (void)n_pixels;
    out.n_rows = full.n_rows;
    out.row_ptr.alloc(size_t(full.n_rows) + 1);
    if (!d_mask) {
        DG_CUDA(cudaMemcpyAsync(out.row_ptr.ptr, full.row_ptr.ptr, out.row_ptr.bytes(),
                                cudaMemcpyDeviceToDevice, s));
        out.col.alloc(size_t(full.nnz));
        out.w.alloc(size_t(full.nnz));
        if (full.nnz) {
            DG_CUDA(cudaMemcpyAsync(out.col.ptr, full.col.ptr, size_t(full.nnz) * 4,
                                    cudaMemcpyDeviceToDevice, s));
            DG_CUDA(cudaMemcpyAsync(out.w.ptr, full.w.ptr, size_t(full.nnz) * 8,
                                    cudaMemcpyDeviceToDevice, s));
        }
        out.nnz = full.nnz;
        DG_CUDA(cudaStreamSynchronize(s));
        return;
    }
    const int64_t nnz = full.nnz;
    DeviceArray<int32_t> keep;
    keep.alloc(size_t(nnz) + 1);
    DG_CUDA(cudaMemsetAsync(keep.ptr, 0, keep.bytes(), s));
    DeviceArray<int64_t> pos;
    pos.alloc(size_t(nnz) + 1);
    DeviceArray<unsigned char> tmp;
    tmp.alloc(scan_temp_bytes(nnz + 1));
    k_keep<<<grid_for(nnz), 256, 0, s>>>(full.col.ptr, nnz, d_mask, keep.ptr);
    DG_CUDA(cudaGetLastError());
    exclusive_scan_i32_to_i64(keep.ptr, pos.ptr, nnz + 1, tmp.ptr, s);
    int64_t total = 0;
    DG_CUDA(cudaMemcpyAsync(&total, pos.ptr + nnz, sizeof total, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    out.nnz = total;
    out.col.alloc(size_t(total));
    out.w.alloc(size_t(total));
    k_compact<<<grid_for(nnz), 256, 0, s>>>(full.col.ptr, full.w.ptr, nnz, keep.ptr, pos.ptr,
                                            out.col.ptr, out.w.ptr);
    DG_CUDA(cudaGetLastError());
    k_compact_rows<<<grid_for(full.n_rows + 1), 256, 0, s>>>(full.row_ptr.ptr, full.n_rows,
                                                             pos.ptr, nnz, total,
                                                             out.row_ptr.ptr);
    DG_CUDA(cudaGetLastError());
    DG_CUDA(cudaStreamSynchronize(s));
}

void denominators(const DeviceCsr &t, const double *d_norm, cudaStream_t s, double *d_den) {
    k_denominators<<<grid_for(t.n_rows, 128), 128, 0, s>>>(t.row_ptr.ptr, t.n_rows, t.col.ptr,
                                                           t.w.ptr, d_norm, d_den);
    DG_CUDA(cudaGetLastError());
}

}  // namespace dg

namespace dg {
namespace {

__global__ void k_eval_math(int which, const double *__restrict__ a, const double *__restrict__ b,
                            int64_t n, double *__restrict__ out) {
    for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < n;
         k += int64_t(gridDim.x) * blockDim.x) {
        switch (which) {
        case 0: out[k] = ddm::cr_atan2(a[k], b[k]); break;
        case 1: out[k] = ddm::cr_sin(a[k]); break;
        case 2: out[k] = atan2(a[k], b[k]); break;
        default: out[k] = sin(a[k]); break;
        }
    }
}

}  // namespace

void eval_math(int which, const double *a, const double *b, int64_t n, double *out,
               cudaStream_t s) {
    if (which < 0 || which > 3) fail(DG_INVALID_INPUT, "unknown function");
    if (n <= 0) return;
    k_eval_math<<<grid_for(n), 256, 0, s>>>(which, a, b, n, out);
    DG_CUDA(cudaGetLastError());
}

}  // namespace dg
