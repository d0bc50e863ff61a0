/*
 * CPU oracle for the lookup-table (CSR) integration path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker that the CUDA library is compared
 * against, never part of the product. Each function restates one piece of
 * the reference crate's CPU algorithm and cites the Rust file:line it follows.
 * Built with -O2 -ffp-contract=off -fno-fast-math so that no a*b+c is fused
 * (Rust does not contract either) and every libm call (atan2, sqrt, sin, cos,
 * fmod) is glibc's, which is what Rust's f64 methods call on Linux.
 */
#include "dioptrin_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI 3.14159265358979323846
#define OR_TAU 6.28318530717958647692
#define OR_EPS DBL_EPSILON

void or_lut_free(or_lut *lut) {
    if (!lut) return;
    free(lut->row_ptr);
    free(lut->col);
    free(lut->w);
    memset(lut, 0, sizeof(*lut));
}

/* ---------------------------------------------------------------- geometry */

/* TrigonometricConstants (geometry.rs:640-660). */
typedef struct {
    double s1, c1, s2, c2, s3, c3;
} trig_t;

static trig_t trig_of(const or_poni *p) {
    trig_t t;
    t.s1 = sin(p->rot1);
    t.c1 = cos(p->rot1);
    t.s2 = sin(p->rot2);
    t.c2 = cos(p->rot2);
    t.s3 = sin(p->rot3);
    t.c3 = cos(p->rot3);
    return t;
}

/* f_x1 / f_x2 / f_x3 (geometry.rs:663-680), evaluated in Rust's left-to-right
 * order: a*b*c is (a*b)*c and a+b-c is (a+b)-c. */
static inline double f_x1(double p1, double p2, double p3, const trig_t *t) {
    return p1 * t->c2 * t->c3 + p2 * (t->c3 * t->s1 * t->s2 - t->c1 * t->s3) -
           p3 * (t->c1 * t->c3 * t->s2 + t->s1 * t->s3);
}
static inline double f_x2(double p1, double p2, double p3, const trig_t *t) {
    return p1 * t->c2 * t->s3 + p2 * (t->c1 * t->c3 + t->s1 * t->s2 * t->s3) -
           p3 * (-(t->c3 * t->s1) + t->c1 * t->s2 * t->s3);
}
static inline double f_x3(double p1, double p2, double p3, const trig_t *t) {
    return p1 * t->s2 - p2 * t->c2 * t->s1 + p3 * t->c1 * t->c2;
}
/* f_tth (geometry.rs:684-686): atan2(sqrt(y*y + x*x), z). */
static inline double f_tth(double x, double y, double z) { return atan2(sqrt(y * y + x * x), z); }
/* f_azimuth (geometry.rs:690-692): atan2(x, y). */
static inline double f_azimuth(double x, double y) { return atan2(x, y); }

/* RadialConverter::convert (integration.rs:160-185). to_degrees multiplies by
 * the f64 quotient 180/pi; q = (4 pi / (lambda * scale)) * sin(tth * 0.5). */
double or_convert_unit(int unit, double wavelength, double tth) {
    switch (unit) {
    case OR_UNIT_TTH_DEG:
        return tth * (180.0 / OR_PI);
    case OR_UNIT_Q_A:
        return (4.0 * OR_PI / (wavelength * 1e10)) * sin(tth * 0.5);
    case OR_UNIT_Q_NM:
        return (4.0 * OR_PI / (wavelength * 1e9)) * sin(tth * 0.5);
    default:
        return tth;
    }
}

/* calc_pixel_positions_with_sample_reference_all (geometry.rs:373-404):
 * centre (i + 0.5) * pixel - poni. */
void or_sample_positions(const or_poni *p, int64_t dim1, int64_t dim2, double *x, double *y,
                         double *z) {
    trig_t t = trig_of(p);
    for (int64_t i = 0; i < dim1; ++i) {
        double d1 = ((double)i + 0.5) * p->pixel1 - p->poni1;
        for (int64_t j = 0; j < dim2; ++j) {
            double d2 = ((double)j + 0.5) * p->pixel2 - p->poni2;
            int64_t k = i * dim2 + j;
            x[k] = f_x1(d1, d2, p->distance, &t);
            y[k] = f_x2(d1, d2, p->distance, &t);
            z[k] = f_x3(d1, d2, p->distance, &t);
        }
    }
}

/* compute_geometry (corrections.rs:57-85): tth, radial, chi, solid angle
 * (cos^3 via powi(3) = c*(c*c), geometry.rs:697-707), polarisation
 * (cos(tth).powi(2) and 0.5*(1 + c2 - f*cos(2chi)*(1 - c2)), geometry.rs:625-636
 * and :715-717) and normalisation pol*sa. */
void or_centres(const or_poni *p, int64_t dim1, int64_t dim2, int unit, int has_pol,
                double pol_factor, double *tth, double *radial, double *chi, double *sa,
                double *pol, double *norm) {
    trig_t t = trig_of(p);
    for (int64_t i = 0; i < dim1; ++i) {
        double d1 = ((double)i + 0.5) * p->pixel1 - p->poni1;
        for (int64_t j = 0; j < dim2; ++j) {
            double d2 = ((double)j + 0.5) * p->pixel2 - p->poni2;
            int64_t k = i * dim2 + j;
            double x = f_x1(d1, d2, p->distance, &t);
            double y = f_x2(d1, d2, p->distance, &t);
            double zz = f_x3(d1, d2, p->distance, &t);
            double tt = f_tth(x, y, zz);
            double az = f_azimuth(x, y);
            double cosa = p->distance / sqrt(d1 * d1 + d2 * d2 + p->distance * p->distance);
            double s = cosa * (cosa * cosa);
            double po = 1.0;
            if (has_pol) {
                double c = cos(tt);
                double c2 = c * c;
                po = 0.5 * (1.0 + c2 - pol_factor * cos(2.0 * az) * (1.0 - c2));
            }
            if (tth) tth[k] = tt;
            if (radial) radial[k] = or_convert_unit(unit, p->wavelength, tt);
            if (chi) chi[k] = az;
            if (sa) sa[k] = s;
            if (pol) pol[k] = po;
            if (norm) norm[k] = po * s;
        }
    }
}

/* angular_corners + corner_grid (geometry.rs:229-278): corner (i, j) at
 * d = i * pixel - poni on the (dim1+1) x (dim2+1) grid. */
void or_corners(const or_poni *p, int64_t dim1, int64_t dim2, int unit, double *radial,
                double *chi) {
    trig_t t = trig_of(p);
    for (int64_t i = 0; i <= dim1; ++i) {
        double d1 = (double)i * p->pixel1 - p->poni1;
        for (int64_t j = 0; j <= dim2; ++j) {
            double d2 = (double)j * p->pixel2 - p->poni2;
            int64_t k = i * (dim2 + 1) + j;
            double x = f_x1(d1, d2, p->distance, &t);
            double y = f_x2(d1, d2, p->distance, &t);
            double z = f_x3(d1, d2, p->distance, &t);
            radial[k] = or_convert_unit(unit, p->wavelength, f_tth(x, y, z));
            chi[k] = f_azimuth(x, y);
        }
    }
}

/* calc_tth_and_azimuth on explicit coordinates (geometry.rs:519-549). */
void or_tth_chi_at(const or_poni *p, const double *d1, const double *d2, int64_t n,
                   double *tth, double *chi) {
    trig_t t = trig_of(p);
    for (int64_t k = 0; k < n; ++k) {
        double a = d1[k] * p->pixel1 - p->poni1;
        double b = d2[k] * p->pixel2 - p->poni2;
        double x = f_x1(a, b, p->distance, &t);
        double y = f_x2(a, b, p->distance, &t);
        double z = f_x3(a, b, p->distance, &t);
        if (tth) tth[k] = f_tth(x, y, z);
        if (chi) chi[k] = f_azimuth(x, y);
    }
}

/* --------------------------------------------------------------- histogram */

/* math::min / math::max (math/mod.rs:8-35): first extreme by strict compare. */
static double seq_min(const double *v, int64_t n) {
    double m = v[0];
    for (int64_t i = 1; i < n; ++i)
        if (v[i] < m) m = v[i];
    return m;
}
static double seq_max(const double *v, int64_t n) {
    double m = v[0];
    for (int64_t i = 1; i < n; ++i)
        if (v[i] > m) m = v[i];
    return m;
}

/* min_max_step (histogram.rs:191-196). */
void or_min_max_step(const double *data, int64_t n, int64_t n_points, double *min, double *max,
                     double *step) {
    double lo = seq_min(data, n);
    double hi = seq_max(data, n) + 10.0 * OR_EPS;
    *min = lo;
    *max = hi;
    *step = (hi - lo) / (double)n_points;
}

/* bins (histogram.rs:199-203): min + (i + 0.5) * step. */
void or_bins(int64_t n_points, double min, double step, double *out) {
    for (int64_t i = 0; i < n_points; ++i) out[i] = min + ((double)i + 0.5) * step;
}

/* `f as usize` in Rust: truncation toward zero, saturating, NaN -> 0. */
static inline uint64_t as_usize(double v) {
    if (!(v > 0.0)) return 0;
    if (v >= 18446744073709551616.0) return UINT64_MAX;
    return (uint64_t)v;
}
/* `f as isize`: truncation, saturating, NaN -> 0. */
static inline int64_t as_isize(double v) {
    if (v != v) return 0;
    if (v >= 9223372036854775808.0) return INT64_MAX;
    if (v <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)v;
}

/* get_bin_clamped (histogram.rs:126-129). */
static inline int64_t bin_clamped(double v, double min, double step, int64_t n) {
    uint64_t b = as_usize((v - min) / step);
    return b < (uint64_t)(n - 1) ? (int64_t)b : n - 1;
}

/* rem_euclid(TAU) for f64: r = x % TAU; r < 0 ? r + TAU : r. */
static inline double rem_euclid_tau(double x) {
    double r = fmod(x, OR_TAU);
    return r < 0.0 ? r + OR_TAU : r;
}
/* wrap_tau (pyfai_1d.rs:170-177). */
static inline double wrap_tau(double x) {
    if (x >= 0.0 && x < OR_TAU) return x;
    return rem_euclid_tau(x);
}

/* ------------------------------------------------------------- CSR growing */

typedef struct {
    int64_t *col;
    double *w;
    int64_t n, cap;
} bucket_t;

static int bucket_push(bucket_t *b, int64_t col, double w) {
    if (b->n == b->cap) {
        int64_t cap = b->cap ? b->cap * 2 : 8;
        int64_t *c = (int64_t *)realloc(b->col, (size_t)cap * sizeof(int64_t));
        if (!c) return -1;
        b->col = c;
        double *ww = (double *)realloc(b->w, (size_t)cap * sizeof(double));
        if (!ww) return -1;
        b->w = ww;
        b->cap = cap;
    }
    b->col[b->n] = col;
    b->w[b->n] = w;
    b->n++;
    return 0;
}

/* lut1d_from_fractions (pixel_split.rs:332-356): concatenate buckets in bin
 * order; within a bucket, entries keep their push order (ascending pixel). */
static int buckets_to_lut(bucket_t *buckets, int64_t n, int weighted, double min, double step,
                          or_lut *out) {
    memset(out, 0, sizeof(*out));
    out->n_rows = n;
    out->hist_min = min;
    out->hist_step = step;
    out->row_ptr = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    if (!out->row_ptr) return -1;
    for (int64_t i = 0; i < n; ++i) out->row_ptr[i + 1] = out->row_ptr[i] + buckets[i].n;
    out->nnz = out->row_ptr[n];
    out->col = (int64_t *)malloc((size_t)(out->nnz ? out->nnz : 1) * sizeof(int64_t));
    if (weighted) out->w = (double *)malloc((size_t)(out->nnz ? out->nnz : 1) * sizeof(double));
    if (!out->col || (weighted && !out->w)) return -1;
    for (int64_t i = 0; i < n; ++i) {
        int64_t at = out->row_ptr[i];
        if (buckets[i].n) {
            memcpy(out->col + at, buckets[i].col, (size_t)buckets[i].n * sizeof(int64_t));
            if (weighted) memcpy(out->w + at, buckets[i].w, (size_t)buckets[i].n * sizeof(double));
        }
        free(buckets[i].col);
        free(buckets[i].w);
    }
    free(buckets);
    return 0;
}

/* ------------------------------------------------------ polygon clipping */

typedef struct {
    double x, y;
} pt_t;

/* polygon_area (pixel_split.rs:14-25): 0.5 * sum(x0*y1 - x1*y0). */
static double polygon_area(const pt_t *poly, int n) {
    if (n < 3) return 0.0;
    double area = 0.0;
    for (int i = 0; i < n; ++i) {
        pt_t a = poly[i], b = poly[(i + 1) % n];
        area += a.x * b.y - b.x * a.y;
    }
    return 0.5 * area;
}

/* intersect_with_x / intersect_with_y (pixel_split.rs:28-45). */
static inline pt_t isect_x(pt_t p0, pt_t p1, double xe) {
    double dx = p1.x - p0.x;
    pt_t r;
    r.x = xe;
    if (fabs(dx) < OR_EPS) {
        r.y = p0.y;
        return r;
    }
    double t = (xe - p0.x) / dx;
    r.y = p0.y + t * (p1.y - p0.y);
    return r;
}
static inline pt_t isect_y(pt_t p0, pt_t p1, double ye) {
    double dy = p1.y - p0.y;
    pt_t r;
    r.y = ye;
    if (fabs(dy) < OR_EPS) {
        r.x = p0.x;
        return r;
    }
    double t = (ye - p0.y) / dy;
    r.x = p0.x + t * (p1.x - p0.x);
    return r;
}

/* One Sutherland-Hodgman half-plane pass (pixel_split.rs:48-145).
 * side: 0 = x >= e, 1 = x <= e, 2 = y >= e, 3 = y <= e. */
static int clip_pass(const pt_t *in, int n, double e, int side, pt_t *out) {
    int m = 0;
    if (n == 0) return 0;
    pt_t prev = in[n - 1];
#define INSIDE(p) (side == 0 ? (p).x >= e : side == 1 ? (p).x <= e : side == 2 ? (p).y >= e : (p).y <= e)
#define ISECT(a, b) (side < 2 ? isect_x((a), (b), e) : isect_y((a), (b), e))
    int prev_in = INSIDE(prev);
    for (int i = 0; i < n; ++i) {
        pt_t cur = in[i];
        int cur_in = INSIDE(cur);
        if (cur_in) {
            if (!prev_in) out[m++] = ISECT(prev, cur);
            out[m++] = cur;
        } else if (prev_in) {
            out[m++] = ISECT(prev, cur);
        }
        prev = cur;
        prev_in = cur_in;
    }
#undef INSIDE
#undef ISECT
    return m;
}

/* clip_polygon_rect_scratch (pixel_split.rs:148-163): left, right, bottom,
 * top, stopping as soon as a pass leaves nothing. */
static int clip_rect(const pt_t *poly, int n, double x0, double x1, double y0, double y1,
                     pt_t *buf1, pt_t *buf2, const pt_t **res) {
    int m = clip_pass(poly, n, x0, 0, buf1);
    if (!m) { *res = buf1; return 0; }
    m = clip_pass(buf1, m, x1, 1, buf2);
    if (!m) { *res = buf2; return 0; }
    m = clip_pass(buf2, m, y0, 2, buf1);
    if (!m) { *res = buf1; return 0; }
    m = clip_pass(buf1, m, y1, 3, buf2);
    *res = buf2;
    return m;
}

/* unwrap_angle (pixel_split.rs:166-175). */
static inline double unwrap_angle(double a, double ref) {
    double d = a - ref;
    if (d > OR_PI) a -= 2.0 * OR_PI;
    else if (d < -OR_PI) a += 2.0 * OR_PI;
    return a;
}

/* singular (pyfai_1d.rs:188-201). */
static int singular(const pt_t poly[4]) {
    double winding = 0.0;
    for (int i = 0; i < 4; ++i) {
        if (poly[i].x == 0.0) return 1;
        double delta = wrap_tau(poly[(i + 1) % 4].y - poly[i].y + OR_PI) - OR_PI;
        if (fabs(delta) >= OR_PI - 64.0 * OR_EPS) return 1;
        winding += delta;
    }
    return fabs(winding) > OR_PI;
}

/* sample (pyfai_1d.rs:208-252) for a grid of n_radial bins over [r0, r1) and
 * one azimuthal bin over [-pi, pi): 128 x 128 x 4 detector-plane samples,
 * hits counted per bin, weight hits / 65536, bins ascending. */
static int sample_pixel(const or_poni *p, int64_t dim2, int64_t pixel, int unit, double r0,
                        double r1, int64_t nr, int clamp_low, bucket_t *buckets) {
    const int N = 128;
    static const double off[4][2] = {{0.25, 0.5}, {0.5, 0.25}, {0.75, 0.5}, {0.5, 0.75}};
    const int64_t count = (int64_t)N * N * 4;
    const double a0 = -OR_PI, a1 = OR_PI;
    const int64_t na = 1;
    int64_t *hits = (int64_t *)calloc((size_t)nr, sizeof(int64_t));
    if (!hits) return -1;
    trig_t t = trig_of(p);
    double prow = (double)(pixel / dim2), pcol = (double)(pixel % dim2);
    for (int row = 0; row < N; ++row)
        for (int col = 0; col < N; ++col)
            for (int o = 0; o < 4; ++o) {
                double d1 = prow + ((double)row + off[o][0]) / (double)N;
                double d2 = pcol + ((double)col + off[o][1]) / (double)N;
                double a = d1 * p->pixel1 - p->poni1;
                double b = d2 * p->pixel2 - p->poni2;
                double x = f_x1(a, b, p->distance, &t);
                double y = f_x2(a, b, p->distance, &t);
                double z = f_x3(a, b, p->distance, &t);
                double r = or_convert_unit(unit, p->wavelength, f_tth(x, y, z));
                double az = f_azimuth(x, y);
                az = a0 + rem_euclid_tau(az - a0);
                if ((r < r0 && !clamp_low) || r >= r1 || az >= a1) continue;
                uint64_t ir = r < r0 ? 0 : as_usize((r - r0) / (r1 - r0) * (double)nr);
                uint64_t ia = as_usize((az - a0) / (a1 - a0) * (double)na);
                if (ir < (uint64_t)nr && ia < (uint64_t)na) hits[ia * nr + ir] += 1;
            }
    for (int64_t b = 0; b < nr; ++b)
        if (hits[b] && bucket_push(&buckets[b], pixel, (double)hits[b] / (double)count)) {
            free(hits);
            return -1;
        }
    free(hits);
    return 0;
}

/* IntegrationGrid2d::new validity for the 1D sampling grid (grid.rs:49-105):
 * n_radial bins over [lo, hi) and one azimuthal bin over [-pi, pi). */
static int grid_ok(double lo, double hi, int64_t n) {
    double step = (hi - lo) / (double)n;
    if (!isfinite(lo) || !isfinite(hi) || !isfinite(step) || step <= 0.0 || lo + step == lo ||
        hi - step == hi)
        return 0;
    if (lo < 0.0) return 0;
    return 1;
}

/* lut1d_ps_fractions (pixel_split.rs:190-328). */
static int ps1d_core(const or_poni *p, int64_t dim1, int64_t dim2, int unit, int64_t n,
                     double min, double step, int clamp_low, const double *rc, const double *ac,
                     const double *centre_radial, const double *centre_chi, bucket_t *buckets) {
    const int64_t w = dim2 + 1;
    const int have_grid = grid_ok(min, min + (double)n * step, n);
    const double r1 = min + (double)n * step;
    pt_t buf1[64], buf2[64];
    for (int64_t idx = 0; idx < dim1 * dim2; ++idx) {
        int64_t b0 = idx / dim2 * w + idx % dim2;
        int64_t i00 = b0, i01 = b0 + 1, i11 = b0 + w + 1, i10 = b0 + w;
        double r00 = rc[i00], r01 = rc[i01], r10 = rc[i10], r11 = rc[i11];
        if (have_grid) {
            pt_t raw[4] = {{rc[i00], ac[i00]}, {rc[i01], ac[i01]}, {rc[i11], ac[i11]},
                           {rc[i10], ac[i10]}};
            if (singular(raw)) {
                if (sample_pixel(p, dim2, idx, unit, min, r1, n, clamp_low, buckets)) return -1;
                continue;
            }
        }
        double cchi = centre_chi[idx];
        double a00 = unwrap_angle(ac[i00], cchi);
        double a01 = unwrap_angle(ac[i01], cchi);
        double a10 = unwrap_angle(ac[i10], cchi);
        double a11 = unwrap_angle(ac[i11], cchi);
        pt_t poly[4] = {{r00, a00}, {r01, a01}, {r11, a11}, {r10, a10}};
        double area_total = fabs(polygon_area(poly, 4));
        if (area_total <= 0.0) {
            double pos = (centre_radial[idx] - min) / step;
            if (pos < 0.0) continue;
            int64_t bin = as_isize(floor(pos));
            if (bin >= 0 && bin < n)
                if (bucket_push(&buckets[bin], idx, 1.0)) return -1;
            continue;
        }
        double rmin = r00, rmax = r00;
        double rv[3] = {r01, r10, r11};
        for (int k = 0; k < 3; ++k) {
            if (rv[k] < rmin) rmin = rv[k];
            if (rv[k] > rmax) rmax = rv[k];
        }
        int64_t start = as_isize(floor((rmin - min) / step));
        int64_t end = as_isize(floor((rmax - min) / step));
        if (end < 0 || start >= n) continue;
        if (start < 0) start = 0;
        if (end >= n) end = n - 1;
        double amin = a00, amax = a00;
        double av[3] = {a01, a10, a11};
        for (int k = 0; k < 3; ++k) {
            if (av[k] < amin) amin = av[k];
            if (av[k] > amax) amax = av[k];
        }
        for (int64_t b = start; b <= end; ++b) {
            double bin_min = min + (double)b * step;
            double bin_max = bin_min + step;
            const pt_t *clipped;
            int m = clip_rect(poly, 4, bin_min, bin_max, amin, amax, buf1, buf2, &clipped);
            double area = fabs(polygon_area(clipped, m));
            if (area > 0.0)
                if (bucket_push(&buckets[b], idx, area / area_total)) return -1;
        }
    }
    return 0;
}

int or_ps1d_fractions(const or_poni *p, int64_t dim1, int64_t dim2, int unit, int64_t n,
                      double min, double step, int clamp_low, or_lut *out) {
    int64_t npix = dim1 * dim2, ncorner = (dim1 + 1) * (dim2 + 1);
    double *rc = (double *)malloc((size_t)ncorner * sizeof(double));
    double *ac = (double *)malloc((size_t)ncorner * sizeof(double));
    double *cr = (double *)malloc((size_t)npix * sizeof(double));
    double *cc = (double *)malloc((size_t)npix * sizeof(double));
    bucket_t *buckets = (bucket_t *)calloc((size_t)n, sizeof(bucket_t));
    int rc_ = -1;
    if (rc && ac && cr && cc && buckets) {
        or_corners(p, dim1, dim2, unit, rc, ac);
        or_centres(p, dim1, dim2, unit, 0, 0.0, NULL, cr, cc, NULL, NULL, NULL);
        rc_ = ps1d_core(p, dim1, dim2, unit, n, min, step, clamp_low, rc, ac, cr, cc, buckets);
        if (rc_ == 0) {
            rc_ = buckets_to_lut(buckets, n, 1, min, step, out);
            buckets = NULL;
        }
    }
    if (buckets) {
        for (int64_t i = 0; i < n; ++i) {
            free(buckets[i].col);
            free(buckets[i].w);
        }
        free(buckets);
    }
    free(rc);
    free(ac);
    free(cr);
    free(cc);
    return rc_;
}

/* build_lut1d_ps_csr (pixel_split.rs:389-419) and _with_range (:426-455). */
int or_build_ps1d(const or_poni *p, int64_t dim1, int64_t dim2, int unit, int64_t n,
                  int has_range, double rmin, double rmax, or_lut *out) {
    double min, step;
    if (has_range) {
        double hi = rmax + 10.0 * OR_EPS;
        min = rmin;
        step = (hi - rmin) / (double)n;
        return or_ps1d_fractions(p, dim1, dim2, unit, n, min, step, 0, out);
    }
    int64_t ncorner = (dim1 + 1) * (dim2 + 1);
    double *rc = (double *)malloc((size_t)ncorner * sizeof(double));
    double *ac = (double *)malloc((size_t)ncorner * sizeof(double));
    if (!rc || !ac) {
        free(rc);
        free(ac);
        return -1;
    }
    or_corners(p, dim1, dim2, unit, rc, ac);
    min = seq_min(rc, ncorner);
    double max = seq_max(rc, ncorner);
    max += 10.0 * OR_EPS;
    step = (max - min) / (double)n;
    free(rc);
    free(ac);
    return or_ps1d_fractions(p, dim1, dim2, unit, n, min, step, 1, out);
}

/* split1d (pyfai_1d.rs:259-354): pyFAI's fullSplit1D rule for one pixel
 * quadrilateral given in pyFAI corner order (A, D, C, B) as (radial, chi)
 * pairs, on n radial bins over [r0, r1) and azimuthal edges [a0, a1). The
 * azimuths are recentred at the canonical seam and unwrapped when pyFAI's
 * area4p test (with its operator precedence, times the corner sign) is
 * positive; each edge's signed area under the line is integrated per radial
 * bin into an f32 buffer; buffer / sum, kept if finite and > 0, renormalised.
 * Writes at most cap pairs; returns their count, or -1 when the pixel spans
 * more than cap bins. */
int or_split1d(const double *poly_in, int64_t n, double r0, double r1, double a0, double a1,
               int sector, double sign, int64_t *bins, double *weights, int64_t cap) {
    pt_t poly[4];
    for (int i = 0; i < 4; ++i) {
        poly[i].x = poly_in[2 * i];
        poly[i].y = poly_in[2 * i + 1];
    }
    double offset;
    if (a0 >= -OR_PI && a1 <= OR_PI) offset = 0.0;
    else if (a0 >= 0.0 && a1 <= OR_TAU) offset = OR_PI;
    else offset = a0 + OR_PI;
    for (int i = 0; i < 4; ++i) poly[i].y = wrap_tau(poly[i].y - offset + OR_PI) - OR_PI;
    pt_t a = poly[0], b = poly[1], c = poly[2], d = poly[3];
    double area = sign * (0.5 * (c.x - a.x) * (d.y - b.y) - (c.y - a.y) * (d.x - b.x));
    if (area > 0.0) {
        for (int i = 0; i < 4; ++i)
            if (poly[i].y < 0.0) poly[i].y += OR_TAU;
        double sum = -0.0;
        for (int i = 0; i < 4; ++i) sum += poly[i].y;
        if (sum * 0.25 > OR_PI)
            for (int i = 0; i < 4; ++i) poly[i].y -= OR_TAU;
    }
    for (int i = 0; i < 4; ++i) poly[i].y += offset;
    if (sector) {
        int below = 1, above = 1;
        for (int i = 0; i < 4; ++i) {
            below &= poly[i].y < a0;
            above &= poly[i].y > a1;
        }
        if (below || above) return 0;
    }
    double dr = (r1 - r0) / (double)n;
    for (int i = 0; i < 4; ++i) poly[i].x = (poly[i].x - r0) / dr;
    double lo = INFINITY, hi = -INFINITY;
    for (int i = 0; i < 4; ++i) {
        lo = fmin(lo, poly[i].x);
        hi = fmax(hi, poly[i].x);
    }
    if (hi < 0.0 || lo >= (double)n) return 0;
    double flo = floor(lo), fhi = floor(hi);
    int64_t first = (int64_t)as_usize(fmax(flo, 0.0));
    int64_t end_i = as_isize(fhi) + 1;
    if (end_i < 0) end_i = 0;
    if (end_i > n) end_i = n;
    if (flo == fhi) {
        if (cap < 1) return -1;
        bins[0] = first;
        weights[0] = 1.0;
        return 1;
    }
    int64_t span = end_i - first;
    if (span > cap) return -1;
    float buffer[256];
    if (span > 256) return -1;
    for (int64_t j = 0; j < span; ++j) buffer[j] = 0.0f;
    for (int i = 0; i < 4; ++i) {
        double x0 = poly[i].x, y0 = poly[i].y, x1 = poly[(i + 1) % 4].x, y1 = poly[(i + 1) % 4].y;
        if (x0 == x1) continue;
        double slope = (y1 - y0) / (x1 - x0);
        double intercept = y0 - slope * x0;
        double sg = x1 > x0 ? 1.0 : -1.0;
        for (int64_t j = 0; j < span; ++j) {
            double left = fmax(fmin(x0, x1), (double)(first + j));
            double right = fmin(fmax(x0, x1), (double)(first + j + 1));
            if (right > left)
                buffer[j] += (float)(sg * (right - left) * (0.5 * slope * (right + left) + intercept));
        }
    }
    double sum = -0.0;
    for (int64_t j = 0; j < span; ++j) sum += (double)buffer[j];
    if (!isfinite(sum) || sum == 0.0) return 0;
    int64_t m = 0;
    for (int64_t j = 0; j < span; ++j) {
        double w = (double)buffer[j] / sum;
        if (isfinite(w) && w > 0.0) {
            bins[m] = first + j;
            weights[m] = w;
            ++m;
        }
    }
    double total = -0.0;
    for (int64_t k = 0; k < m; ++k) total += weights[k];
    for (int64_t k = 0; k < m; ++k) weights[k] /= total;
    return (int)m;
}

/* pyfai_radial_range (pyfai_1d.rs:36-46): corner radial min (at least 0) and
 * max * (1 + f32::EPSILON). */
void or_pyfai_radial_range(const or_poni *p, int64_t dim1, int64_t dim2, int unit, double *lo,
                           double *hi) {
    int64_t ncorner = (dim1 + 1) * (dim2 + 1);
    double *rc = (double *)malloc((size_t)ncorner * sizeof(double));
    double *ac = (double *)malloc((size_t)ncorner * sizeof(double));
    if (!rc || !ac) {
        free(rc);
        free(ac);
        *lo = *hi = NAN;
        return;
    }
    or_corners(p, dim1, dim2, unit, rc, ac);
    double mn = INFINITY, mx = -INFINITY;
    for (int64_t i = 0; i < ncorner; ++i) {
        mn = fmin(mn, rc[i]);
        mx = fmax(mx, rc[i]);
    }
    *lo = fmax(mn, 0.0);
    *hi = mx * (1.0 + (double)FLT_EPSILON);
    free(rc);
    free(ac);
}

/* build_lut1d_pyfai_csr (pyfai_1d.rs:55-109) without an azimuthal sector and
 * with the corner sign of a geometry without a detector object (+1,
 * pyfai_1d.rs:131-137): singular pixels by detector-plane sampling, the rest by
 * split1d. Returns -2 past the 64 Mi entry bound, -3 for a grid
 * IntegrationGrid2d::new rejects. */
int or_build_pf1d(const or_poni *p, int64_t dim1, int64_t dim2, int unit, int64_t n,
                  int has_range, double rmin, double rmax, or_lut *out) {
    double r0 = rmin, r1 = rmax;
    if (!has_range) or_pyfai_radial_range(p, dim1, dim2, unit, &r0, &r1);
    if (!grid_ok(r0, r1, n)) return -3;
    int64_t ncorner = (dim1 + 1) * (dim2 + 1);
    double *rc = (double *)malloc((size_t)ncorner * sizeof(double));
    double *ac = (double *)malloc((size_t)ncorner * sizeof(double));
    bucket_t *buckets = (bucket_t *)calloc((size_t)n, sizeof(bucket_t));
    int rc_ = -1;
    if (rc && ac && buckets) {
        or_corners(p, dim1, dim2, unit, rc, ac);
        const int64_t w = dim2 + 1;
        int64_t entries = 0;
        int64_t bins[256];
        double ws[256];
        rc_ = 0;
        for (int64_t idx = 0; idx < dim1 * dim2 && rc_ == 0; ++idx) {
            int64_t b0 = idx / dim2 * w + idx % dim2;
            int64_t ia = b0, ib = b0 + 1, ic = b0 + w + 1, id = b0 + w;
            /* corner_indices order A, B, C, D taken as [a, d, c, b] */
            pt_t poly[4] = {{rc[ia], ac[ia]}, {rc[id], ac[id]}, {rc[ic], ac[ic]}, {rc[ib], ac[ib]}};
            if (singular(poly)) {
                int64_t before = 0;
                for (int64_t k = 0; k < n; ++k) before += buckets[k].n;
                if (sample_pixel(p, dim2, idx, unit, r0, r1, n, !has_range, buckets)) rc_ = -1;
                int64_t after = 0;
                for (int64_t k = 0; k < n; ++k) after += buckets[k].n;
                entries += after - before;
            } else {
                double flat[8] = {poly[0].x, poly[0].y, poly[1].x, poly[1].y,
                                  poly[2].x, poly[2].y, poly[3].x, poly[3].y};
                int m = or_split1d(flat, n, r0, r1, -OR_PI, OR_PI, 0, 1.0, bins, ws, 256);
                if (m < 0) {
                    rc_ = -1;
                    break;
                }
                entries += m;
                for (int k = 0; k < m; ++k)
                    if (bucket_push(&buckets[bins[k]], idx, ws[k])) rc_ = -1;
            }
            if (entries > 64LL * 1024 * 1024) rc_ = -2;
        }
        if (rc_ == 0) {
            rc_ = buckets_to_lut(buckets, n, 1, r0, (r1 - r0) / (double)n, out);
            buckets = NULL;
        }
    }
    if (buckets) {
        for (int64_t i = 0; i < n; ++i) {
            free(buckets[i].col);
            free(buckets[i].w);
        }
        free(buckets);
    }
    free(rc);
    free(ac);
    return rc_;
}

/* build_lut1d_csr (counting_csr.rs:54-89) and _with_range (:95-134). */
int or_build_counting1d(const double *radial, int64_t npix, int64_t n, int has_range,
                        double rmin, double rmax, or_lut *out) {
    double min, max, step;
    if (has_range) {
        max = rmax + 10.0 * OR_EPS;
        min = rmin;
        step = (max - min) / (double)n;
    } else {
        or_min_max_step(radial, npix, n, &min, &max, &step);
    }
    bucket_t *buckets = (bucket_t *)calloc((size_t)n, sizeof(bucket_t));
    if (!buckets) return -1;
    for (int64_t i = 0; i < npix; ++i) {
        double v = radial[i];
        int64_t b;
        if (has_range) {
            /* get_bin_in_range (histogram.rs:136-141) */
            if (!(v >= min && v <= max)) continue;
        }
        b = bin_clamped(v, min, step, n);
        if (bucket_push(&buckets[b], i, 1.0)) return -1;
    }
    return buckets_to_lut(buckets, n, 0, min, step, out);
}

/* hull_grid (lut/common.rs:33-65). Returns the number of points. */
static int64_t hull_grid(int64_t dim1, int64_t dim2, int64_t n_ss, double *d1, double *d2) {
    int64_t k = 0;
    double off = 0.5 / (double)n_ss, st = 1.0 / (double)n_ss;
    for (int64_t i = 0; i < dim1 * n_ss; ++i) { d1[k] = off + (double)i * st; d2[k++] = off; }
    for (int64_t i = 0; i < dim1 * n_ss; ++i) {
        d1[k] = off + (double)i * st;
        d2[k++] = (double)dim2 - off;
    }
    for (int64_t i = 1; i < dim2 * n_ss; ++i) { d1[k] = off; d2[k++] = off + (double)i * st; }
    for (int64_t i = 1; i < dim2 * n_ss; ++i) {
        d1[k] = (double)dim1 - off;
        d2[k++] = off + (double)i * st;
    }
    return k;
}

/* build_lut1d_ss_csr (supersampled.rs:517-552) via the exact
 * build_counted_csr (:21-104): per pixel, samples d1 = row + (i + .5)/n,
 * d2 = ((col*n + j) + .5)/n, counted per distinct bin in first-seen order,
 * rows filled in pixel order, weight = count / n^2. */
int or_build_ss1d(const or_poni *p, int64_t dim1, int64_t dim2, int unit, int64_t n,
                  int64_t n_ss, int has_range, double rmin, double rmax, or_lut *out) {
    double min, max, step;
    int64_t npix = dim1 * dim2;
    if (has_range) {
        max = rmax + 10.0 * OR_EPS;
        min = rmin;
        step = (max - min) / (double)n;
    } else {
        /* ss_tth_min_max_step (histogram.rs:151-166) */
        int64_t hn = 2 * (dim1 + dim2) * n_ss;
        double *hd1 = (double *)malloc((size_t)hn * sizeof(double));
        double *hd2 = (double *)malloc((size_t)hn * sizeof(double));
        double *ht = (double *)malloc((size_t)hn * sizeof(double));
        double *cr = (double *)malloc((size_t)npix * sizeof(double));
        if (!hd1 || !hd2 || !ht || !cr) return -1;
        int64_t m = hull_grid(dim1, dim2, n_ss, hd1, hd2);
        or_tth_chi_at(p, hd1, hd2, m, ht, NULL);
        for (int64_t i = 0; i < m; ++i) ht[i] = or_convert_unit(unit, p->wavelength, ht[i]);
        or_centres(p, dim1, dim2, unit, 0, 0.0, NULL, cr, NULL, NULL, NULL, NULL);
        double a = seq_min(cr, npix), b = seq_min(ht, m);
        min = b < a ? b : a; /* f64::min: NaN-free here */
        a = seq_max(cr, npix);
        b = seq_max(ht, m);
        max = (b > a ? b : a) + 3.0 * OR_EPS;
        step = (max - min) / (double)n;
        free(hd1);
        free(hd2);
        free(ht);
        free(cr);
    }
    bucket_t *buckets = (bucket_t *)calloc((size_t)n, sizeof(bucket_t));
    if (!buckets) return -1;
    trig_t t = trig_of(p);
    int64_t *cb = (int64_t *)malloc((size_t)(n_ss * n_ss) * sizeof(int64_t));
    int64_t *cn = (int64_t *)malloc((size_t)(n_ss * n_ss) * sizeof(int64_t));
    double denom = (double)(n_ss * n_ss);
    for (int64_t row = 0; row < dim1; ++row)
        for (int64_t col = 0; col < dim2; ++col) {
            int nc = 0;
            for (int64_t i = 0; i < n_ss; ++i) {
                double d1 = (double)row + ((double)i + 0.5) / (double)n_ss;
                for (int64_t j = 0; j < n_ss; ++j) {
                    double d2 = ((double)(col * n_ss + j) + 0.5) / (double)n_ss;
                    double a = d1 * p->pixel1 - p->poni1;
                    double bb = d2 * p->pixel2 - p->poni2;
                    double x = f_x1(a, bb, p->distance, &t);
                    double y = f_x2(a, bb, p->distance, &t);
                    double z = f_x3(a, bb, p->distance, &t);
                    double r = or_convert_unit(unit, p->wavelength, f_tth(x, y, z));
                    int64_t bin;
                    if (has_range) {
                        if (!(r >= min && r <= max)) continue;
                    }
                    bin = bin_clamped(r, min, step, n);
                    int f = -1;
                    for (int q = 0; q < nc; ++q)
                        if (cb[q] == bin) { f = q; break; }
                    if (f < 0) { cb[nc] = bin; cn[nc++] = 1; }
                    else cn[f]++;
                }
            }
            int64_t pixel = row * dim2 + col;
            for (int q = 0; q < nc; ++q) bucket_push(&buckets[cb[q]], pixel, (double)cn[q]);
        }
    free(cb);
    free(cn);
    int rc_ = buckets_to_lut(buckets, n, 1, min, step, out);
    if (rc_ == 0)
        for (int64_t k = 0; k < out->nnz; ++k) out->w[k] /= denom;
    return rc_;
}

/* ---------------------------------------------------------------- gather */

/* ================================================================ 2D tables */

/* IntegrationGrid2d::new (grid.rs:49-105): bin counts, finite, increasing and
 * resolvable edges, nonnegative radial start, azimuthal span of at most one
 * turn, a start outside +-2pi moved into [-pi, pi). Returns 0 or -1. */
int or_grid2d_new(int64_t nr, int64_t na, double r0, double r1, double a0, double a1,
                  or_grid2d *g) {
    memset(g, 0, sizeof(*g));
    if (nr <= 0 || na <= 0) return -1;
    double lo[2] = {r0, a0}, hi[2] = {r1, a1};
    int64_t cnt[2] = {nr, na};
    for (int k = 0; k < 2; ++k) {
        double step = (hi[k] - lo[k]) / (double)cnt[k];
        if (!isfinite(lo[k]) || !isfinite(hi[k]) || !isfinite(step) || step <= 0.0 ||
            lo[k] + step == lo[k] || hi[k] - step == hi[k])
            return -1;
    }
    if (r0 < 0.0) return -1;
    if (a1 - a0 > OR_TAU + 1e-12) return -1;
    if (!(a0 >= -OR_TAU && a0 <= OR_TAU)) {
        double start = rem_euclid_tau(a0);
        if (start >= OR_PI) start -= OR_TAU;
        double span = a1 - a0;
        a0 = start;
        a1 = start + span;
    }
    g->n_radial = nr;
    g->n_azimuthal = na;
    g->r0 = r0;
    g->r1 = r1;
    g->a0 = a0;
    g->a1 = a1;
    return 0;
}

static inline double grid_dr(const or_grid2d *g) { return (g->r1 - g->r0) / (double)g->n_radial; }
static inline double grid_da(const or_grid2d *g) { return (g->a1 - g->a0) / (double)g->n_azimuthal; }

/* f64::clamp. */
static inline double clampd(double x, double lo, double hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

/* IntegrationGrid2d::bin (grid.rs:176-222); -1 for no bin. */
int64_t or_grid2d_bin(const or_grid2d *g, double radial, double azimuthal) {
    double r0 = g->r0, r1 = g->r1, a0 = g->a0, a1 = g->a1;
    if (!isfinite(radial) || !isfinite(azimuthal)) return -1;
    if (!g->clamp_radial_outside &&
        (radial < r0 || radial > r1 || (radial == r1 && !g->clamp_radial_end)))
        return -1;
    double offset;
    if (g->clamp_azimuthal_outside) {
        offset = clampd(azimuthal - a0, 0.0, a1 - a0);
    } else if (g->clamp_index_rounding) {
        double wrapped = (azimuthal >= a0 && azimuthal < a1)
                             ? azimuthal
                             : a0 + rem_euclid_tau(azimuthal - a0);
        if (wrapped >= a1 && a1 - a0 < OR_TAU) return -1;
        offset = wrapped - a0;
    } else {
        double az = a0 + rem_euclid_tau(azimuthal - a0);
        if (az >= a1) return -1;
        offset = az - a0;
    }
    uint64_t r = as_usize((radial - r0) / grid_dr(g));
    uint64_t a = as_usize(offset / grid_da(g));
    if (g->clamp_radial_end || g->clamp_index_rounding || g->clamp_radial_outside)
        if (r > (uint64_t)(g->n_radial - 1)) r = (uint64_t)(g->n_radial - 1);
    if (g->clamp_index_rounding || g->clamp_azimuthal_outside)
        if (a > (uint64_t)(g->n_azimuthal - 1)) a = (uint64_t)(g->n_azimuthal - 1);
    if (r < (uint64_t)g->n_radial && a < (uint64_t)g->n_azimuthal)
        return (int64_t)(a * (uint64_t)g->n_radial + r);
    return -1;
}

/* Radial and azimuthal extremes of the hull grid (lut/common.rs:33-65). */
static int hull_extremes(const or_poni *p, int64_t dim1, int64_t dim2, int64_t n_ss, int unit,
                         double *rlo, double *rhi, double *alo, double *ahi) {
    int64_t hn = 2 * (dim1 + dim2) * n_ss;
    double *hd1 = (double *)malloc((size_t)hn * sizeof(double));
    double *hd2 = (double *)malloc((size_t)hn * sizeof(double));
    double *ht = (double *)malloc((size_t)hn * sizeof(double));
    double *hc = (double *)malloc((size_t)hn * sizeof(double));
    if (!hd1 || !hd2 || !ht || !hc) {
        free(hd1);
        free(hd2);
        free(ht);
        free(hc);
        return -1;
    }
    int64_t m = hull_grid(dim1, dim2, n_ss, hd1, hd2);
    or_tth_chi_at(p, hd1, hd2, m, ht, hc);
    for (int64_t i = 0; i < m; ++i) ht[i] = or_convert_unit(unit, p->wavelength, ht[i]);
    *rlo = seq_min(ht, m);
    *rhi = seq_max(ht, m);
    *alo = seq_min(hc, m);
    *ahi = seq_max(hc, m);
    free(hd1);
    free(hd2);
    free(ht);
    free(hc);
    return 0;
}

/* The grid prepare_cuda2d uses (cuda.rs:1111-1157 via device.rs:2502 and
 * the shared-grid key of methods.rs:365-388): explicit or default radial
 * edges (default_radial_edges_2d, grid.rs:975-1028), explicit or default
 * azimuthal edges (default_azimuthal_edges_2d, grid.rs:700-755; (-pi, pi)
 * for pyfai_full), index-rounding clamps, then per method: pyFAI histogram
 * mode, the counting radial end, the supersampled outside clamps
 * (azimuthal_range_grid, grid.rs:579-624). Returns 0 or -1. */
int or_grid2d_for(const or_poni *p, int64_t dim1, int64_t dim2, int method, int64_t n_ss,
                  int unit, int64_t nr, int64_t na, int has_rr, double rmin, double rmax,
                  int has_ar, double amin, double amax, or_grid2d *g) {
    int64_t npix = dim1 * dim2, ncorner = (dim1 + 1) * (dim2 + 1);
    double *cr = (double *)malloc((size_t)npix * sizeof(double));
    double *cc = (double *)malloc((size_t)npix * sizeof(double));
    double *rc = (double *)malloc((size_t)ncorner * sizeof(double));
    double *ac = (double *)malloc((size_t)ncorner * sizeof(double));
    int rc_ = -1;
    if (!cr || !cc || !rc || !ac) goto done;
    or_centres(p, dim1, dim2, unit, 0, 0.0, NULL, cr, cc, NULL, NULL, NULL);
    or_corners(p, dim1, dim2, unit, rc, ac);
    double r0, r1, a0, a1;
    if (has_rr) {
        r0 = rmin;
        r1 = rmax;
    } else if (method == 0) {
        r0 = seq_min(cr, npix);
        r1 = seq_max(cr, npix) + 10.0 * OR_EPS;
    } else if (method == 1) {
        r0 = seq_min(rc, ncorner);
        r1 = seq_max(rc, ncorner) + 10.0 * OR_EPS;
    } else if (method == 2) {
        or_pyfai_radial_range(p, dim1, dim2, unit, &r0, &r1);
    } else {
        double hlo, hhi, alo, ahi;
        if (hull_extremes(p, dim1, dim2, n_ss, unit, &hlo, &hhi, &alo, &ahi)) goto done;
        double a = seq_min(cr, npix), b = seq_max(cr, npix);
        r0 = hlo < a ? hlo : a;
        r1 = (hhi > b ? hhi : b) + 3.0 * OR_EPS;
    }
    if (has_ar) {
        a0 = amin;
        a1 = amax;
    } else if (method == 2) {
        a0 = -OR_PI;
        a1 = OR_PI;
    } else {
        if (method == 0) {
            a0 = seq_min(cc, npix);
            a1 = seq_max(cc, npix) + 10.0 * OR_EPS;
        } else if (method == 3) {
            double hlo, hhi, alo, ahi;
            if (hull_extremes(p, dim1, dim2, n_ss, unit, &hlo, &hhi, &alo, &ahi)) goto done;
            double a = seq_min(cc, npix), b = seq_max(cc, npix);
            a0 = alo < a ? alo : a;
            a1 = (ahi > b ? ahi : b) + 3.0 * OR_EPS;
        } else {
            a0 = seq_min(ac, ncorner);
            a1 = seq_max(ac, ncorner) + 10.0 * OR_EPS;
        }
        if (!(a1 - a0 > 1e-12)) {
            a0 = -OR_PI;
            a1 = OR_PI;
        }
    }
    if (or_grid2d_new(nr, na, r0, r1, a0, a1, g)) goto done;
    g->clamp_index_rounding = 1;
    if (method == 2) g->pyfai = 1;
    else if (!has_rr && method == 0) g->clamp_radial_end = 1;
    else if (!has_rr && method == 3) g->clamp_radial_outside = 1;
    if (method == 3 && !has_ar) g->clamp_azimuthal_outside = 1;
    rc_ = 0;
done:
    free(cr);
    free(cc);
    free(rc);
    free(ac);
    return rc_;
}

/* (bin, weight) list of one pixel; repeated bins add up (shared_grid.rs). */
typedef struct {
    int64_t *bin;
    double *w;
    int64_t n, cap;
} entries_t;

static int entries_add(entries_t *e, int64_t bin, double w) {
    for (int64_t k = 0; k < e->n; ++k)
        if (e->bin[k] == bin) {
            e->w[k] += w;
            return 0;
        }
    if (e->n == e->cap) {
        int64_t cap = e->cap ? 2 * e->cap : 16;
        int64_t *b = (int64_t *)realloc(e->bin, (size_t)cap * sizeof(int64_t));
        if (!b) return -1;
        e->bin = b;
        double *w2 = (double *)realloc(e->w, (size_t)cap * sizeof(double));
        if (!w2) return -1;
        e->w = w2;
        e->cap = cap;
    }
    e->bin[e->n] = bin;
    e->w[e->n] = w;
    e->n++;
    return 0;
}

/* sample_pixel (shared_grid.rs:202-232), n_ss = 128 with four offsets:
 * detector-plane samples binned on the grid, weight 1/65536 each. */
static int sample_pixel_2d(const or_poni *p, int64_t dim2, int64_t pixel, int unit,
                           const or_grid2d *g, entries_t *e) {
    const int64_t n_ss = 128;
    static const double off[4][2] = {{0.25, 0.5}, {0.5, 0.25}, {0.75, 0.5}, {0.5, 0.75}};
    const double weight = 1.0 / ((double)(n_ss * n_ss) * 4.0);
    trig_t t = trig_of(p);
    int64_t row = pixel / dim2, col = pixel % dim2;
    for (int64_t i = 0; i < n_ss; ++i)
        for (int64_t j = 0; j < n_ss; ++j)
            for (int o = 0; o < 4; ++o) {
                double d1 = (double)row + ((double)i + off[o][0]) / (double)n_ss;
                double d2 = ((double)(col * n_ss + j) + off[o][1]) / (double)n_ss;
                double a = d1 * p->pixel1 - p->poni1;
                double b = d2 * p->pixel2 - p->poni2;
                double x = f_x1(a, b, p->distance, &t);
                double y = f_x2(a, b, p->distance, &t);
                double z = f_x3(a, b, p->distance, &t);
                double r = or_convert_unit(unit, p->wavelength, f_tth(x, y, z));
                int64_t bin = or_grid2d_bin(g, r, f_azimuth(x, y));
                if (bin >= 0 && entries_add(e, bin, weight)) return -1;
            }
    return 0;
}

/* split_polygon (shared_grid.rs:152-200): clip against every bin rectangle of
 * the three periodic copies (-2pi, 0, +2pi) of the polygon. */
static int split_polygon_2d(const pt_t poly[4], double area, const or_grid2d *g, entries_t *e) {
    double r0 = g->r0, a0 = g->a0, dr = grid_dr(g), da = grid_da(g);
    double rmn = INFINITY, rmx = -INFINITY;
    for (int i = 0; i < 4; ++i) {
        rmn = fmin(rmn, poly[i].x);
        rmx = fmax(rmx, poly[i].x);
    }
    int64_t rs = as_isize(floor((rmn - r0) / dr));
    if (rs < 0) rs = 0;
    int64_t re = as_isize(floor((rmx - r0) / dr));
    if (re > g->n_radial - 1) re = g->n_radial - 1;
    pt_t buf1[64], buf2[64];
    const double shifts[3] = {-OR_TAU, 0.0, OR_TAU};
    for (int sh = 0; sh < 3; ++sh) {
        pt_t q[4];
        double amn = INFINITY, amx = -INFINITY;
        for (int i = 0; i < 4; ++i) {
            q[i].x = poly[i].x;
            q[i].y = poly[i].y + shifts[sh];
            amn = fmin(amn, q[i].y);
            amx = fmax(amx, q[i].y);
        }
        int64_t as_ = as_isize(floor((amn - a0) / da));
        if (as_ < 0) as_ = 0;
        int64_t ae = as_isize(floor((amx - a0) / da));
        if (ae > g->n_azimuthal - 1) ae = g->n_azimuthal - 1;
        for (int64_t ar = as_; ar <= ae; ++ar)
            for (int64_t rr = rs; rr <= re; ++rr) {
                double r = r0 + (double)rr * dr;
                double a = a0 + (double)ar * da;
                const pt_t *clipped;
                int m = clip_rect(q, 4, r, r + dr, a, a + da, buf1, buf2, &clipped);
                double w = fabs(polygon_area(clipped, m)) / area;
                if (w > 0.0 && entries_add(e, ar * g->n_radial + rr, w)) return -1;
            }
    }
    return 0;
}

/* line (pyfai_split.rs:146-168): one contour edge's signed area, rasterised
 * into azimuthal rows in strips of one radial column. */
static void pyfai_line(float *buffer, int64_t stride, pt_t start, pt_t stop) {
    if (start.x == stop.x) return;
    float slope = (float)((stop.y - start.y) / (stop.x - start.x));
    float intercept = (float)(stop.y - (double)slope * stop.x);
    double lo = fmin(start.x, stop.x), hi = fmax(start.x, stop.x);
    double sign = stop.x > start.x ? 1.0 : -1.0;
    uint64_t rb = as_usize(floor(lo)), re = as_usize(ceil(hi));
    for (uint64_t r = rb; r < re; ++r) {
        double left = fmax(lo, (double)r), right = fmin(hi, (double)(r + 1));
        float area =
            (float)(sign * (right - left) * (0.5 * (double)slope * (right + left) + (double)intercept));
        float width = (float)(right - left);
        float remaining = fabsf(area);
        for (int64_t a = 0; a < stride; ++a) {
            if (remaining <= 0.0f) break;
            float increment = fminf(width, remaining);
            buffer[(int64_t)r * stride + a] += copysignf(increment, area);
            remaining -= increment;
        }
    }
}

/* pyfai_split::split (pyfai_split.rs:35-144); poly in pyFAI order (top-left,
 * bottom-left, bottom-right, top-right) with raw angles. Returns the number
 * of entries, -1 for None (the caller falls back to fractional clipping),
 * -2 when the raster exceeds the oracle's buffer. */
int or_pyfai_split2d(const double *poly_in, const or_grid2d *g, double sign, int64_t *bins,
                     double *weights, int64_t cap) {
    pt_t poly[4];
    for (int i = 0; i < 4; ++i) {
        poly[i].x = poly_in[2 * i];
        poly[i].y = poly_in[2 * i + 1];
    }
    double a0 = g->a0, a1 = g->a1, r0 = g->r0, r1 = g->r1;
    double canonical = (a0 >= -OR_PI && a1 <= OR_PI) ? -OR_PI : (a0 >= 0.0 && a1 <= OR_TAU) ? 0.0 : a0;
    double offset = canonical + OR_PI;
    for (int i = 0; i < 4; ++i) poly[i].y = wrap_tau(poly[i].y - offset + OR_PI) - OR_PI;
    pt_t a = poly[0], b = poly[1], c = poly[2], d = poly[3];
    double area = sign * (0.5 * (c.x - a.x) * (d.y - b.y) - (c.y - a.y) * (d.x - b.x));
    if (area > 0.0) {
        for (int i = 0; i < 4; ++i)
            if (poly[i].y < 0.0) poly[i].y += OR_TAU;
        double s = -0.0;
        for (int i = 0; i < 4; ++i) s += poly[i].y;
        if (s * 0.25 > OR_PI)
            for (int i = 0; i < 4; ++i) poly[i].y -= OR_TAU;
    }
    for (int i = 0; i < 4; ++i) poly[i].y += offset;
    int all_lo_r = 1, all_hi_r = 1, all_lo_a = 1, all_hi_a = 1;
    for (int i = 0; i < 4; ++i) {
        all_lo_r &= poly[i].x < r0;
        all_hi_r &= poly[i].x > r1;
        all_lo_a &= poly[i].y < a0;
        all_hi_a &= poly[i].y > a1;
    }
    if (all_lo_r || all_hi_r || all_lo_a || all_hi_a) return 0;
    double dr = grid_dr(g), da = grid_da(g);
    for (int i = 0; i < 4; ++i) {
        poly[i].x = (clampd(poly[i].x, r0, r1) - r0) / dr;
        poly[i].y = (clampd(poly[i].y, a0, a1) - a0) / da;
    }
    double mr = INFINITY, ma = INFINITY;
    for (int i = 0; i < 4; ++i) {
        mr = fmin(mr, poly[i].x);
        ma = fmin(ma, poly[i].y);
    }
    uint64_t ir = as_usize(floor(mr)), ia = as_usize(floor(ma));
    for (int i = 0; i < 4; ++i) {
        poly[i].x -= (double)ir;
        poly[i].y -= (double)ia;
    }
    double xr = 0.0, xa = 0.0;
    for (int i = 0; i < 4; ++i) {
        xr = fmax(xr, poly[i].x);
        xa = fmax(xa, poly[i].y);
    }
    uint64_t nr = as_usize(ceil(xr)), na = as_usize(ceil(xa));
    if (nr == 0 || na == 0) return -1;
    if ((nr + 1) * (na + 1) > 4096) return -2;
    float buffer[4096];
    for (uint64_t k = 0; k < (nr + 1) * (na + 1); ++k) buffer[k] = 0.0f;
    for (int i = 0; i < 4; ++i) pyfai_line(buffer, (int64_t)(na + 1), poly[i], poly[(i + 1) % 4]);
    int64_t m = 0;
    double total = 0.0;
    for (uint64_t r = 0; r < nr; ++r)
        for (uint64_t q = 0; q < na; ++q) {
            double value = sign * (double)buffer[r * (na + 1) + q];
            if (!isfinite(value)) return -1;
            if (value > 0.0 && ir + r < (uint64_t)g->n_radial && ia + q < (uint64_t)g->n_azimuthal) {
                if (m >= cap) return -2;
                bins[m] = (int64_t)((ia + q) * (uint64_t)g->n_radial + ir + r);
                weights[m] = value;
                total += value;
                ++m;
            }
        }
    if (total <= 0.0) return -1;
    for (int64_t k = 0; k < m; ++k) weights[k] /= total;
    return (int)m;
}

/* shared_grid::build (shared_grid.rs:13-150) and, for supersampling,
 * build_shared_grid_ss_csr through the exact counted path
 * (supersampled.rs:1437-1477, :21-104 with normalize_bins false): per pixel
 * entries, then rows filled in pixel order. method 0 counting, 1 pixel
 * split (fractional), 2 pyfai_full (pyFAI histogram mode), 3 supersampled. */
int or_build_2d(const or_poni *p, int64_t dim1, int64_t dim2, int method, int64_t n_ss,
                int unit, const or_grid2d *g, or_lut *out) {
    int64_t npix = dim1 * dim2, ncorner = (dim1 + 1) * (dim2 + 1);
    int64_t nb = g->n_radial * g->n_azimuthal;
    double *cr = (double *)malloc((size_t)npix * sizeof(double));
    double *cc = (double *)malloc((size_t)npix * sizeof(double));
    double *rc = (double *)malloc((size_t)ncorner * sizeof(double));
    double *ac = (double *)malloc((size_t)ncorner * sizeof(double));
    bucket_t *buckets = (bucket_t *)calloc((size_t)nb, sizeof(bucket_t));
    entries_t e = {0};
    int64_t pb[4096];
    double pw[4096];
    int rc_ = -1;
    if (!cr || !cc || !rc || !ac || !buckets) goto done;
    or_centres(p, dim1, dim2, unit, 0, 0.0, NULL, cr, cc, NULL, NULL, NULL);
    or_corners(p, dim1, dim2, unit, rc, ac);
    trig_t t = trig_of(p);
    const int64_t w = dim2 + 1;
    rc_ = 0;
    for (int64_t pixel = 0; pixel < npix && rc_ == 0; ++pixel) {
        e.n = 0;
        if (method == 0) {
            int64_t bin = or_grid2d_bin(g, cr[pixel], cc[pixel]);
            if (bin >= 0 && entries_add(&e, bin, 1.0)) rc_ = -1;
        } else if (method == 3) {
            int64_t row = pixel / dim2, col = pixel % dim2;
            int64_t cb[256], cn[256];
            int nc = 0;
            for (int64_t i = 0; i < n_ss; ++i) {
                double d1 = (double)row + ((double)i + 0.5) / (double)n_ss;
                for (int64_t j = 0; j < n_ss; ++j) {
                    double d2 = ((double)(col * n_ss + j) + 0.5) / (double)n_ss;
                    double a = d1 * p->pixel1 - p->poni1;
                    double bb = d2 * p->pixel2 - p->poni2;
                    double x = f_x1(a, bb, p->distance, &t);
                    double y = f_x2(a, bb, p->distance, &t);
                    double z = f_x3(a, bb, p->distance, &t);
                    double r = or_convert_unit(unit, p->wavelength, f_tth(x, y, z));
                    int64_t bin = or_grid2d_bin(g, r, f_azimuth(x, y));
                    if (bin < 0) continue;
                    int f = -1;
                    for (int q = 0; q < nc; ++q)
                        if (cb[q] == bin) {
                            f = q;
                            break;
                        }
                    if (f < 0) {
                        cb[nc] = bin;
                        cn[nc++] = 1;
                    } else {
                        cn[f]++;
                    }
                }
            }
            for (int q = 0; q < nc && rc_ == 0; ++q)
                if (entries_add(&e, cb[q], (double)cn[q] / (double)(n_ss * n_ss))) rc_ = -1;
        } else {
            int64_t b0 = pixel / dim2 * w + pixel % dim2;
            int64_t idx[4] = {b0, b0 + 1, b0 + w + 1, b0 + w};
            int axis_on_edge = 0, has_zero = 0;
            double winding = 0.0;
            for (int i = 0; i < 4; ++i) {
                double delta = ac[idx[(i + 1) % 4]] - ac[idx[i]];
                delta = rem_euclid_tau(delta + OR_PI) - OR_PI;
                if (fabs(delta) >= OR_PI - 64.0 * OR_EPS) axis_on_edge = 1;
                winding += delta;
                if (rc[idx[i]] == 0.0) has_zero = 1;
            }
            if (fabs(winding) > OR_PI || axis_on_edge || has_zero) {
                if (sample_pixel_2d(p, dim2, pixel, unit, g, &e)) rc_ = -1;
            } else {
                int done_pixel = 0;
                if (g->pyfai) {
                    double poly[8] = {rc[idx[0]], ac[idx[0]], rc[idx[3]], ac[idx[3]],
                                      rc[idx[2]], ac[idx[2]], rc[idx[1]], ac[idx[1]]};
                    int m = or_pyfai_split2d(poly, g, 1.0, pb, pw, 4096);
                    if (m == -2) {
                        rc_ = -1;
                    } else if (m >= 0) {
                        for (int k = 0; k < m && rc_ == 0; ++k)
                            if (entries_add(&e, pb[k], pw[k])) rc_ = -1;
                        done_pixel = 1;
                    }
                }
                if (!done_pixel && rc_ == 0) {
                    double center = g->a0 + rem_euclid_tau(cc[pixel] - g->a0);
                    pt_t poly[4];
                    for (int i = 0; i < 4; ++i) {
                        poly[i].x = rc[idx[i]];
                        poly[i].y = center + rem_euclid_tau(ac[idx[i]] - center + OR_PI) - OR_PI;
                    }
                    double area = fabs(polygon_area(poly, 4));
                    if (area > 0.0) {
                        if (split_polygon_2d(poly, area, g, &e)) rc_ = -1;
                    } else {
                        int64_t bin = or_grid2d_bin(g, cr[pixel], cc[pixel]);
                        if (bin >= 0 && entries_add(&e, bin, 1.0)) rc_ = -1;
                    }
                }
            }
        }
        for (int64_t k = 0; k < e.n && rc_ == 0; ++k)
            if (bucket_push(&buckets[e.bin[k]], pixel, e.w[k])) rc_ = -1;
    }
    if (rc_ == 0) {
        rc_ = buckets_to_lut(buckets, nb, 1, g->r0, grid_dr(g), out);
        buckets = NULL;
    }
done:
    if (buckets) {
        for (int64_t i = 0; i < nb; ++i) {
            free(buckets[i].col);
            free(buckets[i].w);
        }
        free(buckets);
    }
    free(e.bin);
    free(e.w);
    free(cr);
    free(cc);
    free(rc);
    free(ac);
    return rc_;
}

/* fixed_table (prepared.rs:163-192). An all-zero mask keeps the table. */
int or_compact(const or_lut *in, const uint8_t *mask, or_lut *out) {
    memset(out, 0, sizeof(*out));
    out->n_rows = in->n_rows;
    out->hist_min = in->hist_min;
    out->hist_step = in->hist_step;
    out->row_ptr = (int64_t *)calloc((size_t)in->n_rows + 1, sizeof(int64_t));
    out->col = (int64_t *)malloc((size_t)(in->nnz ? in->nnz : 1) * sizeof(int64_t));
    if (in->w) out->w = (double *)malloc((size_t)(in->nnz ? in->nnz : 1) * sizeof(double));
    if (!out->row_ptr || !out->col || (in->w && !out->w)) return -1;
    int64_t m = 0;
    for (int64_t r = 0; r < in->n_rows; ++r) {
        for (int64_t k = in->row_ptr[r]; k < in->row_ptr[r + 1]; ++k) {
            int64_t j = in->col[k];
            if (mask && mask[j]) continue;
            out->col[m] = j;
            if (in->w) out->w[m] = in->w[k];
            ++m;
        }
        out->row_ptr[r + 1] = m;
    }
    out->nnz = m;
    return 0;
}

/* normalization::<false> (prepared.rs:229-262) through row() with NORM and
 * no mask: n = n + w*x (weighted) or n + x (unweighted), sequential. */
void or_denominators(const or_lut *lut, const double *norm, double *den) {
    for (int64_t r = 0; r < lut->n_rows; ++r) {
        double n = 0.0;
        for (int64_t k = lut->row_ptr[r]; k < lut->row_ptr[r + 1]; ++k) {
            double x = norm[lut->col[k]];
            n = lut->w ? n + lut->w[k] * x : n + x;
        }
        den[r] = n;
    }
}

/* row() strict (prepared.rs:1011-1118): s = s + w*x; v = v + w*w*max(x, 0). */
void or_row_sums(const or_lut *lut, const double *signal, double *ss, double *vv) {
    for (int64_t r = 0; r < lut->n_rows; ++r) {
        double s = 0.0, v = 0.0;
        for (int64_t k = lut->row_ptr[r]; k < lut->row_ptr[r + 1]; ++k) {
            double x = signal[lut->col[k]];
            double var = x > 0.0 ? x : 0.0; /* f64::max(x, 0.0), x never NaN-sensitive here */
            if (x != x) var = 0.0;          /* f64::max ignores NaN */
            if (lut->w) {
                double w = lut->w[k];
                s = s + w * x;
                v = v + w * w * var;
            } else {
                s += x;
                v += var;
            }
        }
        if (ss) ss[r] = s;
        if (vv) vv[r] = v;
    }
}

/* normalize_bin (prepared.rs:985-996). */
static inline void normalize_bin(double s, double n, double v, double *y, double *e) {
    *y = n == 0.0 ? 0.0 : s / n;
    double q = n == 0.0 ? 0.0 : v / (n * n);
    if (!(q >= 0.0)) q = (q != q) ? q : 0.0; /* f64::max(q, 0.0): NaN -> 0 */
    if (q != q) q = 0.0;
    *e = sqrt(q);
}

void or_integrate_strict(const or_lut *lut, const double *den, const double *signal, int errors,
                         double *intensity, double *sigma) {
    for (int64_t r = 0; r < lut->n_rows; ++r) {
        double s = 0.0, v = 0.0;
        for (int64_t k = lut->row_ptr[r]; k < lut->row_ptr[r + 1]; ++k) {
            double x = signal[lut->col[k]];
            double var = (x != x) ? 0.0 : (x > 0.0 ? x : 0.0);
            if (lut->w) {
                double w = lut->w[k];
                s = s + w * x;
                if (errors) v = v + w * w * var;
            } else {
                s += x;
                if (errors) v += var;
            }
        }
        double y, e;
        normalize_bin(s, den[r], v, &y, &e);
        intensity[r] = y;
        if (errors && sigma) sigma[r] = e;
    }
}

/* Raw per-row sums with a mask check, strict sequential order: row()
 * (prepared.rs:1011-1118) with SIGNAL, NORM, VAR and COUNT; an entry whose
 * pixel has a nonzero mask byte is skipped. S = sum w*s, N = sum w*norm,
 * V = sum w*w*max(s, 0) (f64::max: a NaN signal gives 0), C = sum w. */
void or_raw_sums(const or_lut *lut, const uint8_t *mask, const double *norm,
                 const double *signal, double *out_s, double *out_n, double *out_v,
                 double *out_c) {
    for (int64_t r = 0; r < lut->n_rows; ++r) {
        double s = 0.0, n = 0.0, v = 0.0, c = 0.0;
        for (int64_t k = lut->row_ptr[r]; k < lut->row_ptr[r + 1]; ++k) {
            int64_t j = lut->col[k];
            if (mask && mask[j]) continue;
            double w = lut->w ? lut->w[k] : 1.0, x = signal[j];
            double var = (x != x) ? 0.0 : (x > 0.0 ? x : 0.0);
            s = s + w * x;
            v = v + w * w * var;
            n = n + w * norm[j];
            c += w;
        }
        out_s[r] = s;
        out_n[r] = n;
        out_v[r] = v;
        out_c[r] = c;
    }
}

/* integrate_with_columns (azimuthal.rs:48-118). */
void or_azimuthal_std(const or_lut *lut, const uint8_t *mask, const double *norm,
                      const double *signal, const double *variance, double *intensity,
                      double *errors, double *spread) {
    for (int64_t r = 0; r < lut->n_rows; ++r) {
        int have = 0;
        double origin = 0.0;
        double ssig = 0.0, sw = 0.0, ssh = 0.0, sv = 0.0;
        for (int64_t k = lut->row_ptr[r]; k < lut->row_ptr[r + 1]; ++k) {
            int64_t j = lut->col[k];
            if (mask && mask[j]) continue;
            double n = norm[j], c = lut->w ? lut->w[k] : 1.0, s = signal[j];
            double x = s / n, w = c * n;
            if (!(isfinite(s) && isfinite(n) && n > 0.0 && isfinite(c) && c > 0.0 && isfinite(x) &&
                  isfinite(w) && w > 0.0))
                continue;
            if (!have) {
                have = 1;
                origin = x;
            }
            ssig += c * s;
            sw += w;
            ssh += w * (x - origin);
            if (variance) sv += c * c * variance[j];
        }
        if (!have) {
            intensity[r] = 0.0;
            if (errors) errors[r] = 0.0;
            spread[r] = NAN;
            continue;
        }
        double mean_shifted = ssh / sw;
        double m2 = -0.0;
        for (int64_t k = lut->row_ptr[r]; k < lut->row_ptr[r + 1]; ++k) {
            int64_t j = lut->col[k];
            if (mask && mask[j]) continue;
            double n = norm[j], c = lut->w ? lut->w[k] : 1.0, s = signal[j];
            double x = s / n, w = c * n;
            if (!(isfinite(s) && isfinite(n) && n > 0.0 && isfinite(c) && c > 0.0 && isfinite(x) &&
                  isfinite(w) && w > 0.0))
                continue;
            double delta = (x - origin) - mean_shifted;
            m2 += w * delta * delta;
        }
        intensity[r] = ssig / sw;
        if (errors) errors[r] = sqrt(sv > 0.0 ? sv : 0.0) / sw;
        double q = m2 / sw;
        spread[r] = sqrt(q > 0.0 ? q : 0.0);
    }
}

/* --------------------------------------------------- threaded CPU baseline */

typedef struct {
    const or_lut *table, *full;
    const double *den, *norm;
    const uint8_t *mask;
    const void *frames;
    int dtype, errors, astd;
    int64_t npix, first, last;
    double *oi, *os, *od;
    int status;
} job_t;

static void *frames_worker(void *arg) {
    job_t *j = (job_t *)arg;
    int64_t nb = j->table->n_rows;
    double *sig = (double *)malloc((size_t)j->npix * sizeof(double));
    double *var = j->errors ? (double *)malloc((size_t)j->npix * sizeof(double)) : NULL;
    if (!sig || (j->errors && !var)) {
        j->status = -1;
        free(sig);
        free(var);
        return NULL;
    }
    for (int64_t f = j->first; f < j->last; ++f) {
        /* Pixel::to_f64 (frame.rs:13-22) */
        for (int64_t i = 0; i < j->npix; ++i) {
            int64_t at = f * j->npix + i;
            switch (j->dtype) {
            case 0: sig[i] = (double)((const uint16_t *)j->frames)[at]; break;
            case 1: sig[i] = (double)((const uint32_t *)j->frames)[at]; break;
            case 2: sig[i] = (double)((const int32_t *)j->frames)[at]; break;
            case 3: sig[i] = (double)((const float *)j->frames)[at]; break;
            default: sig[i] = ((const double *)j->frames)[at]; break;
            }
        }
        double *oi = j->oi + f * nb;
        double *os = j->os ? j->os + f * nb : NULL;
        if (j->astd) {
            if (var)
                for (int64_t i = 0; i < j->npix; ++i) var[i] = sig[i] > 0.0 ? sig[i] : 0.0;
            or_azimuthal_std(j->full, j->mask, j->norm, sig, var, oi, os, j->od + f * nb);
        } else {
            or_integrate_strict(j->table, j->den, sig, j->errors, oi, os);
        }
    }
    free(sig);
    free(var);
    return NULL;
}

int or_integrate_frames_mt(const or_lut *table, const double *den, const or_lut *full,
                           const uint8_t *mask, const double *norm, const void *frames, int dtype,
                           int64_t npix, int64_t n_frames, int errors, int azimuthal_std,
                           int threads, double *out_i, double *out_sigma, double *out_std) {
    if (threads < 1) threads = 1;
    if (threads > n_frames) threads = (int)(n_frames ? n_frames : 1);
    pthread_t *tid = (pthread_t *)malloc((size_t)threads * sizeof(pthread_t));
    job_t *jobs = (job_t *)calloc((size_t)threads, sizeof(job_t));
    if (!tid || !jobs) {
        free(tid);
        free(jobs);
        return -1;
    }
    int64_t per = (n_frames + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        job_t *j = &jobs[t];
        j->table = table;
        j->full = full;
        j->den = den;
        j->norm = norm;
        j->mask = mask;
        j->frames = frames;
        j->dtype = dtype;
        j->errors = errors;
        j->astd = azimuthal_std;
        j->npix = npix;
        j->first = (int64_t)t * per;
        j->last = j->first + per < n_frames ? j->first + per : n_frames;
        if (j->first > j->last) j->first = j->last;
        j->oi = out_i;
        j->os = out_sigma;
        j->od = out_std;
        pthread_create(&tid[t], NULL, frames_worker, j);
    }
    int status = 0;
    for (int t = 0; t < threads; ++t) {
        pthread_join(tid[t], NULL);
        if (jobs[t].status) status = -1;
    }
    free(tid);
    free(jobs);
    return status;
}

/* ================================================== Bitshuffle + LZ4 chunks */

static uint64_t be64(const uint8_t *p) {
    uint64_t v = 0;
    for (int i = 0; i < 8; ++i) v = (v << 8) | p[i];
    return v;
}
static uint32_t be32(const uint8_t *p) {
    return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}

/* One LZ4 block (the published LZ4 block format: sequences of a token,
 * literal length with 255-extensions, literals, a 2-byte little-endian
 * offset, a match length of (token & 15) + 4 with 255-extensions; the last
 * sequence has literals only). Returns the decoded length or -1. */
static int64_t lz4_block_decode(const uint8_t *in, int64_t n, uint8_t *out, int64_t cap) {
    int64_t ip = 0, op = 0;
    while (ip < n) {
        unsigned token = in[ip++];
        int64_t lit = token >> 4;
        if (lit == 15) {
            unsigned s;
            do {
                if (ip >= n) return -1;
                s = in[ip++];
                lit += s;
            } while (s == 255);
        }
        if (lit > n - ip || lit > cap - op) return -1;
        memcpy(out + op, in + ip, (size_t)lit);
        ip += lit;
        op += lit;
        if (ip >= n) break; /* last sequence: literals only */
        if (ip + 2 > n) return -1;
        int64_t offset = (int64_t)in[ip] | ((int64_t)in[ip + 1] << 8);
        ip += 2;
        if (offset == 0 || offset > op) return -1;
        int64_t mlen = (token & 15) + 4;
        if ((token & 15) == 15) {
            unsigned s;
            do {
                if (ip >= n) return -1;
                s = in[ip++];
                mlen += s;
            } while (s == 255);
        }
        if (mlen > cap - op) return -1;
        for (int64_t k = 0; k < mlen; ++k) out[op + k] = out[op + k - offset];
        op += mlen;
    }
    return op;
}

/* Inverse bitshuffle of count elements (count a multiple of 8): plane p
 * (bit p of an element, least significant first) holds count/8 bytes whose
 * bit i of byte k is bit p of element 8k + i. Elements are little-endian. */
static void bitunshuffle(const uint8_t *in, int64_t count, int elem_bytes, uint8_t *out) {
    int64_t plane = count / 8;
    memset(out, 0, (size_t)(count * elem_bytes));
    for (int p = 0; p < 8 * elem_bytes; ++p)
        for (int64_t e = 0; e < count; ++e)
            if ((in[p * plane + e / 8] >> (e % 8)) & 1)
                out[e * elem_bytes + p / 8] |= (uint8_t)(1u << (p % 8));
}

/* A Bitshuffle/LZ4 chunk as HDF5's bitshuffle filter writes it
 * (device.rs:2062-2140 reads the same layout): big-endian u64 uncompressed
 * bytes and u32 block bytes (0: 8192); every full block and then the
 * remainder rounded down to 8 elements as a big-endian u32 compressed length
 * and an LZ4 block of the bitshuffled elements; the last (< 8) elements
 * verbatim. Decodes n_elems elements into out. 0, or -1 on malformed input. */
int or_bslz4_decode(const uint8_t *chunk, int64_t len, int elem_bytes, int64_t n_elems,
                    uint8_t *out) {
    if (len < 12) return -1;
    uint64_t total = be64(chunk);
    if (total != (uint64_t)(n_elems * elem_bytes)) return -1;
    int64_t block = be32(chunk + 8);
    if (block == 0) block = 8192;
    if (block % (8 * elem_bytes)) return -1;
    int64_t block_elems = block / elem_bytes;
    int64_t n_full = n_elems / block_elems, rem = n_elems % block_elems;
    int64_t rem_comp = rem / 8 * 8, tail = rem % 8;
    uint8_t *tmp = (uint8_t *)malloc((size_t)block);
    if (!tmp) return -1;
    int64_t off = 12;
    int rc = 0;
    for (int64_t b = 0; b <= n_full && rc == 0; ++b) {
        int64_t elems = b < n_full ? block_elems : rem_comp;
        if (elems == 0) break;
        if (off + 4 > len) { rc = -1; break; }
        int64_t clen = be32(chunk + off);
        off += 4;
        if (clen > len - off) { rc = -1; break; }
        int64_t got = lz4_block_decode(chunk + off, clen, tmp, elems * elem_bytes);
        if (got != elems * elem_bytes) { rc = -1; break; }
        bitunshuffle(tmp, elems, elem_bytes, out + b * block_elems * elem_bytes);
        off += clen;
    }
    if (rc == 0 && tail) {
        int64_t raw = tail * elem_bytes;
        if (off + raw > len) rc = -1;
        else memcpy(out + (n_full * block_elems + rem_comp) * elem_bytes, chunk + off, (size_t)raw);
    }
    free(tmp);
    return rc;
}
