/*
 * CPU oracle for the lookup-table (CSR) integration path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference
 * crate's CPU algorithm (geometry, bin grids, CSR builders, mask compaction,
 * strict f64 row gather and the azimuthal spread), compiled with
 * -O2 -ffp-contract=off -fno-fast-math against glibc libm so that it performs
 * the same IEEE-754 operations in the same order as the Rust code. Only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark may call it;
 * the product library never links or loads it.
 *
 * Parity status: pinned against the reference's own golden vectors
 * (the geometry vectors in test_data/test_reference) and against the known
 * answers in the reference's unit tests (counting CSR, pixel-split fractions,
 * azimuthal spread, normalisation). See tests/test_oracle_golden.py.
 */
#ifndef DIOPTRIN_ORACLE_H
#define DIOPTRIN_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_poni {
    double pixel1, pixel2, distance, poni1, poni2, rot1, rot2, rot3, wavelength;
} or_poni;

enum { OR_UNIT_TTH_RAD = 0, OR_UNIT_TTH_DEG = 1, OR_UNIT_Q_A = 2, OR_UNIT_Q_NM = 3 };

/* A CSR lookup table. `w == NULL` means unweighted (every entry weighs 1). */
typedef struct or_lut {
    int64_t n_rows;
    int64_t nnz;
    int64_t *row_ptr; /* n_rows + 1 */
    int64_t *col;     /* nnz */
    double *w;        /* nnz or NULL */
    double hist_min;
    double hist_step;
} or_lut;

void or_lut_free(or_lut *lut);

/* Sample-frame positions of pixel centres (geometry.rs:405-438). */
void or_sample_positions(const or_poni *p, int64_t dim1, int64_t dim2,
                         double *x, double *y, double *z);
/* Per-pixel centre arrays (corrections.rs:57-85). `has_pol == 0` gives pol = 1. */
void or_centres(const or_poni *p, int64_t dim1, int64_t dim2, int unit, int has_pol,
                double pol_factor, double *tth, double *radial, double *chi, double *sa,
                double *pol, double *norm);
/* Corner grid (dim1+1)*(dim2+1): radial (in `unit`) and chi (geometry.rs:229-278). */
void or_corners(const or_poni *p, int64_t dim1, int64_t dim2, int unit, double *radial,
                double *chi);
/* tth/chi at arbitrary detector coordinates (geometry.rs:519-549). */
void or_tth_chi_at(const or_poni *p, const double *d1, const double *d2, int64_t n,
                   double *tth, double *chi);
double or_convert_unit(int unit, double wavelength, double tth);

/* Bin grid helpers (histogram.rs:184-199). */
void or_min_max_step(const double *data, int64_t n, int64_t n_points, double *min,
                     double *max, double *step);
void or_bins(int64_t n_points, double min, double step, double *out);

/* PixelSplit 1D (pixel_split.rs:190-455). has_range selects _with_range. */
int or_build_ps1d(const or_poni *p, int64_t dim1, int64_t dim2, int unit, int64_t n_points,
                  int has_range, double rmin, double rmax, or_lut *out);
/* lut1d_ps_fractions with explicit (min, step, clamp_low), flattened to CSR. */
int or_ps1d_fractions(const or_poni *p, int64_t dim1, int64_t dim2, int unit,
                      int64_t n_points, double min, double step, int clamp_low,
                      or_lut *out);
/* Counting 1D (counting_csr.rs:54-134). */
/* pyFAI full splitting, 1D (pyfai_1d.rs:36-354). */
int or_split1d(const double *poly, int64_t n, double r0, double r1, double a0, double a1,
               int sector, double sign, int64_t *bins, double *weights, int64_t cap);
void or_pyfai_radial_range(const or_poni *p, int64_t dim1, int64_t dim2, int unit, double *lo,
                           double *hi);
int or_build_pf1d(const or_poni *p, int64_t dim1, int64_t dim2, int unit, int64_t n_points,
                  int has_range, double rmin, double rmax, or_lut *out);
/* 2D tables on an explicit grid (integration/grid.rs:26-222, shared_grid.rs,
 * pyfai_split.rs, supersampled.rs:1437-1477). */
typedef struct or_grid2d {
    int64_t n_radial, n_azimuthal;
    double r0, r1, a0, a1;
    int clamp_radial_end, clamp_index_rounding, clamp_radial_outside, clamp_azimuthal_outside;
    int pyfai; /* pyFAI histogram splitting (pyfai_full) */
} or_grid2d;
int or_grid2d_new(int64_t n_radial, int64_t n_azimuthal, double r0, double r1, double a0,
                  double a1, or_grid2d *g);
int64_t or_grid2d_bin(const or_grid2d *g, double radial, double azimuthal);
int or_grid2d_for(const or_poni *p, int64_t dim1, int64_t dim2, int method, int64_t n_ss,
                  int unit, int64_t n_radial, int64_t n_azimuthal, int has_radial_range,
                  double rmin, double rmax, int has_azimuthal_range, double amin, double amax,
                  or_grid2d *g);
int or_pyfai_split2d(const double *poly, const or_grid2d *g, double sign, int64_t *bins,
                     double *weights, int64_t cap);
int or_build_2d(const or_poni *p, int64_t dim1, int64_t dim2, int method, int64_t n_ss,
                int unit, const or_grid2d *g, or_lut *out);
/* Bitshuffle/LZ4 chunk decoding (HDF5 bitshuffle filter layout). */
int or_bslz4_decode(const uint8_t *chunk, int64_t len, int elem_bytes, int64_t n_elems,
                    uint8_t *out);
int or_build_counting1d(const double *radial, int64_t npix, int64_t n_points, int has_range,
                        double rmin, double rmax, or_lut *out);
/* Supersampled 1D (supersampled.rs:517-593), exact per-sample path. */
int or_build_ss1d(const or_poni *p, int64_t dim1, int64_t dim2, int unit, int64_t n_points,
                  int64_t n_ss, int has_range, double rmin, double rmax, or_lut *out);

/* Mask compaction (prepared.rs:163-192). mask != 0 drops the entry. */
int or_compact(const or_lut *in, const uint8_t *mask, or_lut *out);
/* Strict f64 denominators Σ w·norm (prepared.rs:229-262, row NORM path). */
void or_denominators(const or_lut *lut, const double *norm, double *den);
/* Strict f64 row gather + normalize_bin (prepared.rs:985-1118). */
void or_integrate_strict(const or_lut *lut, const double *den, const double *signal,
                         int errors, double *intensity, double *sigma);
void or_raw_sums(const or_lut *lut, const uint8_t *mask, const double *norm,
                 const double *signal, double *out_s, double *out_n, double *out_v,
                 double *out_c);
/* Raw strict sums S = Σ w·s and V = Σ w²·max(s,0) per row. */
void or_row_sums(const or_lut *lut, const double *signal, double *sum_signal,
                 double *sum_variance);
/* Weighted population spread (azimuthal.rs:48-118). variance may be NULL. */
void or_azimuthal_std(const or_lut *lut, const uint8_t *mask, const double *norm,
                      const double *signal, const double *variance, double *intensity,
                      double *errors, double *spread);

/* Multi-threaded CPU baseline: integrate `n_frames` frames of a typed dtype
 * (0=u16, 1=u32, 2=i32, 3=f32, 4=f64) on `threads` host threads, frames in
 * parallel (the reference's batch1d array path). `table` is the compacted
 * table with `den`; the spread uses `full` + `mask` + `norm`. */
int or_integrate_frames_mt(const or_lut *table, const double *den, const or_lut *full,
                           const uint8_t *mask, const double *norm, const void *frames,
                           int dtype, int64_t npix, int64_t n_frames, int errors,
                           int azimuthal_std, int threads, double *out_i, double *out_sigma,
                           double *out_std);

#ifdef __cplusplus
}
#endif
#endif
