/*
 * oracle.h -- FP64 CPU restatement of the MIDAS caking hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This code is the checker for the CUDA library
 * (libmidas_b200.so); only the tests, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference legs use it.  The product never calls it.
 *
 * Parity is pinned: tests/test_oracle_golden.py checks these functions against
 * golden vectors produced by the reference's own Python package
 * (packages/midas_integrate, generated by tests/golden/make_golden.py), and
 * against the reference's IntegrationCore.c compiled into oracle/_ref.
 */
#ifndef MIDAS_ORACLE_H
#define MIDAS_ORACLE_H
#include <stdint.h>

typedef struct {
  float y, z;
  double frac;
  float deltaR, areaWeight;
} or_record;

/* semantics: 0 = midas_integrate kernels.py, 1 = IntegratorFitPeaksGPUStream.cu, 2 = IntegrationCore.c,
 * 3 = IntegratorZarrOMP.c (the sums of 2, a nonzero sum divided by the whole area)
 * mode: 0 floor, 1 bilinear, 2 gradient
 * image: dark-subtracted frame, double, nz*ny (flat index z*ny + y)
 * cake_out: n_bins, area_out (may be NULL): normaliser per bin */
int or_integrate(const or_record *rec, const int32_t *nmap, int64_t n_bins, int ny, int nz,
                 double bc_y, double bc_z, const double *image, int mode, int semantics,
                 int normalize, double *cake_out, double *area_out);

/* in-bounds area per bin (kernels.py:306-311) */
void or_area_in(const or_record *rec, const int32_t *nmap, int64_t n_bins, int ny, int nz,
                double *area);

/* integrate_with_variance: var_cake = sum over pixels of (coalesced weight)^2 * var_image,
 * over the squared normaliser when normalising */
int or_integrate_var(const or_record *rec, const int32_t *nmap, int64_t n_bins, int ny, int nz,
                     double bc_y, double bc_z, const double *var_image, int mode, int sem, int normalize,
                     double *var_cake);

/* profile_1d: area-weighted (lo_aw) and simple-mean (lo_sm) eta reductions */
void or_profile(const double *cake, const double *area_in, int n_r, int n_eta, double *lo_aw,
                double *lo_sm);

/* the OpenMP integrator's lineout: mean of the nonzero, non-NaN bins of each row (lo_sm),
 * and the area-weighted mean over its valid, non-NaN bins (lo_aw) */
void or_profile_omp(const double *cake, const double *area_in, int n_r, int n_eta, double *lo_aw,
                    double *lo_sm);

/* one LM fit (same algorithm as the device fitter, in FP64).  model 0 = PV, 1 = TCH.
 * out: 11 doubles (layout of MI_FIT_NOUT).  Returns iterations, or <0 if rejected. */
int or_fit(const double *x, const double *y, int n_x, double peak, int half_window, int model,
           int max_iter, double x_bin, double px_um, double lsd_um, double *out);

/* fitPeaksAutoDetect's background subtraction and peak detection (SNIP, Savitzky-Golay,
 * prominence, greedy separation): corrected [n] and up to max_sel selected bins; returns
 * their number */
int or_snip_detect(const double *x, const double *y, int n, int n_iter, double x_bin, int max_sel,
                   double *corrected, int *sel);

#endif
