/*
 * oracle.c -- FP64 CPU restatement of the MIDAS caking hot path (test infrastructure).
 *
 * or_integrate follows, per semantics (3 = IntegratorZarrOMP.c:1709-1778: the IntegrationCore
 * sums, a nonzero sum divided by the bin's whole area):
 *   0: integrate() of packages/midas_integrate/midas_integrate/kernels.py:416-473 with the
 *      CSR of build_csr (kernels.py:242-375) written as the explicit per-record loops of
 *      packages/midas_integrate/tests/test_kernels.py:55-114 (floor: truncated (y,z),
 *      off-detector records skipped; bilinear: np.floor + clamp; gradient: sample point
 *      shifted by -deltaR along the radius, kernels.py:343-353); normaliser = in-bounds
 *      areaWeight sum (kernels.py:306-318).
 *   1: integrate_noMapMask of FF_HEDM/src/IntegratorFitPeaksGPUStream.cu:975-1050
 *      (floor offset (long long)z*NY + y evaluated in float, :915; fp32 gradient shift,
 *      :1007-1018; normaliser = sum of all areaWeight, :1034-1040) with FP64 sums.
 *   2: integration_apply_map of FF_HEDM/src/IntegrationCore.c:14-82 (bilinear at the
 *      record's position, gradient shift in FP64 only when deltaR != 0 and R > 1, base
 *      pixel from floorf() of the float-rounded position, clamps under-then-over;
 *      normaliser = sum of all areaWeight); no floor mode.
 * or_integrate_var follows integrate_with_variance (kernels.py:474-536): coalesced weights
 *   squared against the variance image, over the squared normaliser.
 * or_profile follows profile_1d (kernels.py:567-601) = calculate_1D_profile_kernel and
 * calculate_1D_profile_simple_mean_kernel (IntegratorFitPeaksGPUStream.cu:1162-1334).
 * or_fit is the FP64 twin of the device Levenberg-Marquardt fitter (same window, same
 * initial guess from pf_estimate_initial_params, FF_HEDM/src/PeakFit.c:218-250, same
 * model definitions incl. pf_calculate_model / pf_tch_eta_fwhm, PeakFit.c:17-92).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define AREA_THRESHOLD 1e-9

/* integration_apply_map, FF_HEDM/src/IntegrationCore.c:52-69 */
static double bilinear_ic(const double *img, int ny, int nz, double sy, double sz) {
  int iy = (int)floorf((float)sy), iz = (int)floorf((float)sz);
  double fy = sy - iy, fz = sz - iz;
  if (iy < 0) { iy = 0; fy = 0; }
  if (iy >= ny - 1) { iy = ny - 2; fy = 1; }
  if (iz < 0) { iz = 0; fz = 0; }
  if (iz >= nz - 1) { iz = nz - 2; fz = 1; }
  const double *p = img + (long)iz * ny + iy;
  return p[0] * ((1 - fy) * (1 - fz)) + p[1] * (fy * (1 - fz)) + p[ny] * ((1 - fy) * fz) + p[ny + 1] * (fy * fz);
}

static double bilinear(const double *img, int ny, int nz, double sy, double sz) {
  double fiy = floor(sy), fiz = floor(sz);
  long iy = (long)fiy, iz = (long)fiz;
  double fy = sy - (double)iy, fz = sz - (double)iz;
  int over_y = iy >= ny - 1, under_y = iy < 0, over_z = iz >= nz - 1, under_z = iz < 0;
  if (over_y) { iy = ny - 2; fy = 1.0; }
  if (under_y) { iy = 0; fy = 0.0; }
  if (over_z) { iz = nz - 2; fz = 1.0; }
  if (under_z) { iz = 0; fz = 0.0; }
  const double *p = img + iz * (long)ny + iy;
  return p[0] * (1 - fy) * (1 - fz) + p[1] * fy * (1 - fz) + p[ny] * (1 - fy) * fz + p[ny + 1] * fy * fz;
}

void or_area_in(const or_record *rec, const int32_t *nmap, int64_t n_bins, int ny, int nz, double *area) {
  for (int64_t b = 0; b < n_bins; ++b) {
    double A = 0;
    for (int k = 0; k < nmap[2 * b]; ++k) {
      const or_record *e = rec + nmap[2 * b + 1] + k;
      long ty = (long)(double)e->y, tz = (long)(double)e->z;
      if (ty >= 0 && ty < ny && tz >= 0 && tz < nz) A += e->areaWeight;
    }
    area[b] = A;
  }
}

int or_integrate(const or_record *rec, const int32_t *nmap, int64_t n_bins, int ny, int nz, double bc_y,
                 double bc_z, const double *image, int mode, int sem, int normalize, double *cake, double *area_out) {
  const long npix = (long)ny * nz;
  if ((sem == 2 || sem == 3) && mode == 0) return -3; /* IntegrationCore / OMP: no floor mode */
  for (int64_t b = 0; b < n_bins; ++b) {
    double I = 0.0, A_in = 0.0, A_all = 0.0;
    const int cnt = nmap[2 * b], off = nmap[2 * b + 1];
    if (cnt < 0) return -2;
    for (int k = 0; k < cnt; ++k) {
      const or_record *e = rec + off + k;
      const double y = e->y, z = e->z;
      const long ty = (long)y, tz = (long)z;
      const int inb = ty >= 0 && ty < ny && tz >= 0 && tz < nz;
      A_all += e->areaWeight;
      if (inb) A_in += e->areaWeight;
      if (mode == 0) {
        if (sem == 1) {
          long long zz = (long long)e->z;
          float s = (float)(zz * (long long)ny) + e->y;
          long long o = (long long)s;
          if (o >= 0 && o < npix) I += image[o] * e->frac;
        } else if (inb) {
          I += image[tz * ny + ty] * e->frac;
        }
      } else if (sem == 2 || sem == 3) {
        /* IntegrationCore.c:38-50; IntegratorZarrOMP.c:1722-1745 samples the same way */
        double sy = y, sz = z;
        if (mode == 2 && e->deltaR != 0.0f) {
          double dy = y - bc_y, dz = z - bc_z;
          double R = sqrt(dy * dy + dz * dz);
          if (R > 1.0) {
            sy -= e->deltaR * dy / R;
            sz -= e->deltaR * dz / R;
          }
        }
        I += bilinear_ic(image, ny, nz, sy, sz) * e->frac;
      } else {
        double sy = y, sz = z;
        if (mode == 2) {
          if (sem == 1) {
            float dy = e->y - (float)bc_y, dz = e->z - (float)bc_z;
            float R = sqrtf(dy * dy + dz * dz);
            float ry = e->y, rz = e->z;
            if (R > 1.0f) {
              ry -= e->deltaR * dy / R;
              rz -= e->deltaR * dz / R;
            }
            sy = ry;
            sz = rz;
          } else {
            double dy = y - bc_y, dz = z - bc_z;
            double R = sqrt(dy * dy + dz * dz);
            double sc = R > 1.0 ? (double)e->deltaR / R : 0.0;
            sy = y - sc * dy;
            sz = z - sc * dz;
          }
        }
        I += bilinear(image, ny, nz, sy, sz) * e->frac;
      }
    }
    double out;
    if (sem == 3) {
      /* IntegratorZarrOMP.c:1749-1753: a nonzero sum is divided by the area, whatever it is */
      out = (I != 0.0 && normalize) ? I / A_all : I;
      if (area_out) area_out[b] = A_all;
    } else if (sem == 1 || sem == 2) {
      out = A_all > AREA_THRESHOLD ? (normalize ? I / A_all : I) : 0.0;
      if (area_out) area_out[b] = A_all;
    } else {
      out = normalize ? (A_in > AREA_THRESHOLD ? I / A_in : 0.0) : I;
      if (area_out) area_out[b] = A_in;
    }
    cake[b] = out;
  }
  return 0;
}

/* ------------------------------------------------------------------ variance
 * or_integrate_var: integrate_with_variance (kernels.py:474-536).  The per-(bin, pixel)
 * weights of every record (the terms or_integrate sums) are coalesced per bin, as the
 * CSR's sum_duplicates does (_square_csr, kernels.py:378-400), squared and applied to the
 * variance image; normalised bins divide by the squared normaliser. */
typedef struct { long pix; double w; } or_term;

static int term_cmp(const void *a, const void *b) {
  const long x = ((const or_term *)a)->pix, y = ((const or_term *)b)->pix;
  return (x > y) - (x < y);
}

static int corner_terms(int ny, int nz, long iy, long iz, double fy, double fz, double frac, or_term *t) {
  (void)nz;
  const long o = iz * (long)ny + iy;
  t[0].pix = o;          t[0].w = frac * (1 - fy) * (1 - fz);
  t[1].pix = o + 1;      t[1].w = frac * fy * (1 - fz);
  t[2].pix = o + ny;     t[2].w = frac * (1 - fy) * fz;
  t[3].pix = o + ny + 1; t[3].w = frac * fy * fz;
  return 4;
}

/* the terms one record adds to its bin, per (mode, semantics), as or_integrate samples */
static int record_terms(const or_record *e, int ny, int nz, double bc_y, double bc_z, int mode, int sem,
                        or_term *t) {
  const long npix = (long)ny * nz;
  const double y = e->y, z = e->z;
  if (mode == 0) {
    if (sem == 1) {
      long long zz = (long long)e->z;
      float s = (float)(zz * (long long)ny) + e->y;
      long long o = (long long)s;
      if (o < 0 || o >= npix) return 0;
      t[0].pix = (long)o; t[0].w = e->frac;
      return 1;
    }
    const long ty = (long)y, tz = (long)z;
    if (!(ty >= 0 && ty < ny && tz >= 0 && tz < nz)) return 0;
    t[0].pix = tz * ny + ty; t[0].w = e->frac;
    return 1;
  }
  double sy = y, sz = z;
  if (sem == 2) {
    if (mode == 2 && e->deltaR != 0.0f) {
      double dy = y - bc_y, dz = z - bc_z;
      double R = sqrt(dy * dy + dz * dz);
      if (R > 1.0) { sy -= e->deltaR * dy / R; sz -= e->deltaR * dz / R; }
    }
    int iy = (int)floorf((float)sy), iz = (int)floorf((float)sz);
    double fy = sy - iy, fz = sz - iz;
    if (iy < 0) { iy = 0; fy = 0; }
    if (iy >= ny - 1) { iy = ny - 2; fy = 1; }
    if (iz < 0) { iz = 0; fz = 0; }
    if (iz >= nz - 1) { iz = nz - 2; fz = 1; }
    return corner_terms(ny, nz, iy, iz, fy, fz, e->frac, t);
  }
  if (mode == 2) {
    if (sem == 1) {
      float dy = e->y - (float)bc_y, dz = e->z - (float)bc_z;
      float R = sqrtf(dy * dy + dz * dz);
      float ry = e->y, rz = e->z;
      if (R > 1.0f) { ry -= e->deltaR * dy / R; rz -= e->deltaR * dz / R; }
      sy = ry; sz = rz;
    } else {
      double dy = y - bc_y, dz = z - bc_z;
      double R = sqrt(dy * dy + dz * dz);
      double sc = R > 1.0 ? (double)e->deltaR / R : 0.0;
      sy = y - sc * dy; sz = z - sc * dz;
    }
  }
  long iy = (long)floor(sy), iz = (long)floor(sz);
  double fy = sy - (double)iy, fz = sz - (double)iz;
  const int over_y = iy >= ny - 1, under_y = iy < 0, over_z = iz >= nz - 1, under_z = iz < 0;
  if (over_y) { iy = ny - 2; fy = 1.0; }
  if (under_y) { iy = 0; fy = 0.0; }
  if (over_z) { iz = nz - 2; fz = 1.0; }
  if (under_z) { iz = 0; fz = 0.0; }
  return corner_terms(ny, nz, iy, iz, fy, fz, e->frac, t);
}

int or_integrate_var(const or_record *rec, const int32_t *nmap, int64_t n_bins, int ny, int nz, double bc_y,
                     double bc_z, const double *var_image, int mode, int sem, int normalize, double *var_cake) {
  if (sem == 2 && mode == 0) return -3;
  or_term *buf = NULL;
  long cap = 0;
  for (int64_t b = 0; b < n_bins; ++b) {
    const int cnt = nmap[2 * b], off = nmap[2 * b + 1];
    if (cnt < 0) { free(buf); return -2; }
    if (4L * cnt > cap) {
      cap = 4L * cnt;
      or_term *nb = (or_term *)realloc(buf, (size_t)cap * sizeof(or_term));
      if (!nb) { free(buf); return -1; }
      buf = nb;
    }
    long n = 0;
    double A_in = 0.0, A_all = 0.0;
    for (int k = 0; k < cnt; ++k) {
      const or_record *e = rec + off + k;
      const long ty = (long)(double)e->y, tz = (long)(double)e->z;
      A_all += e->areaWeight;
      if (ty >= 0 && ty < ny && tz >= 0 && tz < nz) A_in += e->areaWeight;
      n += record_terms(e, ny, nz, bc_y, bc_z, mode, sem, buf + n);
    }
    qsort(buf, (size_t)n, sizeof(or_term), term_cmp);
    double V = 0.0;
    for (long i = 0; i < n;) {
      double w = 0.0;
      long j = i;
      for (; j < n && buf[j].pix == buf[i].pix; ++j) w += buf[j].w;
      V += w * w * var_image[buf[i].pix];
      i = j;
    }
    double out;
    if (sem == 1 || sem == 2)
      out = A_all > AREA_THRESHOLD ? (normalize ? V / (A_all * A_all) : V) : 0.0;
    else
      out = normalize ? (A_in > AREA_THRESHOLD ? V / (A_in * A_in) : 0.0) : V;
    var_cake[b] = out;
  }
  free(buf);
  return 0;
}

void or_profile(const double *cake, const double *area_in, int n_r, int n_eta, double *lo_aw, double *lo_sm) {
  for (int r = 0; r < n_r; ++r) {
    double sia = 0, sa = 0, si = 0;
    int n = 0;
    for (int e = 0; e < n_eta; ++e) {
      const long b = (long)r * n_eta + e;
      const double A = area_in[b];
      if (A > AREA_THRESHOLD) {
        sia += cake[b] * A;
        sa += A;
        si += cake[b];
        ++n;
      }
    }
    if (lo_aw) lo_aw[r] = sa > AREA_THRESHOLD ? sia / sa : 0.0;
    if (lo_sm) lo_sm[r] = n > 0 ? si / n : 0.0;
  }
}

/* IntegratorZarrOMP.c:1829-1843: per R row the mean of the nonzero, non-NaN bins, and the
 * area-weighted mean over the valid (in-bounds area > 1e-9), non-NaN bins */
void or_profile_omp(const double *cake, const double *area_in, int n_r, int n_eta, double *lo_aw, double *lo_sm) {
  for (int r = 0; r < n_r; ++r) {
    double sia = 0, sa = 0, si = 0;
    int n = 0;
    for (int e = 0; e < n_eta; ++e) {
      const long b = (long)r * n_eta + e;
      const double I = cake[b], A = area_in[b];
      if (isnan(I)) continue;
      if (A > AREA_THRESHOLD) {
        sia += I * A;
        sa += A;
      }
      if (I != 0.0) {
        si += I;
        ++n;
      }
    }
    if (lo_aw) lo_aw[r] = sa > AREA_THRESHOLD ? sia / sa : 0.0;
    if (lo_sm) lo_sm[r] = n > 0 ? si / n : 0.0;
  }
}

/* ------------------------------------------------------------------ fitter */
#define NP 6

static void tch(double sig, double gam, double *fw, double *eta, double *dfw_ds, double *dfw_dg, double *de_ds,
                double *de_dg) {
  const double ln2x8 = 5.545177444479562;
  const double s = fmax(sig, 1e-12);
  const double fg = sqrt(fmax(ln2x8 * s, 0.0)) / 100.0;
  const double fl = fmax(gam, 1e-6) / 100.0;
  const double dfg_ds = (sig > 1e-12) ? fg / (2.0 * s) : 0.0;
  const double dfl_dg = (gam > 1e-6) ? 0.01 : 0.0;
  const double g2 = fg * fg, g3 = g2 * fg, g4 = g3 * fg, g5 = g4 * fg;
  const double l2 = fl * fl, l3 = l2 * fl, l4 = l3 * fl, l5 = l4 * fl;
  const double P = g5 + 2.69269 * g4 * fl + 2.42843 * g3 * l2 + 4.47163 * g2 * l3 + 0.07842 * fg * l4 + l5;
  double F = pow(fmax(P, 1e-300), 0.2);
  const double dP_dg = 5 * g4 + 4 * 2.69269 * g3 * fl + 3 * 2.42843 * g2 * l2 + 2 * 4.47163 * fg * l3 + 0.07842 * l4;
  const double dP_dl = 2.69269 * g4 + 2 * 2.42843 * g3 * fl + 3 * 4.47163 * g2 * l2 + 4 * 0.07842 * fg * l3 + 5 * l4;
  const double dF_dP = (F > 1e-15) ? 0.2 * F / fmax(P, 1e-300) : 0.0;
  if (F < 1e-15) F = 1e-15;
  const double dF_dg = dF_dP * dP_dg, dF_dl = dF_dP * dP_dl;
  const double r = fl / F;
  double e = 1.36603 * r - 0.47719 * r * r + 0.11116 * r * r * r;
  double de_dr = 1.36603 - 2 * 0.47719 * r + 3 * 0.11116 * r * r;
  if (e < 0 || e > 1) de_dr = 0;
  e = fmin(fmax(e, 0.0), 1.0);
  const double dr_dl = 1.0 / F - fl * dF_dl / (F * F);
  const double dr_dg = -fl * dF_dg / (F * F);
  *fw = F;
  *eta = e;
  *dfw_ds = dF_dg * dfg_ds;
  *dfw_dg = dF_dl * dfl_dg;
  *de_ds = de_dr * dr_dg * dfg_ds;
  *de_dg = de_dr * dr_dl * dfl_dg;
}

static double model(int kind, const double *p, double xl, double xn, double *g) {
  if (kind == 0) {
    const double c = p[0], h = p[1], w = fmax(p[2], 1e-6), et = p[3];
    const double hw = 0.5 * w, u = (xl - c) / hw, u2 = u * u;
    const double L = 1.0 / (1.0 + u2), G = exp(-0.6931471805599453 * u2);
    const double P = et * L + (1.0 - et) * G;
    const double dP_du2 = -et * L * L - (1.0 - et) * 0.6931471805599453 * G;
    g[0] = h * dP_du2 * (-2.0 * u / hw);
    g[1] = P;
    g[2] = h * dP_du2 * (-u2 / hw);
    g[3] = h * (L - G);
    g[4] = 1.0;
    g[5] = xn;
    return p[4] + p[5] * xn + h * P;
  }
  const double A = p[0], c = p[1];
  double F, et, dF_ds, dF_dg, de_ds, de_dg;
  tch(p[2], p[3], &F, &et, &dF_ds, &dF_dg, &de_ds, &de_dg);
  const double sg = F * 0.42466090014400953, Gn = 0.3989422804014327 / sg, hw = 0.5 * F;
  const double dx = xl - c, dx2 = dx * dx;
  const double G = Gn * exp(-0.5 * dx2 / (sg * sg));
  const double den = dx2 + hw * hw;
  const double L = 0.3183098861837907 * hw / den;
  const double P = et * L + (1.0 - et) * G;
  const double dG_dc = G * dx / (sg * sg), dL_dc = L * 2.0 * dx / den;
  const double dG_dsg = G * (-1.0 / sg + dx2 / (sg * sg * sg));
  const double dL_dhw = 0.3183098861837907 * (den - 2.0 * hw * hw) / (den * den);
  const double dP_dF = et * dL_dhw * 0.5 + (1.0 - et) * dG_dsg * 0.42466090014400953;
  const double dP_de = L - G;
  g[0] = P;
  g[1] = A * (et * dL_dc + (1.0 - et) * dG_dc);
  g[2] = A * (dP_dF * dF_ds + dP_de * de_ds);
  g[3] = A * (dP_dF * dF_dg + dP_de * de_dg);
  g[4] = 1.0;
  g[5] = xn;
  return p[4] + p[5] * xn + A * P;
}

static int chol_solve(double A[NP][NP], const double *b, double *x) {
  double L[NP][NP], y[NP];
  memset(L, 0, sizeof(L));
  for (int i = 0; i < NP; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = A[i][j];
      for (int k = 0; k < j; ++k) s -= L[i][k] * L[j][k];
      if (i == j) {
        if (!(s > 0.0)) return 0;
        L[i][i] = sqrt(s);
      } else {
        L[i][j] = s / L[j][j];
      }
    }
  for (int i = 0; i < NP; ++i) {
    double s = b[i];
    for (int k = 0; k < i; ++k) s -= L[i][k] * y[k];
    y[i] = s / L[i][i];
  }
  for (int i = NP - 1; i >= 0; --i) {
    double s = y[i];
    for (int k = i + 1; k < NP; ++k) s -= L[k][i] * x[k];
    x[i] = s / L[i][i];
  }
  return 1;
}

static void clamp_params(int kind, double *p, double half_span, double x_bin) {
  if (kind == 0) {
    p[0] = fmin(fmax(p[0], -half_span), half_span);
    p[1] = fmax(p[1], 0.0);
    p[2] = fmin(fmax(p[2], 0.05 * x_bin), 4.0 * half_span);
    p[3] = fmin(fmax(p[3], 0.0), 1.0);
  } else {
    p[0] = fmax(p[0], 0.0);
    p[1] = fmin(fmax(p[1], -half_span), half_span);
    p[2] = fmax(p[2], 1e-6);
    p[3] = fmax(p[3], 0.01);
  }
}

static void eval(int kind, const double *p, const double *x, const double *y, int s0, int n, double xref, double xlo,
                 double xr, double JtJ[NP][NP], double *Jtr, double *chi2) {
  double jj[NP][NP], jr[NP], c2 = 0;
  memset(jj, 0, sizeof(jj));
  memset(jr, 0, sizeof(jr));
  for (int i = 0; i < n; ++i) {
    const double xi = x[s0 + i];
    double g[NP];
    const double m = model(kind, p, xi - xref, 2.0 * (xi - xlo) / xr - 1.0, g);
    const double r = y[s0 + i] - m;
    for (int u = 0; u < NP; ++u) {
      for (int v = 0; v <= u; ++v) jj[u][v] += g[u] * g[v];
      jr[u] += g[u] * r;
    }
    c2 += r * r;
  }
  if (JtJ)
    for (int u = 0; u < NP; ++u)
      for (int v = 0; v <= u; ++v) JtJ[u][v] = JtJ[v][u] = jj[u][v];
  if (Jtr)
    for (int u = 0; u < NP; ++u) Jtr[u] = jr[u];
  *chi2 = c2;
}

int or_fit(const double *x, const double *y, int n_x, double loc, int half, int kind, int max_iter, double x_bin,
           double px, double lsd, double *out) {
  memset(out, 0, 11 * sizeof(double));
  int best = -1;
  double bd = 1e300;
  for (int i = 0; i < n_x; ++i) {
    const double d = fabs(x[i] - loc);
    if (d < bd) { bd = d; best = i; }
  }
  if (best < 0 || !(bd < 2.0 * x_bin)) return -1;
  const int s0 = best - half < 0 ? 0 : best - half;
  const int s1 = best + half > n_x - 1 ? n_x - 1 : best + half;
  const int n = s1 - s0 + 1;
  if (n < NP + 1) return -2;
  const double xref = x[best], xlo = x[s0], xhi = x[s1];
  const double xr = fmax(xhi - xlo, 1e-12);
  const double half_span = fmax(xhi - xref, xref - xlo);
  int bgw = n / 4 < 5 ? n / 4 : 5;
  if (bgw < 1) bgw = 1;
  double bgs = 0;
  for (int i = 0; i < bgw; ++i) bgs += y[s0 + i] + y[s1 - i];
  const double bg = bgs / (2.0 * bgw);
  double amp = y[best] - bg;
  if (amp <= 0) amp = y[best];
  const double hm = bg + 0.5 * amp;
  int li = best - s0, ri = best - s0;
  while (li > 0 && y[s0 + li] > hm) --li;
  while (ri < n - 1 && y[s0 + ri] > hm) ++ri;
  double fwb = (double)(ri - li);
  if (!(fwb > 1.0)) fwb = 2.0;
  const double fwx = fwb * x_bin;
  double p[NP];
  if (kind == 0) {
    p[0] = 0; p[1] = amp; p[2] = fwx; p[3] = 0.5; p[4] = bg; p[5] = 0;
  } else {
    const double fg0 = 0.5 * fwx;
    double sg = (fg0 * 100.0) * (fg0 * 100.0) / 5.545177444479562;
    if (sg < 1e-6) sg = 1.0;
    double gm = fwx * 0.5 * 100.0;
    if (gm < 0.01) gm = 1.0;
    double ar = amp * fwx * 1.5;
    if (ar <= 0) ar = 1.0;
    p[0] = ar; p[1] = 0; p[2] = sg; p[3] = gm; p[4] = bg; p[5] = 0;
  }
  clamp_params(kind, p, half_span, x_bin);
  double JtJ[NP][NP], Jtr[NP], chi2;
  eval(kind, p, x, y, s0, n, xref, xlo, xr, JtJ, Jtr, &chi2);
  double lam = 1e-3;
  int it = 0, stall = 0;
  for (; it < max_iter; ++it) {
    double A[NP][NP], d[NP], pn[NP];
    for (int u = 0; u < NP; ++u)
      for (int v = 0; v < NP; ++v) A[u][v] = JtJ[u][v] + (u == v ? lam * fmax(JtJ[u][u], 1e-30) : 0.0);
    int ok = chol_solve(A, Jtr, d);
    for (int u = 0; u < NP; ++u) pn[u] = ok ? p[u] + d[u] : p[u];
    clamp_params(kind, pn, half_span, x_bin);
    double c2n;
    eval(kind, pn, x, y, s0, n, xref, xlo, xr, NULL, NULL, &c2n);
    if (ok && c2n <= chi2) {
      double rel = 0;
      for (int u = 0; u < NP; ++u) rel = fmax(rel, fabs(pn[u] - p[u]) / fmax(fabs(p[u]), 1e-3));
      const double dec = chi2 - c2n;
      memcpy(p, pn, sizeof(p));
      eval(kind, p, x, y, s0, n, xref, xlo, xr, JtJ, Jtr, &chi2);
      lam = fmax(lam * 0.1, 1e-12);
      if (rel < 1e-10 || dec <= 1e-14 * chi2) {
        if (++stall >= 2) { ++it; break; }
      } else {
        stall = 0;
      }
    } else {
      lam *= 10.0;
      if (lam > 1e12) { ++it; break; }
    }
  }
  double area, center, sig = 0, gam = 0, fw, et, height;
  if (kind == 0) {
    center = xref + p[0];
    height = p[1];
    fw = p[2];
    et = p[3];
    area = height * fw * (et * 1.5707963267948966 + (1.0 - et) * 1.0644670194312262);
  } else {
    double t0, t1, t2, t3;
    tch(p[2], p[3], &fw, &et, &t0, &t1, &t2, &t3);
    area = p[0];
    center = xref + p[1];
    sig = p[2];
    gam = p[3];
    const double sgm = fw * 0.42466090014400953;
    height = area * (et * (2.0 / (3.141592653589793 * fw)) + (1.0 - et) * 0.3989422804014327 / sgm);
  }
  out[0] = area;
  out[1] = center;
  out[2] = sig;
  out[3] = gam;
  out[4] = fw;
  out[5] = et;
  out[6] = chi2 / fmax((double)(n - NP), 1.0);
  out[7] = height;
  out[8] = p[4];
  out[9] = p[5];
  out[10] = (px > 0 && lsd > 0) ? atan(center * px / lsd) * 57.29577951308232 : 0.0;
  return it;
}

/* ------------------------------------------------------------------ peak detection
 * or_snip_detect restates fitPeaksAutoDetect's detection (FF_HEDM/src/PeakFit.c:549-755):
 * SNIP background on the log-log-sqrt transformed profile (Morhac's LLS clipping with
 * windows n_iter .. 1), the background-subtracted profile clipped at 0 (corrected), a
 * 7-point quadratic Savitzky-Golay smoothing, its negative second difference, candidates
 * at its positive local maxima where the corrected profile is positive, prominence over
 * +-min_sep bins, greedy selection by prominence (ties: lower bin) at least min_sep bins
 * apart, up to max_sel, returned in bin order.  Returns the number selected. */
int or_snip_detect(const double *x, const double *y, int n, int n_iter, double x_bin, int max_sel, double *corrected,
                   int *sel) {
  double *v = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  double *t = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) v[i] = log(log(sqrt(fmax(y[i], 0.0) + 1.0) + 1.0) + 1.0);
  for (int p = n_iter; p >= 1; --p) {
    memcpy(t, v, sizeof(double) * n);
    for (int i = p; i < n - p; ++i) {
      const double avg = (t[i - p] + t[i + p]) / 2.0;
      if (v[i] > avg) v[i] = avg;
    }
  }
  for (int i = 0; i < n; ++i) {
    double bg = 0.0;
    if (n_iter > 0) {
      const double w = exp(exp(v[i]) - 1.0) - 1.0;
      bg = fmax(w * w - 1.0, 0.0);
    }
    corrected[i] = fmax(y[i] - bg, 0.0);
  }
  int ns = 0;
  if (n >= 10 && max_sel > 0) {
    static const double c7[7] = {-2, 3, 6, 7, 6, 3, -2};
    for (int i = 0; i < n; ++i) {
      if (i < 3 || i >= n - 3) t[i] = corrected[i];
      else {
        double s = 0;
        for (int j = 0; j < 7; ++j) s += c7[j] * corrected[i - 3 + j];
        t[i] = s / 21.0;
      }
    }
    for (int i = 0; i < n; ++i) v[i] = (i >= 1 && i < n - 1) ? -(t[i + 1] - 2.0 * t[i] + t[i - 1]) : 0.0;
    const double bw = n > 1 ? fabs(x[1] - x[0]) : 1.0;
    const int msep = (int)fmax(3.0, x_bin * 3.0 / bw);
    int *cb = (int *)malloc(sizeof(int) * (n / 2 + 1));
    double *cp = (double *)malloc(sizeof(double) * (n / 2 + 1));
    int nc = 0;
    for (int i = 2; i < n - 2 && nc < n / 2; ++i)
      if (v[i] > 0 && v[i] >= v[i - 1] && v[i] >= v[i + 1] && corrected[i] > 0) {
        double lm = v[i], rm = v[i];
        for (int j = i - 1; j >= 0 && j >= i - msep; --j) lm = fmin(lm, v[j]);
        for (int j = i + 1; j < n && j <= i + msep; ++j) rm = fmin(rm, v[j]);
        double pr = v[i] - fmax(lm, rm);
        if (pr < 0) pr = v[i];
        cb[nc] = i;
        cp[nc] = pr;
        ++nc;
      }
    while (ns < max_sel) {
      int bi = -1;
      for (int c = 0; c < nc; ++c)
        if (cb[c] >= 0 && (bi < 0 || cp[c] > cp[bi] || (cp[c] == cp[bi] && cb[c] < cb[bi]))) bi = c;
      if (bi < 0) break;
      int close = 0;
      for (int k = 0; k < ns; ++k) close |= abs(cb[bi] - sel[k]) < msep;
      if (!close) sel[ns++] = cb[bi];
      cb[bi] = -1;
    }
    for (int i = 1; i < ns; ++i)
      for (int j = i; j > 0 && sel[j] < sel[j - 1]; --j) { const int q = sel[j]; sel[j] = sel[j - 1]; sel[j - 1] = q; }
    free(cb);
    free(cp);
  }
  free(v);
  free(t);
  return ns;
}
