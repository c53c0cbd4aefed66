// mi_fitjob.cu -- kernel (d'), fit plans: batched multi-peak fit jobs.
//
// A fit plan fixes, once per (x axis, peak list, options), the fit jobs the reference would
// form, and then fits every job of every series (a lineout, or one eta column of a cake)
// of a batch in one launch, one warp per series.
//
// Job construction follows the reference exactly:
//   MI_FIT_KIND_PEAKS  fitPeaks (FF_HEDM/src/PeakFit.c:275-470; fit_peaks,
//                      packages/midas_integrate/midas_integrate/peakfit.py:334): each peak's
//                      nearest bin (kept when closer than 2 bins), peaks sorted by bin, ROI
//                      = bin +- half_window clamped to the axis, a peak whose ROI starts at
//                      or before the current job's end joins that job.  Model: area-
//                      normalised TCH pseudo-Voigt per peak + bg0 + bg1 * xn over the job's
//                      x range (pf_calculate_model, PeakFit.c:50-92), 4 parameters per peak
//                      + 2; initial values and box bounds of fitPeaks (PeakFit.c:363-440).
//   MI_FIT_KIND_ETA    the per-eta fits of IntegratorZarrOMP.c:1902-2030: for every eta
//                      column with at least 5 nonzero samples, each peak (or each doublet of
//                      adjacent peaks closer than doublet_sep, in the given order) is fit on
//                      the bins whose centre lies within +- half_window bins of the peak(s),
//                      skipped when that range has fewer than 6 bins.  Model: height-
//                      normalised pseudo-Voigt with one mixing and one flat background
//                      (pf_pv_singlet_obj / pf_pv_doublet_obj, PeakFit.c:882-1040): per peak
//                      centre, FWHM, height; initial values and bounds of pf_fit_singlet_pv /
//                      pf_fit_doublet_pv (PeakFit.c:922-1110).  Output: the centre and
//                      SNR = height / rms residual when SNR > 1, as the reference writes.
//
// The reference minimises with NLopt L-BFGS (Nelder-Mead fallback); here the same least-
// squares objective is minimised by Levenberg-Marquardt with the step projected onto the
// box bounds: model and Jacobian rows in FP32 (x carried relative to the window centre),
// J^T J, J^T r and chi^2 reduced in FP64, the damped normal equations solved by an FP64
// Cholesky factorisation.  Per warp the window's samples, the Jacobian rows and the normal
// matrix live in shared memory.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "mi_fitcore.cuh"
#include "mi_internal.h"

namespace mi {

struct FitJobDev {
  int32_t s0, s1;     // sample range [s0, s1] of the ROI
  int32_t n_p, p0;    // peaks of the job: entries [p0, p0 + n_p) of the plan's peak table
};

struct FitPlanArgs {
  const FitJobDev *jobs;
  const double *pk_x;     // per job peak: the bin position used as initial centre
  const int32_t *pk_bin;  // its bin (KIND_PEAKS: nearest bin)
  const int32_t *pk_id;   // its index in the caller's peak list
  const double *x;        // axis [n_x]
  const void *src;
  int src_f64;
  int64_t ld_series, ld_sub, ld_x;
  int n_series, n_sub, n_x, n_jobs, n_peaks, kind, max_iter, np_max, n_max;
  double x_bin, px, lsd;
  double *out;
  int32_t *iters;
  uint32_t warp_bytes;
};

constexpr int kJobWarps = 4;

// shared-memory carve-up of one warp
struct JobSmem {
  double *y, *r, *jtj, *am, *jtr, *d;
  float *xl, *xn, *J, *p, *pn, *lb, *ub, *pk;
};

__host__ __device__ inline uint32_t job_warp_bytes(int n_max, int np, JobSmem *S, uint8_t *base) {
  auto a16 = [](uint32_t x) { return (x + 15u) & ~15u; };
  uint32_t o = 0;
  const uint32_t oy = o;   o = a16(o + 8u * n_max);
  const uint32_t orr = o;  o = a16(o + 8u * n_max);
  const uint32_t ojj = o;  o = a16(o + 8u * np * np);
  const uint32_t oam = o;  o = a16(o + 8u * np * np);
  const uint32_t ojr = o;  o = a16(o + 8u * np);
  const uint32_t od = o;   o = a16(o + 8u * np);
  const uint32_t oxl = o;  o = a16(o + 4u * n_max);
  const uint32_t oxn = o;  o = a16(o + 4u * n_max);
  const uint32_t oJ = o;   o = a16(o + 4u * n_max * np);
  const uint32_t op = o;   o = a16(o + 4u * np);
  const uint32_t opn = o;  o = a16(o + 4u * np);
  const uint32_t olb = o;  o = a16(o + 4u * np);
  const uint32_t oub = o;  o = a16(o + 4u * np);
  const uint32_t opk = o;  o = a16(o + 4u * 8u * MI_FIT_JOB_MAX_PEAKS);
  if (S && base) {
    S->y = (double *)(base + oy);
    S->r = (double *)(base + orr);
    S->jtj = (double *)(base + ojj);
    S->am = (double *)(base + oam);
    S->jtr = (double *)(base + ojr);
    S->d = (double *)(base + od);
    S->xl = (float *)(base + oxl);
    S->xn = (float *)(base + oxn);
    S->J = (float *)(base + oJ);
    S->p = (float *)(base + op);
    S->pn = (float *)(base + opn);
    S->lb = (float *)(base + olb);
    S->ub = (float *)(base + oub);
    S->pk = (float *)(base + opk);
  }
  return o;
}

// Model of a job at sample i (x relative to the window centre xl, normalised xn), gradient
// into g (stride 1).  TCH: per peak (A, c, sig, gam) then (bg0, bg1); the per-peak FWHM and
// mixing (and their derivatives) are precomputed in pk[8 k ..].  PVH: per peak (c, G, I)
// then (mu, bg).
__device__ inline float job_model(int kind, int n_p, const float *p, const float *pk, float xl, float xn, float *g) {
  if (kind == MI_FIT_KIND_PEAKS) {
    float m = p[4 * n_p] + p[4 * n_p + 1] * xn;
    for (int k = 0; k < n_p; ++k) {
      const float A = p[4 * k], c = p[4 * k + 1];
      const float F = pk[8 * k], et = pk[8 * k + 1], dF_ds = pk[8 * k + 2], dF_dg = pk[8 * k + 3],
                  de_ds = pk[8 * k + 4], de_dg = pk[8 * k + 5];
      const float sg = F * 0.42466090014400953f;
      const float Gn = 0.3989422804014327f / sg;
      const float hw = 0.5f * F;
      const float dx = xl - c, dx2 = dx * dx;
      const float G = Gn * expf(-0.5f * dx2 / (sg * sg));
      const float den = dx2 + hw * hw;
      const float L = 0.3183098861837907f * hw / den;
      const float P = et * L + (1.0f - et) * G;
      const float dG_dc = G * dx / (sg * sg);
      const float dL_dc = L * 2.0f * dx / den;
      const float dG_dsg = G * (-1.0f / sg + dx2 / (sg * sg * sg));
      const float dL_dhw = 0.3183098861837907f * (den - 2.0f * hw * hw) / (den * den);
      const float dP_dF = et * dL_dhw * 0.5f + (1.0f - et) * dG_dsg * 0.42466090014400953f;
      const float dP_de = L - G;
      g[4 * k] = P;
      g[4 * k + 1] = A * (et * dL_dc + (1.0f - et) * dG_dc);
      g[4 * k + 2] = A * (dP_dF * dF_ds + dP_de * de_ds);
      g[4 * k + 3] = A * (dP_dF * dF_dg + dP_de * de_dg);
      m += A * P;
    }
    g[4 * n_p] = 1.0f;
    g[4 * n_p + 1] = xn;
    return m;
  }
  const float mu = p[3 * n_p], C0 = 2.772588722239781f;   // 4 ln 2
  float m = p[3 * n_p + 1], dmu = 0.0f;
  for (int k = 0; k < n_p; ++k) {
    const float c = p[3 * k], Gm = p[3 * k + 1], I = p[3 * k + 2];
    const float dr = xl - c, dr2 = dr * dr;
    const float iG2 = 1.0f / (Gm * Gm);
    const float den = 1.0f + 4.0f * dr2 * iG2;
    const float L = 1.0f / den;
    const float Gs = expf(-C0 * dr2 * iG2);
    const float P = mu * L + (1.0f - mu) * Gs;
    const float dLdc = 8.0f * dr * iG2 / (den * den);
    const float dGdc = Gs * 2.0f * C0 * dr * iG2;
    const float dLdG = 8.0f * dr2 * iG2 / (Gm * den * den);
    const float dGdG = Gs * 2.0f * C0 * dr2 * iG2 / Gm;
    g[3 * k] = I * (mu * dLdc + (1.0f - mu) * dGdc);
    g[3 * k + 1] = I * (mu * dLdG + (1.0f - mu) * dGdG);
    g[3 * k + 2] = P;
    dmu += I * (L - Gs);
    m += I * P;
  }
  g[3 * n_p] = dmu;
  g[3 * n_p + 1] = 1.0f;
  return m;
}

// every lane: evaluate the job at parameters q over the window; chi^2 (all lanes) and,
// with jac, J rows, residuals, J^T r and the lower triangle of J^T J in shared memory
__device__ double job_eval(int kind, const JobSmem &S, int n, int np, int n_p, const float *q, bool jac, int lane) {
  if (kind == MI_FIT_KIND_PEAKS) {
    if (lane < n_p) {
      float F, et, t0, t1, t2, t3;
      tch(q[4 * lane + 2], q[4 * lane + 3], &F, &et, &t0, &t1, &t2, &t3);
      float *pk = S.pk + 8 * lane;
      pk[0] = F; pk[1] = et; pk[2] = t0; pk[3] = t1; pk[4] = t2; pk[5] = t3;
    }
    __syncwarp();
  }
  double c2 = 0.0;
  float g[4 * MI_FIT_JOB_MAX_PEAKS + 2];
  for (int i = lane; i < n; i += 32) {
    const float m = job_model(kind, n_p, q, S.pk, S.xl[i], S.xn[i], g);
    const double r = S.y[i] - (double)m;
    c2 += r * r;
    if (jac) {
      S.r[i] = r;
      for (int u = 0; u < np; ++u) S.J[i * np + u] = g[u];
    }
  }
  c2 = warp_sum(c2);
  if (jac) {
    __syncwarp();
    const int npair = np * (np + 1) / 2;
    for (int t = lane; t < npair + np; t += 32) {
      double s = 0.0;
      if (t < npair) {
        // pair t -> (u, v), v <= u
        int u = (int)((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
        while ((u + 1) * (u + 2) / 2 <= t) ++u;
        while (u * (u + 1) / 2 > t) --u;
        const int v = t - u * (u + 1) / 2;
        for (int i = 0; i < n; ++i) s += (double)S.J[i * np + u] * (double)S.J[i * np + v];
        S.jtj[u * np + v] = s;
        S.jtj[v * np + u] = s;
      } else {
        const int u = t - npair;
        for (int i = 0; i < n; ++i) s += (double)S.J[i * np + u] * S.r[i];
        S.jtr[u] = s;
      }
    }
    __syncwarp();
  }
  return c2;
}

// lane 0: solve (J^T J + lam diag) d = J^T r by Cholesky in FP64; false if not positive
__device__ bool job_solve(const JobSmem &S, int np, double lam) {
  double *A = S.am;
  for (int u = 0; u < np; ++u)
    for (int v = 0; v <= u; ++v) A[u * np + v] = S.jtj[u * np + v] + (u == v ? lam * fmax(S.jtj[u * np + u], 1e-30) : 0.0);
  for (int i = 0; i < np; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = A[i * np + j];
      for (int k = 0; k < j; ++k) s -= A[i * np + k] * A[j * np + k];
      if (i == j) {
        if (!(s > 0.0)) return false;
        A[i * np + i] = sqrt(s);
      } else {
        A[i * np + j] = s / A[j * np + j];
      }
    }
  for (int i = 0; i < np; ++i) {
    double s = S.jtr[i];
    for (int k = 0; k < i; ++k) s -= A[i * np + k] * S.d[k];
    S.d[i] = s / A[i * np + i];
  }
  for (int i = np - 1; i >= 0; --i) {
    double s = S.d[i];
    for (int k = i + 1; k < np; ++k) s -= A[k * np + i] * S.d[k];
    S.d[i] = s / A[i * np + i];
  }
  return true;
}

// fitting parameters shared by every job of a launch
struct JobParams {
  int kind, max_iter;
  double x_bin, px, lsd;
  const double *x;   // the axis [n_x]
};

// One job of one series, by one warp: window, initial values and bounds, projected LM,
// outputs.  sample(i) is sample i of the series; rows go to out + id * MI_FIT_NOUT and
// iteration counts to its[id], id = pk_id[entry] (or the entry itself when pk_id is null).
template <typename Sample>
__device__ void fit_one_job(const JobParams &c, const JobSmem &S, const FitJobDev jd, const double *pk_x,
                            const int32_t *pk_bin, const int32_t *pk_id, Sample sample, double *out, int32_t *its,
                            int lane) {
  const int n = jd.s1 - jd.s0 + 1, n_p = jd.n_p;
  const int np = c.kind == MI_FIT_KIND_PEAKS ? 4 * n_p + 2 : 3 * n_p + 2;
  if (n <= np) {
    // fewer samples than parameters: the job's peaks are not fit
    for (int k = lane; k < n_p; k += 32) its[pk_id ? pk_id[jd.p0 + k] : jd.p0 + k] = -2;
    __syncwarp();
    return;
  }
  // window samples: x relative to the window's centre bin, normalised x, values
  const int cb = (jd.s0 + jd.s1) / 2;
  const double xref = c.x[cb], xlo = c.x[jd.s0], xhi = c.x[jd.s1];
  const double xr = fmax(xhi - xlo, 1e-12);
  for (int i = lane; i < n; i += 32) {
    const double xi = c.x[jd.s0 + i];
    S.xl[i] = (float)(xi - xref);
    S.xn[i] = (float)(2.0 * (xi - xlo) / xr - 1.0);
    S.y[i] = sample(jd.s0 + i);
  }
  __syncwarp();
  // initial values and bounds (lane 0)
  if (lane == 0) {
    if (c.kind == MI_FIT_KIND_PEAKS) {
      double rmax = -1e30, rmin = 1e30;
      for (int i = 0; i < n; ++i) { rmax = fmax(rmax, S.y[i]); rmin = fmin(rmin, S.y[i]); }
      const double range = fmax(rmax - rmin, 1.0);
      const int bgw = max(1, min(5, n / 4));
      double bgs = 0.0;
      for (int i = 0; i < bgw; ++i) bgs += S.y[i] + S.y[n - 1 - i];
      const double bg = bgs / (2.0 * bgw);   // pf_estimate_initial_params: same for every peak
      for (int k = 0; k < n_p; ++k) {
        const int loc = pk_bin[jd.p0 + k] - jd.s0;
        double amp = S.y[loc] - bg;
        if (amp <= 0) amp = S.y[loc];
        const double hm = bg + 0.5 * amp;
        int li = loc, ri = loc;
        while (li > 0 && S.y[li] > hm) --li;
        while (ri < n - 1 && S.y[ri] > hm) ++ri;
        double fwb = (double)(ri - li);
        if (!(fwb > 1.0)) fwb = 2.0;
        const double fwx = fwb * c.x_bin;
        const double fg0 = 0.5 * fwx;
        double sg = (fg0 * 100.0) * (fg0 * 100.0) / 5.545177444479562;
        if (sg < 1e-6) sg = 1.0;
        double gm = fwx * 0.5 * 100.0;
        if (gm < 0.01) gm = 1.0;
        double ar = amp * fwx * 1.5;
        if (ar <= 0) ar = range * c.x_bin;
        const double c0 = pk_x[jd.p0 + k] - xref;
        const double crange = fmax(fwx, (double)n * c.x_bin * 0.5);
        double ahi = range * (double)n * c.x_bin * 2.0;
        if (ahi < 1.0) ahi = 1.0;
        const double shi = (c.x_bin * 2e4) * (c.x_bin * 2e4) / 5.545177444479562;
        const double ghi = c.x_bin * 2e4;
        const double lo4[4] = {0.0, c0 - crange, 1e-6, 0.01}, hi4[4] = {ahi, c0 + crange, shi, ghi};
        double v4[4] = {fmax(fmin(ar, ahi * 0.9), 0.01), c0, fmax(fmin(sg, shi * 0.5), 2e-6),
                        fmax(fmin(gm, ghi * 0.5), 0.02)};
        for (int u = 0; u < 4; ++u) {
          if (v4[u] <= lo4[u]) v4[u] = lo4[u] + (hi4[u] - lo4[u]) * 0.01;
          if (v4[u] >= hi4[u]) v4[u] = hi4[u] - (hi4[u] - lo4[u]) * 0.01;
          S.p[4 * k + u] = (float)v4[u];
          S.lb[4 * k + u] = (float)lo4[u];
          S.ub[4 * k + u] = (float)hi4[u];
        }
      }
      double b0 = bg, b0lo = fmin(rmin - range * 0.5, -1.0), b0hi = rmax + range;
      if (b0 <= b0lo) b0 = b0lo + 0.01;
      if (b0 >= b0hi) b0 = b0hi - 0.01;
      S.p[4 * n_p] = (float)b0;
      S.lb[4 * n_p] = (float)b0lo;
      S.ub[4 * n_p] = (float)b0hi;
      S.p[4 * n_p + 1] = 0.0f;
      S.lb[4 * n_p + 1] = (float)-range;
      S.ub[4 * n_p + 1] = (float)range;
    } else {
      double bg0 = 0.5 * (S.y[0] + S.y[n - 1]);
      if (bg0 < 0) bg0 = 0;
      double mx = -1e20;
      for (int i = 0; i < n; ++i) mx = fmax(mx, S.y[i]);
      const double step = c.x_bin, gam0 = 3.0 * step;
      const double xfirst = xlo - xref, xlast = xhi - xref;
      if (n_p == 1) {
        const double c0 = pk_x[jd.p0] - xref;
        S.p[0] = (float)c0;  S.lb[0] = (float)xfirst;  S.ub[0] = (float)xlast;
        S.p[1] = (float)gam0;  S.lb[1] = (float)(step / 2);  S.ub[1] = (float)(step * n / 2);
        S.p[2] = (float)(mx - bg0);  S.lb[2] = (float)((mx - bg0) / 100);  S.ub[2] = (float)(mx * 1.5);
      } else {
        double ig = mx - bg0;
        if (ig < 1e-6) ig = 1e-6;
        const double c1 = pk_x[jd.p0] - xref, c2 = pk_x[jd.p0 + 1] - xref, cm = 0.5 * (c1 + c2);
        S.p[0] = (float)c1;  S.lb[0] = (float)xfirst;  S.ub[0] = (float)cm;
        S.p[3] = (float)c2;  S.lb[3] = (float)cm;  S.ub[3] = (float)xlast;
        for (int k = 0; k < 2; ++k) {
          S.p[3 * k + 1] = (float)gam0;  S.lb[3 * k + 1] = (float)(step / 2);  S.ub[3 * k + 1] = (float)(step * n / 2);
          S.p[3 * k + 2] = (float)(ig / 2);  S.lb[3 * k + 2] = (float)(ig / 100);  S.ub[3 * k + 2] = (float)(mx * 1.5);
        }
      }
      S.p[3 * n_p] = 0.5f;  S.lb[3 * n_p] = 0.0f;  S.ub[3 * n_p] = 1.0f;
      S.p[3 * n_p + 1] = (float)bg0;  S.lb[3 * n_p + 1] = 0.0f;
      S.ub[3 * n_p + 1] = (float)(bg0 > 0 ? bg0 * 1.5 : mx * 0.5);
    }
  }
  __syncwarp();
  // ---- LM with the step projected onto the bounds
  double chi2 = job_eval(c.kind, S, n, np, n_p, S.p, true, lane);
  double lam = 1e-3;
  int it = 0, stall = 0;
  for (; it < c.max_iter; ++it) {
    int ok = 0;
    if (lane == 0) {
      ok = job_solve(S, np, lam) ? 1 : 0;
      for (int u = 0; u < np; ++u) {
        float v = ok ? (float)((double)S.p[u] + S.d[u]) : S.p[u];
        S.pn[u] = fminf(fmaxf(v, S.lb[u]), S.ub[u]);
      }
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    __syncwarp();
    const double c2n = job_eval(c.kind, S, n, np, n_p, S.pn, false, lane);
    if (ok && c2n <= chi2) {
      double rel = 0.0;
      for (int u = 0; u < np; ++u)
        rel = fmax(rel, fabs((double)S.pn[u] - (double)S.p[u]) / fmax(fabs((double)S.p[u]), 1e-3));
      const double dec = chi2 - c2n;
      __syncwarp();
      for (int u = lane; u < np; u += 32) S.p[u] = S.pn[u];
      __syncwarp();
      chi2 = job_eval(c.kind, S, n, np, n_p, S.p, true, lane);
      lam = fmax(lam * 0.1, 1e-12);
      if (rel < 1e-6 || dec <= 1e-9 * chi2) {
        if (++stall >= 2) { ++it; break; }
      } else {
        stall = 0;
      }
    } else {
      lam *= 10.0;
      if (lam > 1e12) { ++it; break; }
    }
  }
  // ---- outputs, FP64 (centres back to absolute x)
  if (lane < n_p) {
    const int k = lane, id = pk_id ? pk_id[jd.p0 + k] : jd.p0 + k;
    double *o = out + (int64_t)id * MI_FIT_NOUT;
    double center;
    if (c.kind == MI_FIT_KIND_PEAKS) {
      float F, et, t0, t1, t2, t3;
      tch(S.p[4 * k + 2], S.p[4 * k + 3], &F, &et, &t0, &t1, &t2, &t3);
      const double area = S.p[4 * k];
      center = xref + (double)S.p[4 * k + 1];
      const double sgm = (double)F * 0.42466090014400953;
      o[0] = area;
      o[1] = center;
      o[2] = S.p[4 * k + 2];
      o[3] = S.p[4 * k + 3];
      o[4] = F;
      o[5] = et;
      o[6] = chi2 / fmax((double)(n - np), 1.0);
      o[7] = area * (et * (2.0 / (3.141592653589793 * (double)F)) + (1.0 - et) * 0.3989422804014327 / sgm);
      o[8] = S.p[4 * n_p];
      o[9] = S.p[4 * n_p + 1];
    } else {
      center = xref + (double)S.p[3 * k];
      const double rms = sqrt(chi2 / (double)n);
      const double snr = rms > 0 ? (double)S.p[3 * k + 2] / rms : 1.0;
      // the reference keeps a fit only when SNR > 1; area, sig, gam, FWHM, eta stay 0
      if (snr > 1.0) {
        o[1] = center;
        o[6] = snr;
        o[7] = S.p[3 * k + 2];
        o[8] = S.p[3 * n_p + 1];
        o[9] = 0.0;
      } else {
        center = 0.0;
      }
    }
    o[10] = (center != 0.0 && c.px > 0 && c.lsd > 0) ? atan(center * c.px / c.lsd) * 57.29577951308232 : 0.0;
    its[id] = it;
  }
  __syncwarp();
}

__global__ void __launch_bounds__(32 * kJobWarps) k_fit_job(const FitPlanArgs a) {
  extern __shared__ __align__(16) uint8_t fsm[];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int64_t series = (int64_t)blockIdx.x * kJobWarps + wl;
  if (series >= (int64_t)a.n_series * a.n_sub) return;
  JobSmem S;
  job_warp_bytes(a.n_max, a.np_max, &S, fsm + (size_t)wl * a.warp_bytes);
  const int64_t f = series / a.n_sub, e = series % a.n_sub;
  const int64_t base = f * a.ld_series + e * a.ld_sub;
  auto sample = [&](int i) -> double {
    const int64_t o = base + (int64_t)i * a.ld_x;
    return a.src_f64 ? ((const double *)a.src)[o] : (double)((const float *)a.src)[o];
  };
  double *out = a.out + series * (int64_t)a.n_peaks * MI_FIT_NOUT;
  int32_t *its = a.iters + series * (int64_t)a.n_peaks;
  // rejected peaks stay zero rows with iteration count -1
  for (int t = lane; t < a.n_peaks * MI_FIT_NOUT; t += 32) out[t] = 0.0;
  for (int t = lane; t < a.n_peaks; t += 32) its[t] = -1;
  __syncwarp();
  if (a.kind == MI_FIT_KIND_ETA) {
    // eta columns with fewer than 5 nonzero samples are skipped (IntegratorZarrOMP.c:1941-1948)
    int nz = 0;
    for (int i = lane; i < a.n_x; i += 32) nz += sample(i) != 0.0;
    for (int o = 16; o > 0; o >>= 1) nz += __shfl_xor_sync(0xffffffffu, nz, o);
    if (nz < 5) {
      for (int t = lane; t < a.n_peaks; t += 32) its[t] = -3;
      return;
    }
  }
  const JobParams c{a.kind, a.max_iter, a.x_bin, a.px, a.lsd, a.x};
  for (int jb = 0; jb < a.n_jobs; ++jb)
    fit_one_job(c, S, a.jobs[jb], a.pk_x, a.pk_bin, a.pk_id, sample, out, its, lane);
}

// ---- automatic peak detection + fit of each lineout (fitPeaksAutoDetect, PeakFit.c:720-877)
//
// One block per lineout.  SNIP background (Morhac's LLS-transformed iterative clipping,
// pf_snip_background, PeakFit.c:549-590), background-subtracted profile clipped at 0;
// Savitzky-Golay smoothing (quadratic, 7 points) and its negative second difference;
// candidates = positive local maxima of that curve on a positive profile, with the
// prominence over +-minSep bins (minSep = max(3, 3 x_bin / bin width)); the most prominent
// candidates taken greedily at least minSep bins apart, up to min(3 max_peaks, n / 2); their
// fitPeaks jobs (overlapping ROIs merged) fit on the corrected profile; then the quality
// filter: area and FWHM > 0, FWHM <= max(5 x median, 2 x_bin) when more than two remain,
// the max_peaks largest areas, in position order.
constexpr int kAutoThreads = 128;

struct AutoArgs {
  const double *x, *lineouts;
  int F, n_x, max_peaks, over, pad, snip, max_iter, fit_warps, n_max, np_max;
  double x_bin, px, lsd;
  double *out;
  int32_t *found;
  uint32_t warp_bytes, off_job;
};

__host__ __device__ inline uint32_t auto_smem(int n, int over, uint32_t warp_bytes, int fit_warps, uint32_t *off_job) {
  auto a16 = [](uint32_t x) { return (x + 15u) & ~15u; };
  uint32_t o = 0;
  o = a16(o + 8u * n);                          // corrected profile
  o = a16(o + 8u * n);                          // SNIP v / negative second difference
  o = a16(o + 8u * n);                          // copy / smoothed / prominence
  o = a16(o + 4u * (uint32_t)(n / 2 + 1));      // candidates: bins
  o = a16(o + 8u * (uint32_t)(n / 2 + 1));      //   prominences
  o = a16(o + 4u * (uint32_t)over);             // selected bins
  o = a16(o + 16u * (uint32_t)over);            // jobs
  o = a16(o + 8u * (uint32_t)over);             // peak x
  o = a16(o + 8u * MI_FIT_NOUT * (uint32_t)over);  // fits of the detected peaks
  o = a16(o + 4u * (uint32_t)over);             // their iteration counts
  o = a16(o + 16u * (uint32_t)over);            // filter entries
  o = a16(o + 64u);                             // counters
  *off_job = o;
  return o + warp_bytes * (uint32_t)fit_warps;
}

__global__ void __launch_bounds__(kAutoThreads) k_fit_autodetect(const AutoArgs a) {
  extern __shared__ __align__(16) uint8_t sm[];
  auto a16 = [](uint32_t x) { return (x + 15u) & ~15u; };
  const int n = a.n_x, over = a.over, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int64_t f = blockIdx.x;
  uint32_t o = 0;
  double *corr = (double *)(sm + o);  o = a16(o + 8u * n);
  double *v = (double *)(sm + o);     o = a16(o + 8u * n);
  double *t = (double *)(sm + o);     o = a16(o + 8u * n);
  int32_t *cbin = (int32_t *)(sm + o);  o = a16(o + 4u * (uint32_t)(n / 2 + 1));
  double *cprom = (double *)(sm + o);   o = a16(o + 8u * (uint32_t)(n / 2 + 1));
  int32_t *sel = (int32_t *)(sm + o);   o = a16(o + 4u * (uint32_t)over);
  FitJobDev *jobs = (FitJobDev *)(sm + o);  o = a16(o + 16u * (uint32_t)over);
  double *pkx = (double *)(sm + o);     o = a16(o + 8u * (uint32_t)over);
  double *raw = (double *)(sm + o);     o = a16(o + 8u * MI_FIT_NOUT * (uint32_t)over);
  int32_t *rit = (int32_t *)(sm + o);   o = a16(o + 4u * (uint32_t)over);
  double2 *ent = (double2 *)(sm + o);   o = a16(o + 16u * (uint32_t)over);   // (area, fwhm) per kept entry
  int32_t *cnt = (int32_t *)(sm + o);   // [0] candidates, [1] selected, [2] jobs, [3] kept, [4] argmax bin
  const double *y = a.lineouts + f * (int64_t)n;
  double *out = a.out + f * (int64_t)a.max_peaks * MI_FIT_NOUT;
  for (int i = tid; i < a.max_peaks * MI_FIT_NOUT; i += kAutoThreads) out[i] = 0.0;
  // ---- SNIP background
  if (a.snip > 0) {
    for (int i = tid; i < n; i += kAutoThreads) v[i] = log(log(sqrt(fmax(y[i], 0.0) + 1.0) + 1.0) + 1.0);
    __syncthreads();
    for (int p = a.snip; p >= 1; --p) {
      for (int i = tid; i < n; i += kAutoThreads) t[i] = v[i];
      __syncthreads();
      for (int i = p + tid; i < n - p; i += kAutoThreads) {
        const double avg = (t[i - p] + t[i + p]) / 2.0;
        if (v[i] > avg) v[i] = avg;
      }
      __syncthreads();
    }
    for (int i = tid; i < n; i += kAutoThreads) {
      const double w = exp(exp(v[i]) - 1.0) - 1.0;
      corr[i] = fmax(y[i] - fmax(w * w - 1.0, 0.0), 0.0);
    }
  } else {
    for (int i = tid; i < n; i += kAutoThreads) corr[i] = fmax(y[i], 0.0);
  }
  if (tid < 8) cnt[tid] = 0;
  __syncthreads();
  const bool detect = n >= 10 && a.max_peaks > 0;
  // ---- smoothing (Savitzky-Golay, quadratic, window 7) and its negative second difference
  if (detect) {
    for (int i = tid; i < n; i += kAutoThreads) {
      if (i < 3 || i >= n - 3) {
        t[i] = corr[i];
      } else {
        t[i] = (-2.0 * corr[i - 3] + 3.0 * corr[i - 2] + 6.0 * corr[i - 1] + 7.0 * corr[i] + 6.0 * corr[i + 1] +
                3.0 * corr[i + 2] - 2.0 * corr[i + 3]) / 21.0;
      }
    }
    __syncthreads();
    for (int i = tid; i < n; i += kAutoThreads)
      v[i] = (i >= 1 && i < n - 1) ? -(t[i + 1] - 2.0 * t[i] + t[i - 1]) : 0.0;
    __syncthreads();
  }
  const double bw = n > 1 ? fabs(a.x[1] - a.x[0]) : 1.0;
  const int msep = (int)fmax(3.0, (a.x_bin * 3.0) / bw);
  // ---- candidates and their prominence (NaN: not a candidate)
  if (detect) {
    for (int i = tid; i < n; i += kAutoThreads) {
      double pr = __longlong_as_double(0x7ff8000000000000ll);
      if (i >= 2 && i < n - 2 && v[i] > 0 && v[i] >= v[i - 1] && v[i] >= v[i + 1] && corr[i] > 0) {
        double lm = v[i], rm = v[i];
        for (int j = i - 1; j >= 0 && j >= i - msep; --j) lm = fmin(lm, v[j]);
        for (int j = i + 1; j < n && j <= i + msep; ++j) rm = fmin(rm, v[j]);
        pr = v[i] - fmax(lm, rm);
        if (pr < 0) pr = v[i];
      }
      t[i] = pr;
    }
    __syncthreads();
    if (tid == 0) {
      // in bin order, at most n / 2 (the reference's candidate buffer)
      int nc = 0;
      for (int i = 0; i < n && nc < n / 2; ++i)
        if (!isnan(t[i])) { cbin[nc] = i; cprom[nc] = t[i]; ++nc; }
      cnt[0] = nc;
    }
    __syncthreads();
  }
  // ---- greedy selection by prominence, at least msep bins apart
  const int nc = cnt[0];
  for (;;) {
    if (!detect || cnt[1] >= over) break;
    // the most prominent remaining candidate (lowest bin on ties)
    double best = -1e300;
    int bi = -1;
    for (int c = tid; c < nc; c += kAutoThreads)
      if (cbin[c] >= 0 && (bi < 0 || cprom[c] > best || (cprom[c] == best && cbin[c] < cbin[bi]))) {
        best = cprom[c];
        bi = c;
      }
    for (int off = 16; off > 0; off >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, off);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
      if (oi >= 0 && (bi < 0 || ob > best || (ob == best && cbin[oi] < cbin[bi]))) { best = ob; bi = oi; }
    }
    __shared__ double s_best[kAutoThreads / 32];
    __shared__ int s_bi[kAutoThreads / 32];
    if (lane == 0) { s_best[wid] = best; s_bi[wid] = bi; }
    __syncthreads();
    if (tid == 0) {
      int b2 = -1;
      double bb = -1e300;
      for (int w = 0; w < kAutoThreads / 32; ++w) {
        const int oi = s_bi[w];
        if (oi >= 0 && (b2 < 0 || s_best[w] > bb || (s_best[w] == bb && cbin[oi] < cbin[b2]))) { bb = s_best[w]; b2 = oi; }
      }
      cnt[4] = b2;
      if (b2 >= 0) {
        const int bin = cbin[b2];
        bool close = false;
        for (int k = 0; k < cnt[1]; ++k) close = close || abs(bin - sel[k]) < msep;
        if (!close) sel[cnt[1]++] = bin;
        cbin[b2] = -1;   // taken or discarded
      }
    }
    __syncthreads();
    if (cnt[4] < 0) break;
  }
  // ---- sort the selected by position; fitPeaks jobs on the corrected profile
  if (tid == 0) {
    const int ns = cnt[1];
    for (int i = 1; i < ns; ++i)
      for (int j = i; j > 0 && sel[j] < sel[j - 1]; --j) { const int q = sel[j]; sel[j] = sel[j - 1]; sel[j - 1] = q; }
    int nj = 0;
    for (int k = 0; k < ns; ++k) {
      const int b = sel[k], s0 = max(0, b - a.pad), s1 = min(n - 1, b + a.pad);
      pkx[k] = a.x[b];
      if (nj > 0 && s0 <= jobs[nj - 1].s1 && jobs[nj - 1].n_p < MI_FIT_JOB_MAX_PEAKS) {
        jobs[nj - 1].s1 = s1;
        jobs[nj - 1].n_p++;
      } else {
        jobs[nj++] = FitJobDev{s0, s1, 1, k};
      }
    }
    cnt[2] = nj;
  }
  __syncthreads();
  const int ns = cnt[1];
  for (int i = tid; i < ns * MI_FIT_NOUT; i += kAutoThreads) raw[i] = 0.0;
  for (int i = tid; i < ns; i += kAutoThreads) rit[i] = -1;
  __syncthreads();
  if (wid < a.fit_warps) {
    JobSmem S;
    job_warp_bytes(a.n_max, a.np_max, &S, sm + a.off_job + (size_t)wid * a.warp_bytes);
    const JobParams c{MI_FIT_KIND_PEAKS, a.max_iter, a.x_bin, a.px, a.lsd, a.x};
    auto sample = [&](int i) -> double { return corr[i]; };
    for (int jb = wid; jb < cnt[2]; jb += a.fit_warps)
      fit_one_job(c, S, jobs[jb], pkx, sel, nullptr, sample, raw, rit, lane);
  }
  __syncthreads();
  // ---- quality filter and output (thread 0; a few dozen entries)
  if (tid == 0) {
    int nv = 0;
    for (int i = 0; i < ns; ++i) {
      const double ar = fabs(raw[i * MI_FIT_NOUT]), fw = raw[i * MI_FIT_NOUT + 4];
      if (ar > 0 && fw > 0) {
        sel[nv] = i;                  // the entry's index among the detected peaks
        ent[nv] = make_double2(ar, fw);
        ++nv;
      }
    }
    if (nv > 2) {
      // median FWHM: the middle of the sorted FWHMs (index nv / 2)
      for (int i = 0; i < nv; ++i) t[i] = ent[i].y;
      for (int i = 1; i < nv; ++i)
        for (int j = i; j > 0 && t[j] < t[j - 1]; --j) { const double q = t[j]; t[j] = t[j - 1]; t[j - 1] = q; }
      const double cap = fmax(5.0 * t[nv / 2], a.x_bin * 2.0);
      int d = 0;
      for (int i = 0; i < nv; ++i)
        if (ent[i].y <= cap) { sel[d] = sel[i]; ent[d] = ent[i]; ++d; }
      nv = d;
    }
    if (nv > a.max_peaks) {
      // the largest areas first (exchange sort, as the reference orders them), keep max_peaks
      for (int i = 0; i < nv - 1; ++i)
        for (int j = i + 1; j < nv; ++j)
          if (ent[j].x > ent[i].x) {
            const double2 q = ent[i]; ent[i] = ent[j]; ent[j] = q;
            const int qi = sel[i]; sel[i] = sel[j]; sel[j] = qi;
          }
      nv = a.max_peaks;
    }
    for (int i = 1; i < nv; ++i)
      for (int j = i; j > 0 && sel[j] < sel[j - 1]; --j) {
        const int qi = sel[j]; sel[j] = sel[j - 1]; sel[j - 1] = qi;
      }
    cnt[3] = nv;
    a.found[f] = nv;
  }
  __syncthreads();
  for (int i = tid; i < cnt[3] * MI_FIT_NOUT; i += kAutoThreads)
    out[i] = raw[sel[i / MI_FIT_NOUT] * MI_FIT_NOUT + i % MI_FIT_NOUT];
}

}  // namespace mi

using namespace mi;

struct mi_fit_plan {
  int device = 0;
  mi_fit_job_opts opts{};
  int n_x = 0, n_peaks = 0, n_jobs = 0, n_valid = 0, max_job_peaks = 0, n_max = 0, np_max = 0;
  double *d_x = nullptr;
  FitJobDev *d_jobs = nullptr;
  double *d_pk_x = nullptr;
  int32_t *d_pk_bin = nullptr, *d_pk_id = nullptr;
  std::vector<FitJobDev> jobs;
  std::vector<int32_t> pk_bin, pk_id;
  std::vector<double> pk_x;
};

static void fit_plan_free(mi_fit_plan *fp) {
  cudaFree(fp->d_x);
  cudaFree(fp->d_jobs);
  cudaFree(fp->d_pk_x);
  cudaFree(fp->d_pk_bin);
  cudaFree(fp->d_pk_id);
}

// the jobs of fitPeaks (PeakFit.c:292-350): nearest bins, sorted, overlapping ROIs merged
static void jobs_peaks(mi_fit_plan *fp, const double *x, const double *peaks) {
  const int n_x = fp->n_x, pad = fp->opts.half_window;
  std::vector<std::pair<int, int>> valid;   // (bin, peak id)
  for (int p = 0; p < fp->n_peaks; ++p) {
    int best = -1;
    double md = 1e10;
    for (int r = 0; r < n_x; ++r) {
      const double d = fabs(x[r] - peaks[p]);
      if (d < md) { md = d; best = r; }
    }
    if (best != -1 && md < fp->opts.x_bin * 2.0) valid.push_back({best, p});
  }
  std::stable_sort(valid.begin(), valid.end(), [](const std::pair<int, int> &a, const std::pair<int, int> &b) {
    return a.first < b.first;
  });
  for (size_t i = 0; i < valid.size(); ++i) {
    const int b = valid[i].first, s = std::max(0, b - pad), e = std::min(n_x - 1, b + pad);
    if (!fp->jobs.empty() && s <= fp->jobs.back().s1 && fp->jobs.back().n_p < MI_FIT_JOB_MAX_PEAKS) {
      fp->jobs.back().s1 = e;
      fp->jobs.back().n_p++;
    } else {
      fp->jobs.push_back(FitJobDev{s, e, 1, (int32_t)fp->pk_bin.size()});
    }
    fp->pk_bin.push_back(b);
    fp->pk_id.push_back(valid[i].second);
    fp->pk_x.push_back(x[b]);
  }
}

// the per-eta jobs of IntegratorZarrOMP.c:1906-1984: doublets of adjacent peaks closer than
// doublet_sep (in the given order), ROI = bins with centres inside +- half_window bins of
// the peak(s), at least 6 bins
static void jobs_eta(mi_fit_plan *fp, const double *x, const double *peaks) {
  const int np = fp->n_peaks;
  std::vector<int> flag(np, 0), pair(np, -1);
  if (fp->opts.doublet_sep > 0.0 && np > 1)
    for (int p = 0; p < np - 1; ++p) {
      if (flag[p]) continue;
      if (fabs(peaks[p + 1] - peaks[p]) < fp->opts.doublet_sep) {
        flag[p] = 1; flag[p + 1] = 2;
        pair[p] = p + 1; pair[p + 1] = p;
      }
    }
  const double pad = fp->opts.half_window * fp->opts.x_bin;
  for (int p = 0; p < np; ++p) {
    if (flag[p] == 2) continue;
    const int q = flag[p] == 1 ? pair[p] : -1;
    const double lo_p = q >= 0 ? std::min(peaks[p], peaks[q]) : peaks[p];
    const double hi_p = q >= 0 ? std::max(peaks[p], peaks[q]) : peaks[p];
    const double rlo = lo_p - pad, rhi = hi_p + pad;
    int lo = -1, hi = -1;
    for (int r = 0; r < fp->n_x; ++r) {
      if (x[r] >= rlo && lo < 0) lo = r;
      if (x[r] <= rhi) hi = r;
    }
    if (lo < 0 || hi < 0 || hi - lo < 5) continue;
    FitJobDev jd{lo, hi, q >= 0 ? 2 : 1, (int32_t)fp->pk_bin.size()};
    fp->jobs.push_back(jd);
    if (q >= 0) {
      const int a = peaks[p] < peaks[q] ? p : q, b = peaks[p] < peaks[q] ? q : p;
      fp->pk_bin.push_back(lo); fp->pk_id.push_back(a); fp->pk_x.push_back(peaks[a]);
      fp->pk_bin.push_back(lo); fp->pk_id.push_back(b); fp->pk_x.push_back(peaks[b]);
    } else {
      fp->pk_bin.push_back(lo); fp->pk_id.push_back(p); fp->pk_x.push_back(peaks[p]);
    }
  }
}

template <typename T>
static int upload(T **dst, const std::vector<T> &v) {
  if (v.empty()) return MI_OK;
  MI_CUDA(cudaMalloc((void **)dst, v.size() * sizeof(T)));
  MI_CUDA(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return MI_OK;
}

extern "C" int mi_fit_plan_create(const double *x, int n_x, const double *peaks, int n_peaks,
                                  const mi_fit_job_opts *opts, int device, mi_fit_plan **out) {
  if (!out) return set_error(MI_E_ARG, "mi_fit_plan_create: null output");
  *out = nullptr;
  if (!x || !opts || (n_peaks > 0 && !peaks)) return set_error(MI_E_ARG, "mi_fit_plan_create: null argument");
  if (n_x <= 0 || n_peaks < 0) return set_error(MI_E_ARG, "mi_fit_plan_create: n_x %d, n_peaks %d", n_x, n_peaks);
  if (opts->kind != MI_FIT_KIND_PEAKS && opts->kind != MI_FIT_KIND_ETA)
    return set_error(MI_E_ARG, "mi_fit_plan_create: unknown kind %d", opts->kind);
  if (!(opts->x_bin > 0)) return set_error(MI_E_ARG, "mi_fit_plan_create: x_bin must be > 0");
  if (opts->half_window < 1) return set_error(MI_E_ARG, "mi_fit_plan_create: half_window must be >= 1");
  mi_fit_plan *fp = new mi_fit_plan();
  fp->device = device;
  fp->opts = *opts;
  if (fp->opts.max_iter <= 0) fp->opts.max_iter = 200;
  fp->n_x = n_x;
  fp->n_peaks = n_peaks;
  if (opts->kind == MI_FIT_KIND_PEAKS) jobs_peaks(fp, x, peaks);
  else jobs_eta(fp, x, peaks);
  fp->n_jobs = (int)fp->jobs.size();
  fp->n_valid = (int)fp->pk_bin.size();
  for (const FitJobDev &j : fp->jobs) {
    fp->max_job_peaks = std::max(fp->max_job_peaks, j.n_p);
    fp->n_max = std::max(fp->n_max, j.s1 - j.s0 + 1);
    const int np = opts->kind == MI_FIT_KIND_PEAKS ? 4 * j.n_p + 2 : 3 * j.n_p + 2;
    fp->np_max = std::max(fp->np_max, np);
  }
  if (device < 0) {
    // host-only plan: the job table without device buffers (mi_fit_plan_info / _jobs only)
    *out = fp;
    return MI_OK;
  }
  int prev = 0;
  cudaGetDevice(&prev);
  int rc = cudaSetDevice(device) == cudaSuccess ? MI_OK : set_error(MI_E_CUDA, "mi_fit_plan_create: bad device");
  if (rc == MI_OK) {
    const uint32_t wb = job_warp_bytes(fp->n_max, fp->np_max, nullptr, nullptr);
    int dev_smem = 0;
    cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (fp->n_jobs > 0 && wb > (uint32_t)dev_smem)
      rc = set_error(MI_E_RANGE, "mi_fit_plan_create: a job of %d samples x %d parameters needs %u B of shared memory",
                     fp->n_max, fp->np_max, wb);
  }
  std::vector<double> xv(x, x + n_x);
  if (rc == MI_OK) rc = upload(&fp->d_x, xv);
  if (rc == MI_OK) rc = upload(&fp->d_jobs, fp->jobs);
  if (rc == MI_OK) rc = upload(&fp->d_pk_x, fp->pk_x);
  if (rc == MI_OK) rc = upload(&fp->d_pk_bin, fp->pk_bin);
  if (rc == MI_OK) rc = upload(&fp->d_pk_id, fp->pk_id);
  cudaSetDevice(prev);
  if (rc != MI_OK) {
    fit_plan_free(fp);
    delete fp;
    return rc;
  }
  *out = fp;
  return MI_OK;
}

extern "C" int mi_fit_plan_info(const mi_fit_plan *fp, int *n_jobs, int *n_valid, int *max_job_peaks) {
  if (!fp) return set_error(MI_E_ARG, "mi_fit_plan_info: null plan");
  if (n_jobs) *n_jobs = fp->n_jobs;
  if (n_valid) *n_valid = fp->n_valid;
  if (max_job_peaks) *max_job_peaks = fp->max_job_peaks;
  return MI_OK;
}

extern "C" int mi_fit_plan_jobs(const mi_fit_plan *fp, int32_t *jobs, int32_t *peak_ids) {
  if (!fp) return set_error(MI_E_ARG, "mi_fit_plan_jobs: null plan");
  for (int j = 0; j < fp->n_jobs && jobs; ++j) {
    jobs[4 * j] = fp->jobs[j].s0;
    jobs[4 * j + 1] = fp->jobs[j].s1;
    jobs[4 * j + 2] = fp->jobs[j].n_p;
    jobs[4 * j + 3] = fp->jobs[j].p0;
  }
  for (int k = 0; k < fp->n_valid && peak_ids; ++k) peak_ids[k] = fp->pk_id[k];
  return MI_OK;
}

extern "C" int mi_fit_plan_run(const mi_fit_plan *fp, const void *src, int src_dtype, int n_series, int n_sub,
                               int64_t ld_series, int64_t ld_sub, int64_t ld_x, double *out, int32_t *iters,
                               void *stream) {
  if (!fp || !src || !out || !iters) return set_error(MI_E_ARG, "mi_fit_plan_run: null argument");
  if (fp->device < 0) return set_error(MI_E_ARG, "mi_fit_plan_run: a host-only plan (device < 0) cannot run");
  if (src_dtype != MI_DT_F32 && src_dtype != MI_DT_F64)
    return set_error(MI_E_ARG, "mi_fit_plan_run: series must be float32 or float64 (dtype %d)", src_dtype);
  if (n_series < 0 || n_sub < 1 || ld_x < 1)
    return set_error(MI_E_ARG, "mi_fit_plan_run: n_series %d, n_sub %d, ld_x %lld", n_series, n_sub,
                     (long long)ld_x);
  const int64_t total = (int64_t)n_series * n_sub;
  if (total == 0 || fp->n_peaks == 0) return MI_OK;
  const int64_t blocks = (total + kJobWarps - 1) / kJobWarps;
  if (blocks > INT32_MAX) return set_error(MI_E_RANGE, "mi_fit_plan_run: too many series");
  FitPlanArgs a;
  a.jobs = fp->d_jobs;
  a.pk_x = fp->d_pk_x;
  a.pk_bin = fp->d_pk_bin;
  a.pk_id = fp->d_pk_id;
  a.x = fp->d_x;
  a.src = src;
  a.src_f64 = src_dtype == MI_DT_F64;
  a.ld_series = ld_series;
  a.ld_sub = ld_sub;
  a.ld_x = ld_x;
  a.n_series = n_series;
  a.n_sub = n_sub;
  a.n_x = fp->n_x;
  a.n_jobs = fp->n_jobs;
  a.n_peaks = fp->n_peaks;
  a.kind = fp->opts.kind;
  a.max_iter = fp->opts.max_iter;
  a.np_max = std::max(fp->np_max, 2);
  a.n_max = std::max(fp->n_max, 1);
  a.x_bin = fp->opts.x_bin;
  a.px = fp->opts.px_um;
  a.lsd = fp->opts.lsd_um;
  a.out = out;
  a.iters = iters;
  a.warp_bytes = job_warp_bytes(a.n_max, a.np_max, nullptr, nullptr);
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != fp->device) MI_CUDA(cudaSetDevice(fp->device));
  const size_t smem = (size_t)a.warp_bytes * kJobWarps;
  int dev_smem = 0;
  int rc = MI_OK;
  cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, fp->device);
  if (smem > (size_t)dev_smem) {
    rc = set_error(MI_E_RANGE, "mi_fit_plan_run: %zu B of shared memory per block (device allows %d)", smem, dev_smem);
  } else {
    cudaError_t e = cudaFuncSetAttribute(k_fit_job, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) {
      k_fit_job<<<(unsigned)blocks, 32 * kJobWarps, smem, (cudaStream_t)stream>>>(a);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) rc = cuda_error(e, "k_fit_job", __FILE__, __LINE__);
  }
  if (prev != fp->device) cudaSetDevice(prev);
  return rc;
}

extern "C" void mi_fit_plan_destroy(mi_fit_plan *fp) {
  if (!fp) return;
  if (fp->device < 0) {
    delete fp;
    return;
  }
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(fp->device);
  fit_plan_free(fp);
  cudaSetDevice(prev);
  delete fp;
}

extern "C" int mi_fit_autodetect(const double *x, const double *lineouts, int n_frames, int n_x, int max_peaks,
                                 double x_bin, int roi_padding, int snip_iter, double px_um, double lsd_um,
                                 double *out, int32_t *n_found, void *stream) {
  if (!x || !lineouts || !out || !n_found) return set_error(MI_E_ARG, "mi_fit_autodetect: null argument");
  if (n_frames < 0 || n_x < 0 || max_peaks < 0 || roi_padding < 1 || !(x_bin > 0))
    return set_error(MI_E_ARG, "mi_fit_autodetect: bad sizes or bin width");
  if (n_frames == 0 || n_x == 0 || max_peaks == 0) return MI_OK;
  AutoArgs a;
  a.x = x;
  a.lineouts = lineouts;
  a.F = n_frames;
  a.n_x = n_x;
  a.max_peaks = max_peaks;
  a.over = std::max(1, std::min(max_peaks * 3, n_x / 2));
  a.pad = roi_padding;
  a.snip = snip_iter;
  a.max_iter = 200;
  a.x_bin = x_bin;
  a.px = px_um;
  a.lsd = lsd_um;
  a.out = out;
  a.found = n_found;
  a.n_max = std::min(n_x, MI_FIT_JOB_MAX_PEAKS * (2 * roi_padding + 1));
  a.np_max = 4 * MI_FIT_JOB_MAX_PEAKS + 2;
  a.warp_bytes = job_warp_bytes(a.n_max, a.np_max, nullptr, nullptr);
  int dev = 0, dev_smem = 0;
  MI_CUDA(cudaGetDevice(&dev));
  MI_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  uint32_t total = 0;
  for (a.fit_warps = kAutoThreads / 32; a.fit_warps >= 1; --a.fit_warps) {
    total = auto_smem(n_x, a.over, a.warp_bytes, a.fit_warps, &a.off_job);
    if (total <= (uint32_t)dev_smem) break;
  }
  if (a.fit_warps < 1)
    return set_error(MI_E_RANGE, "mi_fit_autodetect: %d samples with +-%d-bin windows need %u B of shared memory",
                     n_x, roi_padding, total);
  MI_CUDA(cudaFuncSetAttribute(k_fit_autodetect, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)total));
  k_fit_autodetect<<<(unsigned)n_frames, kAutoThreads, total, (cudaStream_t)stream>>>(a);
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}
