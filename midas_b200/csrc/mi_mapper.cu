// mi_mapper.cu -- DetectorMapper on the device (and, from the same source, on the host).
//
// Builds the Map.bin / nMap.bin pixel-split map: for every detector pixel (and
// sub-pixel when SubPixelLevel > 1) the four corners are mapped to (R, eta)
// with the tilt + p0..p14 distortion + parallax forward model, brought back to
// the ideal (y, z) plane, and the exact overlap area of that quadrilateral with
// each candidate annular-sector bin is computed by clipping (corner tests,
// segment/circle and segment/ray intersections) and Green's theorem with arc
// edges.  The steps and thresholds follow mapper_build_map
// (FF_HEDM/src/MapperCore.c:45-424) and the helpers of
// FF_HEDM/src/DetectorGeometry.c (dg_pixel_to_REta_corr :95, dg_polygon_area
// :432, dg_circle_seg_intersect :507, dg_ray_seg_intersect :536,
// dg_point_in_quad :555, dg_find_unique_vertices :572); the code is written
// for one thread per pixel with a count pass, a scan and a fill pass.
#include <cub/cub.cuh>
#include <math.h>
#include <omp.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "mi_internal.h"

#define MI_HD __host__ __device__

namespace mi {

struct MapGeom {
  int ny, nz;
  double px, lsd, bcy, bcz, rhod, parallax, polf, spw;
  double T[3][3];
  double p[15];
  int sa, pol, spl;
};

struct MapBins {
  int n_r, n_eta;
  const double *rlo, *rhi, *elo, *ehi;
};

constexpr double kD2R = 0.017453292519943295;  // pi / 180
constexpr double kR2D = 57.29577951308232;     // 180 / pi
constexpr double kGeomEps = 1e-6;
constexpr int kMaxVerts = 48;

MI_HD inline double eta_of(double y, double z) { return kR2D * atan2(-y, z); }
MI_HD inline double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
MI_HD inline bool within(double v, double lo, double hi) { return v - kGeomEps <= hi && v + kGeomEps >= lo; }

static void tilt_matrix(double tx, double ty, double tz, double T[3][3]) {
  const double a = kD2R * tx, b = kD2R * ty, c = kD2R * tz;
  const double Rx[3][3] = {{1, 0, 0}, {0, cos(a), -sin(a)}, {0, sin(a), cos(a)}};
  const double Ry[3][3] = {{cos(b), 0, sin(b)}, {0, 1, 0}, {-sin(b), 0, cos(b)}};
  const double Rz[3][3] = {{cos(c), -sin(c), 0}, {sin(c), cos(c), 0}, {0, 0, 1}};
  double M[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) M[i][j] = Ry[i][0] * Rz[0][j] + Ry[i][1] * Rz[1][j] + Ry[i][2] * Rz[2][j];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) T[i][j] = Rx[i][0] * M[0][j] + Rx[i][1] * M[1][j] + Rx[i][2] * M[2][j];
}

// forward model: pixel (Y, Z) -> (R px, eta deg)
MI_HD inline void pix_to_reta(const MapGeom &g, double Y, double Z, double *R, double *E) {
  const double yc = (-Y + g.bcy) * g.px, zc = (Z - g.bcz) * g.px;
  const double x0 = g.T[0][1] * yc + g.T[0][2] * zc;
  const double x1 = g.T[1][1] * yc + g.T[1][2] * zc;
  const double x2 = g.T[2][1] * yc + g.T[2][2] * zc;
  const double X = g.lsd + x0;
  const double rad = (g.lsd / X) * sqrt(x1 * x1 + x2 * x2);
  const double eta = eta_of(x1, x2);
  const double rn = g.rhod != 0.0 ? rad / g.rhod : 0.0;
  const double et = 90.0 - eta;
  const double *p = g.p;
  double d = 1.0;
  if (p[0] != 0 || p[1] != 0 || p[2] != 0 || p[4] != 0 || p[5] != 0 || p[7] != 0 || p[9] != 0 ||
      p[11] != 0 || p[13] != 0) {
    const double r2 = rn * rn, r3 = r2 * rn, r4 = r2 * r2, r5 = r4 * rn, r6 = r3 * r3;
    d = p[0] * r2 * cos(kD2R * (2 * et + p[6])) + p[1] * r4 * cos(kD2R * (4 * et + p[3])) + p[2] * r2 +
        p[4] * r6 + p[5] * r4 + p[7] * r4 * cos(kD2R * (et + p[8])) +
        p[9] * r3 * cos(kD2R * (3 * et + p[10])) + p[11] * r5 * cos(kD2R * (5 * et + p[12])) +
        p[13] * r6 * cos(kD2R * (6 * et + p[14])) + 1.0;
  }
  double rt = rad * d / g.px;
  if (g.parallax != 0.0) rt += g.parallax * sin(atan(rad / g.lsd)) / g.px;
  *R = rt;
  *E = eta;
}

MI_HD inline void reta_to_yz(double R, double E, double *y, double *z) {
  *y = -R * sin(E * kD2R);
  *z = R * cos(E * kD2R);
}

// quad corners c[k*2+l] = (dy[k], dz[l]); perimeter order 0,1,3,2
MI_HD inline int qord(int e) { return e == 0 ? 0 : (e == 1 ? 1 : (e == 2 ? 3 : 2)); }

MI_HD inline bool in_quad(double py, double pz, const double q[4][2]) {
  int pos = 0, neg = 0;
  for (int e = 0; e < 4; ++e) {
    const int i0 = qord(e), i1 = qord((e + 1) & 3);
    const double ey = q[i1][0] - q[i0][0], ez = q[i1][1] - q[i0][1];
    const double cr = ey * (pz - q[i0][1]) - ez * (py - q[i0][0]);
    if (cr > 0) ++pos;
    else if (cr < 0) ++neg;
  }
  return pos == 0 || neg == 0;
}

MI_HD inline int seg_circle(double y1, double z1, double y2, double z2, double R, double h[2][2]) {
  const double dy = y2 - y1, dz = z2 - z1;
  const double a = dy * dy + dz * dz;
  if (a < 1e-30) return 0;
  const double b = 2.0 * (y1 * dy + z1 * dz);
  const double c = y1 * y1 + z1 * z1 - R * R;
  const double disc = b * b - 4.0 * a * c;
  if (disc < 0) return 0;
  const double s = sqrt(disc), inv2a = 0.5 / a;
  int n = 0;
  const double t1 = (-b - s) * inv2a;
  if (t1 >= -kGeomEps && t1 <= 1.0 + kGeomEps) {
    const double t = fmax(0.0, fmin(1.0, t1));
    h[n][0] = y1 + t * dy; h[n][1] = z1 + t * dz; ++n;
  }
  const double t2 = (-b + s) * inv2a;
  if (t2 >= -kGeomEps && t2 <= 1.0 + kGeomEps && fabs(t2 - t1) > 1e-12) {
    const double t = fmax(0.0, fmin(1.0, t2));
    h[n][0] = y1 + t * dy; h[n][1] = z1 + t * dz; ++n;
  }
  return n;
}

MI_HD inline bool seg_ray(double y1, double z1, double y2, double z2, double eta, double *hy, double *hz) {
  const double er = eta * kD2R, ce = cos(er), se = sin(er);
  const double dy = y2 - y1, dz = z2 - z1;
  const double den = dy * ce + dz * se;
  if (fabs(den) < 1e-30) return false;
  double t = -(y1 * ce + z1 * se) / den;
  if (t < -kGeomEps || t > 1.0 + kGeomEps) return false;
  t = fmax(0.0, fmin(1.0, t));
  *hy = y1 + t * dy;
  *hz = z1 + t * dz;
  return (-se) * (*hy) + ce * (*hz) >= 0;
}

// angular order around the centroid (the comparator of dg_polygon_area): a "after" b
MI_HD inline bool after(double ax, double ay, double bx, double by) {
  if (ax >= 0 && bx < 0) return true;
  if (ax < 0 && bx >= 0) return false;
  if (ax == 0 && bx == 0) {
    // ay/by are centroid-relative here; the reference compares the absolute y
    return false;
  }
  const double det = ax * by - bx * ay;
  if (det < 0) return true;
  if (det > 0) return false;
  return ax * ax + ay * ay > bx * bx + by * by;
}

MI_HD inline double poly_area(double (*v)[2], int n, double rmin, double rmax) {
  double cx = 0, cy = 0;
  for (int i = 0; i < n; ++i) { cx += v[i][0]; cy += v[i][1]; }
  cx /= n;
  cy /= n;
  // insertion sort by angular order
  for (int i = 1; i < n; ++i) {
    const double x = v[i][0], y = v[i][1];
    int j = i - 1;
    while (j >= 0) {
      const double ax = v[j][0] - cx, ay = v[j][1] - cy, bx = x - cx, by = y - cy;
      bool gt;
      if (ax == 0 && bx == 0) {
        gt = (ay >= 0 || by >= 0) ? (v[j][1] > y) : (y > v[j][1]);
      } else {
        gt = after(ax, ay, bx, by);
      }
      if (!gt) break;
      v[j + 1][0] = v[j][0];
      v[j + 1][1] = v[j][1];
      --j;
    }
    v[j + 1][0] = x;
    v[j + 1][1] = y;
  }
  const double r2min = rmin * rmin, r2max = rmax * rmax, tol = 1e-6;
  double A = 0;
  for (int i = 0; i < n; ++i) {
    const int k = (i + 1) % n;
    const double r1 = v[i][0] * v[i][0] + v[i][1] * v[i][1];
    const double r2 = v[k][0] * v[k][0] + v[k][1] * v[k][1];
    const bool on_min = fabs(r1 - r2min) < tol * r2min && fabs(r2 - r2min) < tol * r2min;
    const bool on_max = fabs(r1 - r2max) < tol * r2max && fabs(r2 - r2max) < tol * r2max;
    if (on_min || on_max) {
      const double R = on_min ? rmin : rmax;
      double d = atan2(v[k][1], v[k][0]) - atan2(v[i][1], v[i][0]);
      if (d > M_PI) d -= 2.0 * M_PI;
      if (d < -M_PI) d += 2.0 * M_PI;
      A += (R * R / 2.0) * d;
    } else {
      A += 0.5 * (v[i][0] * v[k][1] - v[k][0] * v[i][1]);
    }
  }
  return A;
}

MI_HD inline double adj_eta(double et, double emin, double emax) {
  if (emin < -180 && sgn(et) != sgn(emin)) et -= 360;
  if (emax > 180 && sgn(et) != sgn(emax)) et += 360;
  return et;
}

// overlap area of pixel quad q with bin [rmin,rmax] x [emin,emax]
MI_HD inline double quad_bin_area(const double q[4][2], double rmin, double rmax, double emin, double emax) {
  double ed[kMaxVerts][2];
  int n = 0;
  double box[4][2];
  reta_to_yz(rmin, emin, &box[0][0], &box[0][1]);
  reta_to_yz(rmin, emax, &box[1][0], &box[1][1]);
  reta_to_yz(rmax, emin, &box[2][0], &box[2][1]);
  reta_to_yz(rmax, emax, &box[3][0], &box[3][1]);
  for (int m = 0; m < 4; ++m) {
    const double R = sqrt(q[m][0] * q[m][0] + q[m][1] * q[m][1]);
    const double E = adj_eta(eta_of(q[m][0], q[m][1]), emin, emax);
    if (R >= rmin && R <= rmax && E >= emin && E <= emax) {
      ed[n][0] = q[m][0]; ed[n][1] = q[m][1]; ++n;
    }
  }
  for (int m = 0; m < 4; ++m)
    if (in_quad(box[m][0], box[m][1], q)) {
      ed[n][0] = box[m][0]; ed[n][1] = box[m][1]; ++n;
    }
  if (n < 4) {
    for (int e = 0; e < 4; ++e) {
      const int i0 = qord(e), i1 = qord((e + 1) & 3);
      const double y1 = q[i0][0], z1 = q[i0][1], y2 = q[i1][0], z2 = q[i1][1];
      double h[2][2];
      int nh = seg_circle(y1, z1, y2, z2, rmin, h);
      for (int k = 0; k < nh; ++k) {
        const double E = adj_eta(eta_of(h[k][0], h[k][1]), emin, emax);
        if (E >= emin - kGeomEps && E <= emax + kGeomEps && n < kMaxVerts) {
          ed[n][0] = h[k][0]; ed[n][1] = h[k][1]; ++n;
        }
      }
      nh = seg_circle(y1, z1, y2, z2, rmax, h);
      for (int k = 0; k < nh; ++k) {
        const double E = adj_eta(eta_of(h[k][0], h[k][1]), emin, emax);
        if (E >= emin - kGeomEps && E <= emax + kGeomEps && n < kMaxVerts) {
          ed[n][0] = h[k][0]; ed[n][1] = h[k][1]; ++n;
        }
      }
      double hy, hz;
      if (seg_ray(y1, z1, y2, z2, emin, &hy, &hz)) {
        const double R = sqrt(hy * hy + hz * hz);
        if (R >= rmin - kGeomEps && R <= rmax + kGeomEps && n < kMaxVerts) { ed[n][0] = hy; ed[n][1] = hz; ++n; }
      }
      if (seg_ray(y1, z1, y2, z2, emax, &hy, &hz)) {
        const double R = sqrt(hy * hy + hz * hz);
        if (R >= rmin - kGeomEps && R <= rmax + kGeomEps && n < kMaxVerts) { ed[n][0] = hy; ed[n][1] = hz; ++n; }
      }
    }
  }
  if (n < 3) return 0.0;
  // unique vertices inside the bin (a vertex equal to a later one is dropped)
  double uv[kMaxVerts][2];
  int nu = 0;
  for (int i = 0; i < n; ++i) {
    bool drop = false;
    for (int j = i + 1; j < n; ++j) {
      const double dy = ed[i][0] - ed[j][0], dz = ed[i][1] - ed[j][1];
      if (sqrt(dy * dy + dz * dz) == 0) drop = true;
    }
    const double R = sqrt(ed[i][0] * ed[i][0] + ed[i][1] * ed[i][1]);
    double E = eta_of(ed[i][0], ed[i][1]);
    if (!within(E, emin, emax)) {
      if (within(E + 360, emin, emax)) E += 360;
      else if (within(E - 360, emin, emax)) E -= 360;
    }
    if (!within(R, rmin, rmax)) drop = true;
    if (!within(E, emin, emax)) drop = true;
    if (!drop) { uv[nu][0] = ed[i][0]; uv[nu][1] = ed[i][1]; ++nu; }
  }
  if (nu < 3) return 0.0;
  return poly_area(uv, nu, rmin, rmax);
}

struct Entry {
  int32_t bin;
  mi_map_record rec;
};

// All entries of pixel (i = y, j = z) in the mapper's order (sub-pixel, R bin, eta bin).
// emit(bin, rec) is called per entry; mask(bin) per bin touched by a masked pixel.
template <typename Emit, typename MaskF>
MI_HD inline void pixel_entries(const MapGeom &g, const MapBins &B, int i, int j, bool masked, Emit emit,
                                MaskF mask) {
  const double ypr = (double)i, zpr = (double)j;
  int spl = 1;
  if (g.spl > 1) {
    double Rc, Ec;
    pix_to_reta(g, ypr, zpr, &Rc, &Ec);
    const double ae = fabs(Ec);
    if (ae <= g.spw || fabs(ae - 90.0) <= g.spw || fabs(ae - 180.0) <= g.spw) spl = g.spl;
  }
  for (int si = 0; si < spl; ++si)
    for (int sj = 0; sj < spl; ++sj) {
      const double dyl = (double)si / spl - 0.5, dyh = (double)(si + 1) / spl - 0.5;
      const double dzl = (double)sj / spl - 0.5, dzh = (double)(sj + 1) / spl - 0.5;
      const double scy = ((double)(2 * si + 1) / (2.0 * spl)) - 0.5;
      const double scz = ((double)(2 * sj + 1) / (2.0 * spl)) - 0.5;
      const double dys[2] = {dyl, dyh}, dzs[2] = {dzl, dzh};
      double emi = 1800, ema = -1800, rmi = 1e8, rma = -1000;
      double q[4][2];
      for (int k = 0; k < 2; ++k)
        for (int l = 0; l < 2; ++l) {
          double R, E;
          pix_to_reta(g, ypr + dys[k], zpr + dzs[l], &R, &E);
          emi = fmin(emi, E); ema = fmax(ema, E);
          rmi = fmin(rmi, R); rma = fmax(rma, R);
          reta_to_yz(R, E, &q[k * 2 + l][0], &q[k * 2 + l][1]);
        }
      double Rt, Et;
      pix_to_reta(g, ypr + scy, zpr + scz, &Rt, &Et);
      // R bins overlapping [rmi, rma]: contiguous for ascending, non-overlapping edges
      int lo = 0, hi = B.n_r;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (B.rhi[mid] >= rmi) hi = mid;
        else lo = mid + 1;
      }
      double elo = emi, ehi = ema;
      if (ehi - elo > 180) {
        const double t = ehi;
        ehi = 360 + elo;
        elo = t;
      }
      for (int kr = lo; kr < B.n_r && B.rlo[kr] <= rma; ++kr) {
        if (!(B.rhi[kr] >= rmi)) continue;
        const double rmin = B.rlo[kr], rmax = B.rhi[kr];
        for (int ke = 0; ke < B.n_eta; ++ke) {
          const double a = B.elo[ke], b = B.ehi[ke];
          if (!((b >= elo && a <= ehi) || (b >= elo + 360 && a <= ehi + 360) ||
                (b >= elo - 360 && a <= ehi - 360)))
            continue;
          const int32_t bin = kr * B.n_eta + ke;
          if (masked) {
            if (si == 0 && sj == 0) mask(bin);
            continue;
          }
          const double A = quad_bin_area(q, rmin, rmax, a, b);
          if (A < 1e-5) continue;
          double corr = A;
          if (g.sa || g.pol) {
            const double tth = atan(Rt * g.px / g.lsd);
            if (g.sa) {
              const double c = cos(tth);
              corr /= (c * c * c);
            }
            if (g.pol) {
              const double s = sin(tth), ce = cos(Et * kD2R);
              const double pf = 1.0 - g.polf * s * s * ce * ce;
              if (pf > 1e-6) corr /= pf;
            }
          }
          mi_map_record rec;
          rec.y = (float)i + (float)scy;
          rec.z = (float)j + (float)scz;
          rec.frac = corr;
          rec.deltaR = (float)(Rt - (rmin + rmax) * 0.5);
          rec.areaWeight = (float)A;
          emit(bin, rec);
        }
      }
    }
}

// ---------------------------------------------------------------------------
// device build
// ---------------------------------------------------------------------------
__global__ void k_map_count(MapGeom g, MapBins B, const uint8_t *mask, int32_t *cnt, int32_t *bin_mask) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)g.ny * g.nz) return;
  const int i = (int)(t / g.nz), j = (int)(t % g.nz);
  const bool m = mask && mask[(int64_t)j * g.ny + i];
  int32_t n = 0;
  pixel_entries(g, B, i, j, m, [&](int32_t, const mi_map_record &) { ++n; },
                [&](int32_t bin) { bin_mask[bin] = 1; });
  cnt[t] = n;
}

__global__ void k_map_fill(MapGeom g, MapBins B, const uint8_t *mask, const int64_t *off, int32_t *keys,
                           mi_map_record *recs, int32_t *bin_counts) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)g.ny * g.nz) return;
  const int i = (int)(t / g.nz), j = (int)(t % g.nz);
  const bool m = mask && mask[(int64_t)j * g.ny + i];
  int64_t o = off[t];
  pixel_entries(g, B, i, j, m,
                [&](int32_t bin, const mi_map_record &r) {
                  keys[o] = bin;
                  recs[o] = r;
                  atomicAdd(bin_counts + bin, 1);
                  ++o;
                },
                [&](int32_t) {});
}

__global__ void k_gather_recs(const int32_t *idx, const mi_map_record *src, mi_map_record *dst, int64_t n) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = src[idx[t]];
}

__global__ void k_iota(int32_t *v, int64_t n) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) v[t] = (int32_t)t;
}

}  // namespace mi

struct mi_map {
  std::vector<mi_map_record> recs;
  std::vector<int32_t> nmap;      // pairs
  std::vector<int32_t> bin_mask;  // n_bins
  int64_t n_bins = 0;
};

using namespace mi;

static int make_geom(const mi_geometry *gi, const mi_binning *b, MapGeom *g) {
  if (!gi || !b) return set_error(MI_E_ARG, "mi_map_build: null argument");
  if (gi->ny < 2 || gi->nz < 2 || gi->px_um <= 0 || gi->lsd_um <= 0)
    return set_error(MI_E_ARG, "mi_map_build: bad geometry");
  if (b->n_r <= 0 || b->n_eta <= 0 || !b->r_lo || !b->r_hi || !b->eta_lo || !b->eta_hi)
    return set_error(MI_E_ARG, "mi_map_build: bad binning");
  if ((int64_t)b->n_r * b->n_eta > INT32_MAX) return set_error(MI_E_RANGE, "mi_map_build: too many bins");
  for (int k = 1; k < b->n_r; ++k)
    if (!(b->r_lo[k] >= b->r_lo[k - 1]) || !(b->r_hi[k] >= b->r_hi[k - 1]))
      return set_error(MI_E_ARG, "mi_map_build: R bin edges must be ascending");
  g->ny = gi->ny;
  g->nz = gi->nz;
  g->px = gi->px_um;
  g->lsd = gi->lsd_um;
  g->bcy = gi->bc_y;
  g->bcz = gi->bc_z;
  g->rhod = gi->rho_d;
  g->parallax = gi->parallax_um;
  g->polf = gi->pol_fraction;
  g->sa = gi->solid_angle ? 1 : 0;
  g->pol = gi->polarization ? 1 : 0;
  g->spl = gi->sub_pixel_level > 1 ? gi->sub_pixel_level : 1;
  g->spw = gi->sub_pixel_cardinal_width;
  for (int k = 0; k < 15; ++k) g->p[k] = gi->p[k];
  tilt_matrix(gi->tx, gi->ty, gi->tz, g->T);
  return MI_OK;
}

static void finish_map(mi_map *m, int64_t n_bins, const std::vector<int32_t> &bin_counts) {
  m->n_bins = n_bins;
  m->nmap.resize(2 * n_bins);
  int64_t o = 0;
  for (int64_t b = 0; b < n_bins; ++b) {
    m->nmap[2 * b] = bin_counts[b];
    m->nmap[2 * b + 1] = (int32_t)o;
    o += bin_counts[b];
  }
}

static int build_host(const MapGeom &g, const MapBins &B, const uint8_t *mask, mi_map *m) {
  const int64_t n_bins = (int64_t)B.n_r * B.n_eta;
  m->bin_mask.assign(n_bins, 0);
  const int nthr = omp_get_max_threads();
  std::vector<std::vector<std::vector<Entry>>> per(g.ny);  // per column i
  std::vector<std::vector<Entry>> cols(g.ny);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthr)
  for (int i = 0; i < g.ny; ++i) {
    std::vector<Entry> &v = cols[i];
    for (int j = 0; j < g.nz; ++j) {
      const bool msk = mask && mask[(int64_t)j * g.ny + i];
      pixel_entries(g, B, i, j, msk, [&](int32_t bin, const mi_map_record &r) { v.push_back({bin, r}); },
                    [&](int32_t bin) {
#pragma omp atomic write
                      m->bin_mask[bin] = 1;
                    });
    }
  }
  std::vector<int32_t> counts(n_bins, 0);
  int64_t total = 0;
  for (auto &v : cols) {
    total += (int64_t)v.size();
    for (auto &e : v) ++counts[e.bin];
  }
  if (total > INT32_MAX) return set_error(MI_E_RANGE, "mi_map_build: more than 2^31 map entries");
  finish_map(m, n_bins, counts);
  m->recs.resize(total);
  std::vector<int64_t> cur(n_bins);
  for (int64_t b = 0; b < n_bins; ++b) cur[b] = m->nmap[2 * b + 1];
  for (auto &v : cols)
    for (auto &e : v) m->recs[cur[e.bin]++] = e.rec;
  return MI_OK;
}

// The whole build runs on a stream of its own with stream-ordered allocations: nothing in
// it waits for the device as a whole (cudaFree does), so other host threads' streams, a
// server's batches among them, keep running while a map is built.
static int build_device(const MapGeom &g, const MapBins &Bh, const uint8_t *mask_h, int device, mi_map *m) {
  const int64_t n_pix = (int64_t)g.ny * g.nz;
  const int64_t n_bins = (int64_t)Bh.n_r * Bh.n_eta;
  MI_CUDA(cudaSetDevice(device));
  cudaStream_t st = nullptr;
  MI_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  std::vector<void *> owned;
  auto dalloc = [&](void **p, size_t bytes) -> cudaError_t {
    cudaError_t e = cudaMallocAsync(p, std::max<size_t>(bytes, 16), st);
    if (e == cudaSuccess) owned.push_back(*p);
    return e;
  };
  auto cleanup = [&]() {
    for (void *p : owned) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  };
  // host <-> device copies on the build's stream, in 4 MB pieces (pageable host memory)
  auto copy = [&](void *dst, const void *src, size_t bytes, cudaMemcpyKind kind) -> cudaError_t {
    constexpr size_t kPiece = size_t(4) << 20;
    for (size_t o = 0; o < bytes; o += kPiece) {
      cudaError_t e = cudaMemcpyAsync((uint8_t *)dst + o, (const uint8_t *)src + o, std::min(kPiece, bytes - o),
                                      kind, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  };
#define MI_DCHK(call)                                                     \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                              \
      int r_ = cuda_error(e_, #call, __FILE__, __LINE__);                 \
      cleanup();                                                          \
      return r_;                                                          \
    }                                                                     \
  } while (0)
  double *d_edges = nullptr;
  MI_DCHK(dalloc((void **)&d_edges, sizeof(double) * (2 * Bh.n_r + 2 * Bh.n_eta)));
  MI_DCHK(copy(d_edges, Bh.rlo, sizeof(double) * Bh.n_r, cudaMemcpyHostToDevice));
  MI_DCHK(copy(d_edges + Bh.n_r, Bh.rhi, sizeof(double) * Bh.n_r, cudaMemcpyHostToDevice));
  MI_DCHK(copy(d_edges + 2 * Bh.n_r, Bh.elo, sizeof(double) * Bh.n_eta, cudaMemcpyHostToDevice));
  MI_DCHK(copy(d_edges + 2 * Bh.n_r + Bh.n_eta, Bh.ehi, sizeof(double) * Bh.n_eta, cudaMemcpyHostToDevice));
  MapBins B = Bh;
  B.rlo = d_edges;
  B.rhi = d_edges + Bh.n_r;
  B.elo = d_edges + 2 * Bh.n_r;
  B.ehi = d_edges + 2 * Bh.n_r + Bh.n_eta;
  uint8_t *d_mask = nullptr;
  if (mask_h) {
    MI_DCHK(dalloc((void **)&d_mask, n_pix));
    MI_DCHK(copy(d_mask, mask_h, n_pix, cudaMemcpyHostToDevice));
  }
  int32_t *d_cnt = nullptr, *d_bmask = nullptr, *d_bcnt = nullptr;
  int64_t *d_off = nullptr;
  MI_DCHK(dalloc((void **)&d_cnt, sizeof(int32_t) * n_pix));
  MI_DCHK(dalloc((void **)&d_off, sizeof(int64_t) * (n_pix + 1)));
  MI_DCHK(dalloc((void **)&d_bmask, sizeof(int32_t) * n_bins));
  MI_DCHK(dalloc((void **)&d_bcnt, sizeof(int32_t) * n_bins));
  MI_DCHK(cudaMemsetAsync(d_bmask, 0, sizeof(int32_t) * n_bins, st));
  MI_DCHK(cudaMemsetAsync(d_bcnt, 0, sizeof(int32_t) * n_bins, st));
  const int thr = 128;
  const unsigned grid = (unsigned)((n_pix + thr - 1) / thr);
  k_map_count<<<grid, thr, 0, st>>>(g, B, d_mask, d_cnt, d_bmask);
  MI_DCHK(cudaGetLastError());
  // exclusive scan of counts (int64)
  {
    size_t tmp_bytes = 0;
    MI_DCHK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_cnt, d_off, n_pix + 0, st));
    void *tmp = nullptr;
    MI_DCHK(dalloc(&tmp, tmp_bytes));
    MI_DCHK(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, d_cnt, d_off, n_pix, st));
  }
  int64_t last_off = 0;
  int32_t last_cnt = 0;
  MI_DCHK(copy(&last_off, d_off + n_pix - 1, sizeof(int64_t), cudaMemcpyDeviceToHost));
  MI_DCHK(copy(&last_cnt, d_cnt + n_pix - 1, sizeof(int32_t), cudaMemcpyDeviceToHost));
  const int64_t total = last_off + last_cnt;
  if (total > INT32_MAX) {
    cleanup();
    return set_error(MI_E_RANGE, "mi_map_build: more than 2^31 map entries");
  }
  int32_t *d_keys = nullptr, *d_keys2 = nullptr, *d_idx = nullptr, *d_idx2 = nullptr;
  mi_map_record *d_recs = nullptr, *d_recs2 = nullptr;
  MI_DCHK(dalloc((void **)&d_keys, sizeof(int32_t) * total));
  MI_DCHK(dalloc((void **)&d_keys2, sizeof(int32_t) * total));
  MI_DCHK(dalloc((void **)&d_idx, sizeof(int32_t) * total));
  MI_DCHK(dalloc((void **)&d_idx2, sizeof(int32_t) * total));
  MI_DCHK(dalloc((void **)&d_recs, sizeof(mi_map_record) * total));
  MI_DCHK(dalloc((void **)&d_recs2, sizeof(mi_map_record) * total));
  k_map_fill<<<grid, thr, 0, st>>>(g, B, d_mask, d_off, d_keys, d_recs, d_bcnt);
  MI_DCHK(cudaGetLastError());
  if (total > 0) {
    k_iota<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(d_idx, total);
    MI_DCHK(cudaGetLastError());
    int end_bit = 1;
    while (end_bit < 31 && ((int64_t)1 << end_bit) < n_bins) ++end_bit;
    size_t tmp_bytes = 0;
    MI_DCHK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_keys, d_keys2, d_idx, d_idx2, (int)total, 0,
                                            end_bit, st));
    void *tmp = nullptr;
    MI_DCHK(dalloc(&tmp, tmp_bytes));
    MI_DCHK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, d_keys, d_keys2, d_idx, d_idx2, (int)total, 0,
                                            end_bit, st));
    k_gather_recs<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(d_idx2, d_recs, d_recs2, total);
    MI_DCHK(cudaGetLastError());
  }
  std::vector<int32_t> counts(n_bins);
  m->bin_mask.resize(n_bins);
  m->recs.resize(total);
  MI_DCHK(copy(counts.data(), d_bcnt, sizeof(int32_t) * n_bins, cudaMemcpyDeviceToHost));
  MI_DCHK(copy(m->bin_mask.data(), d_bmask, sizeof(int32_t) * n_bins, cudaMemcpyDeviceToHost));
  if (total > 0)
    MI_DCHK(copy(m->recs.data(), d_recs2, sizeof(mi_map_record) * total, cudaMemcpyDeviceToHost));
  finish_map(m, n_bins, counts);
  cleanup();
#undef MI_DCHK
  return MI_OK;
}

extern "C" {

int mi_map_build(const mi_geometry *geom, const mi_binning *bins, int device, mi_map **out) {
  if (!out) return set_error(MI_E_ARG, "mi_map_build: null output");
  *out = nullptr;
  MapGeom g;
  int rc = make_geom(geom, bins, &g);
  if (rc) return rc;
  MapBins B{bins->n_r, bins->n_eta, bins->r_lo, bins->r_hi, bins->eta_lo, bins->eta_hi};
  mi_map *m = new (std::nothrow) mi_map();
  if (!m) return set_error(MI_E_OOM, "mi_map_build: host allocation failed");
  if (device < 0) {
    rc = build_host(g, B, geom->mask_host, m);
  } else {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device >= ndev) {
      delete m;
      return set_error(MI_E_CUDA, "mi_map_build: CUDA device %d not available", device);
    }
    int prev = 0;
    cudaGetDevice(&prev);
    rc = build_device(g, B, geom->mask_host, device, m);
    cudaSetDevice(prev);
  }
  if (rc) {
    delete m;
    return rc;
  }
  *out = m;
  return MI_OK;
}

int mi_map_sizes(const mi_map *m, int64_t *n_records, int64_t *n_bins) {
  if (!m) return set_error(MI_E_ARG, "mi_map_sizes: null map");
  if (n_records) *n_records = (int64_t)m->recs.size();
  if (n_bins) *n_bins = m->n_bins;
  return MI_OK;
}

int mi_map_copy(const mi_map *m, mi_map_record *records, int32_t *nmap, int32_t *bin_mask) {
  if (!m) return set_error(MI_E_ARG, "mi_map_copy: null map");
  if (records && !m->recs.empty()) memcpy(records, m->recs.data(), m->recs.size() * sizeof(mi_map_record));
  if (nmap) memcpy(nmap, m->nmap.data(), m->nmap.size() * sizeof(int32_t));
  if (bin_mask) memcpy(bin_mask, m->bin_mask.data(), m->bin_mask.size() * sizeof(int32_t));
  return MI_OK;
}

void mi_map_destroy(mi_map *m) { delete m; }

}  // extern "C"
