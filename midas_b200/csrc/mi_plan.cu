// mi_plan.cu -- plan creation: map validation, per-mode CSR, tiling, upload.
//
// Host side of the drop-in boundary.  The CSR construction restates
// build_csr() of packages/midas_integrate/midas_integrate/kernels.py:242-375
// (floor: one term per record, off-detector records dropped; bilinear and
// gradient: four clamped corner terms per record, duplicates summed, exact
// zeros removed), with the GPU-stream normaliser of
// FF_HEDM/src/IntegratorFitPeaksGPUStream.cu:994-1049 as a selectable
// semantic.  The tiled encoding is this library's own (see mi_internal.h).
#include <omp.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <numeric>

#include "mi_internal.h"

#ifndef MI_MMA_MIN_PIECE
#define MI_MMA_MIN_PIECE 2   // fewest pixels of a run piece placed in skipped slots
#endif

namespace mi {

static thread_local char g_err[1024] = "";

int set_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int cuda_error(cudaError_t e, const char *what, const char *file, int line) {
  return set_error(e == cudaErrorMemoryAllocation ? MI_E_OOM : MI_E_CUDA,
                   "CUDA error %s (%s) in %s at %s:%d", cudaGetErrorName(e),
                   cudaGetErrorString(e), what, file, line);
}

cudaError_t copy_pieces(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind) {
  // A synchronous copy from or to pageable memory keeps other host threads' copy calls on
  // the device waiting until it ends (a serving thread's frame upload waited for a plan's
  // map upload); in pieces, such a call waits for one piece at most.
  constexpr size_t kPiece = size_t(4) << 20;
  for (size_t o = 0; o < bytes; o += kPiece) {
    const cudaError_t e = cudaMemcpy((uint8_t *)dst + o, (const uint8_t *)src + o, std::min(kPiece, bytes - o), kind);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

size_t dtype_size(int dtype) {
  switch (dtype) {
    case MI_DT_U8: return 1;
    case MI_DT_U16: return 2;
    case MI_DT_U32: return 4;
    case MI_DT_I64: return 8;
    case MI_DT_F32: return 4;
    case MI_DT_F64: return 8;
    case MI_DT_I32: return 4;
    default: return 0;
  }
}

// ---------------------------------------------------------------------------
// CSR of one mode.  Per record (y, z, frac, deltaR, areaWeight):
//  * in-bounds test on the truncated (y, z) (kernels.py:306-311) decides
//    whether areaWeight enters area_in (the profile / Python normaliser);
//  * MI_SEM_GPUSTREAM normalises by the sum of all areaWeight of the bin
//    (IntegratorFitPeaksGPUStream.cu:1034-1040).
// ---------------------------------------------------------------------------
struct Term {
  int32_t col;
  double w;
};

static inline void add_bilinear(double sy, double sz, double frac, int ny, int nz,
                                std::vector<Term> &t) {
  // kernels.py:_build_bilinear_csr: floor, then clamp (over first, then under)
  double fiy = std::floor(sy), fiz = std::floor(sz);
  int64_t iy = (int64_t)fiy, iz = (int64_t)fiz;
  double fy = sy - (double)iy, fz = sz - (double)iz;
  bool over_y = iy >= (ny - 1), under_y = iy < 0;
  bool over_z = iz >= (nz - 1), under_z = iz < 0;
  if (over_y) { iy = ny - 2; fy = 1.0; }
  if (under_y) { iy = 0; fy = 0.0; }
  if (over_z) { iz = nz - 2; fz = 1.0; }
  if (under_z) { iz = 0; fz = 0.0; }
  int64_t base = iz * (int64_t)ny + iy;
  double one_fy = 1.0 - fy, one_fz = 1.0 - fz;
  t.push_back({(int32_t)base, one_fy * one_fz * frac});
  t.push_back({(int32_t)(base + 1), fy * one_fz * frac});
  t.push_back({(int32_t)(base + ny), one_fy * fz * frac});
  t.push_back({(int32_t)(base + ny + 1), fy * fz * frac});
}

// integration_apply_map (IntegrationCore.c:52-63): the base pixel is floorf() of the FP64
// position (rounded to float on the way in), the fractions are taken from the FP64
// position, and the clamps run under-then-over
static inline void add_bilinear_ic(double sy, double sz, double frac, int ny, int nz,
                                   std::vector<Term> &t) {
  int iy = (int)floorf((float)sy), iz = (int)floorf((float)sz);
  double fy = sy - iy, fz = sz - iz;
  if (iy < 0) { iy = 0; fy = 0; }
  if (iy >= ny - 1) { iy = ny - 2; fy = 1; }
  if (iz < 0) { iz = 0; fz = 0; }
  if (iz >= nz - 1) { iz = nz - 2; fz = 1; }
  const int64_t base = (int64_t)iz * ny + iy;
  t.push_back({(int32_t)base, (1 - fy) * (1 - fz) * frac});
  t.push_back({(int32_t)(base + 1), fy * (1 - fz) * frac});
  t.push_back({(int32_t)(base + ny), (1 - fy) * fz * frac});
  t.push_back({(int32_t)(base + ny + 1), fy * fz * frac});
}

static void bin_terms(const mi_map_desc &m, int64_t b, int mode, int sem,
                      std::vector<Term> &t, double *area_in, double *area_all,
                      int64_t *oob) {
  t.clear();
  const int32_t cnt = m.nmap[2 * b], off = m.nmap[2 * b + 1];
  double ain = 0.0, aall = 0.0;
  const int ny = m.ny, nz = m.nz;
  for (int32_t k = 0; k < cnt; ++k) {
    const mi_map_record &r = m.records[(int64_t)off + k];
    const double y = (double)r.y, z = (double)r.z;
    // numpy astype(int64) truncates toward zero
    const int64_t ty = (int64_t)y, tz = (int64_t)z;
    const bool inb = ty >= 0 && ty < ny && tz >= 0 && tz < nz;
    aall += (double)r.areaWeight;
    if (inb) ain += (double)r.areaWeight;
    else ++*oob;
    if (mode == MI_MODE_FLOOR) {
      if (sem == MI_SEM_GPUSTREAM) {
        // PrecomputeOffsets_kernel: (long long)z * NY + y evaluated in float,
        // then truncated (IntegratorFitPeaksGPUStream.cu:915-916)
        long long zz = (long long)r.z;
        float s = (float)(zz * (long long)ny) + r.y;
        long long o = (long long)s;
        if (o >= 0 && o < (long long)ny * nz) t.push_back({(int32_t)o, r.frac});
      } else if (inb) {
        t.push_back({(int32_t)(tz * ny + ty), r.frac});
      }
    } else if (sem == MI_SEM_IC || sem == MI_SEM_OMP) {
      // IntegrationCore.c:38-50: FP64 shift, only for records with deltaR != 0 and R > 1
      double sy = y, sz = z;
      if (mode == MI_MODE_GRADIENT && r.deltaR != 0.0f) {
        const double dy = y - m.bc_y, dz = z - m.bc_z;
        const double R = std::sqrt(dy * dy + dz * dz);
        if (R > 1.0) {
          sy -= r.deltaR * dy / R;
          sz -= r.deltaR * dz / R;
        }
      }
      add_bilinear_ic(sy, sz, r.frac, ny, nz, t);
    } else {
      double sy = y, sz = z;
      if (mode == MI_MODE_GRADIENT) {
        if (sem == MI_SEM_GPUSTREAM) {
          // fp32 resampling of integrate_noMapMask (…Stream.cu:1007-1018)
          float dy = r.y - (float)m.bc_y, dz = r.z - (float)m.bc_z;
          float R = sqrtf(dy * dy + dz * dz);
          float ry = r.y, rz = r.z;
          if (R > 1.0f) {
            ry -= r.deltaR * dy / R;
            rz -= r.deltaR * dz / R;
          }
          sy = ry;
          sz = rz;
        } else {
          // kernels.py:347-353 (fp64)
          double dy = y - m.bc_y, dz = z - m.bc_z;
          double R = std::sqrt(dy * dy + dz * dz);
          double sc = R > 1.0 ? (double)r.deltaR / R : 0.0;
          sy = y - sc * dy;
          sz = z - sc * dz;
        }
      }
      add_bilinear(sy, sz, r.frac, ny, nz, t);
    }
  }
  *area_in = ain;
  *area_all = aall;
  // coalesce duplicates (sum), drop exact zeros (scipy sum_duplicates + eliminate_zeros)
  std::stable_sort(t.begin(), t.end(), [](const Term &a, const Term &b) { return a.col < b.col; });
  size_t o = 0;
  for (size_t i = 0; i < t.size();) {
    size_t j = i;
    double s = 0.0;
    while (j < t.size() && t[j].col == t[i].col) s += t[j++].w;
    if (s != 0.0 || mode == MI_MODE_FLOOR) t[o++] = {t[i].col, s};
    i = j;
  }
  t.resize(o);
  if (mode == MI_MODE_FLOOR) {
    // floor CSR keeps explicit zeros only if frac was zero; drop them too (no effect on sums)
    size_t q = 0;
    for (size_t i = 0; i < t.size(); ++i)
      if (t[i].w != 0.0) t[q++] = t[i];
    t.resize(q);
  }
}

int build_host_csr(const mi_map_desc &m, int mode, int sem, HostCSR *out) {
  const int64_t n_bins = (int64_t)m.n_r * m.n_eta;
  // validation (kernels.py:288-301), plus negative offsets
  for (int64_t b = 0; b < n_bins; ++b) {
    const int64_t c = m.nmap[2 * b], o = m.nmap[2 * b + 1];
    if (c < 0) return set_error(MI_E_MAP, "nMap.bin bin %lld has negative count %lld", (long long)b, (long long)c);
    if (c > 0 && (o < 0 || o + c > m.n_records))
      return set_error(MI_E_MAP, "bin %lld references past end of Map.bin (offset %lld, count %lld, n_records %lld)",
                       (long long)b, (long long)o, (long long)c, (long long)m.n_records);
  }
  std::vector<int64_t> counts(n_bins + 1, 0);
  out->area_in.assign(n_bins, 0.0);
  out->area_norm.assign(n_bins, 0.0);
  std::vector<double> area_all(n_bins, 0.0);
  out->area_gs.assign(n_bins, 0.0);
  int64_t oob_total = 0;
  // pass 1: term counts
#pragma omp parallel reduction(+ : oob_total)
  {
    std::vector<Term> t;
    t.reserve(1024);
#pragma omp for schedule(dynamic, 256)
    for (int64_t b = 0; b < n_bins; ++b) {
      double ain, aall;
      int64_t oob = 0;
      bin_terms(m, b, mode, sem, t, &ain, &aall, &oob);
      counts[b + 1] = (int64_t)t.size();
      out->area_in[b] = ain;
      area_all[b] = aall;
      oob_total += oob;
      // initialize_PerFrameArr_Area_kernel (IntegratorFitPeaksGPUStream.cu:858-873): the
      // record's float position inside [0, ny) x [0, nz), and its flat index
      // (long long)z * ny + y, evaluated in float, below ny * nz
      double ags = 0.0;
      const int64_t n_pix = (int64_t)m.ny * m.nz;
      for (int32_t k = 0; k < m.nmap[2 * b]; ++k) {
        const mi_map_record &r = m.records[(int64_t)m.nmap[2 * b + 1] + k];
        if (r.y < 0 || r.y >= m.ny || r.z < 0 || r.z >= m.nz) continue;
        const float flat = (float)((int64_t)r.z * m.ny) + r.y;
        if ((int64_t)flat >= n_pix) continue;
        ags += r.areaWeight;
      }
      out->area_gs[b] = ags;
    }
  }
  out->row_ptr.assign(n_bins + 1, 0);
  for (int64_t b = 0; b < n_bins; ++b) out->row_ptr[b + 1] = out->row_ptr[b] + counts[b + 1];
  const int64_t nnz = out->row_ptr[n_bins];
  out->col.resize(nnz);
  out->w.resize(nnz);
#pragma omp parallel
  {
    std::vector<Term> t;
    t.reserve(1024);
#pragma omp for schedule(dynamic, 256)
    for (int64_t b = 0; b < n_bins; ++b) {
      double ain, aall;
      int64_t oob = 0;
      bin_terms(m, b, mode, sem, t, &ain, &aall, &oob);
      int64_t o = out->row_ptr[b];
      for (const Term &x : t) {
        out->col[o] = x.col;
        out->w[o] = x.w;
        ++o;
      }
    }
  }
  for (int64_t b = 0; b < n_bins; ++b)
    out->area_norm[b] = (sem == MI_SEM_PY) ? out->area_in[b] : area_all[b];
  out->oob = oob_total;
  return MI_OK;
}

// ---------------------------------------------------------------------------
// Tiling
// ---------------------------------------------------------------------------
struct HostTile {
  int r0, n_rows, e0, n_cols, nnz, n_u;
};

struct Builder {
  const HostCSR &csr;
  int n_r, n_eta;
  int64_t n_pix;
  TileLimits lim;
  Builder(const HostCSR &c, int nr, int ne, int64_t np, TileLimits l)
      : csr(c), n_r(nr), n_eta(ne), n_pix(np), lim(l) {}
};

// Greedily cover rows [r0, r0+nrows) x cols [e_begin, e_end) with tiles.
static int tile_item(const Builder &B, int r0, int nrows, int e_begin, int e_end,
                     std::vector<int32_t> &stamp, int32_t &stamp_id,
                     std::vector<HostTile> &tiles) {
  const TileLimits &L = B.lim;
  auto col_terms = [&](int r, int e) {
    int64_t b = (int64_t)r * B.n_eta + e;
    return std::make_pair(B.csr.row_ptr[b], B.csr.row_ptr[b + 1]);
  };
  // unique pixels of a rectangle
  std::vector<int32_t> added;
  auto rect_fits = [&](int rc, int h, int e0, int ncols, int *nu_out, int *nnz_out) {
    ++stamp_id;
    int nu = 0, nnz = 0;
    for (int e = e0; e < e0 + ncols; ++e)
      for (int r = rc; r < rc + h; ++r) {
        auto pr = col_terms(r, e);
        nnz += (int)(pr.second - pr.first);
        for (int64_t j = pr.first; j < pr.second; ++j) {
          int32_t c = B.csr.col[j];
          if (stamp[c] != stamp_id) { stamp[c] = stamp_id; ++nu; }
        }
      }
    *nu_out = nu;
    *nnz_out = nnz;
    return nu <= L.max_u && nnz <= L.max_nnz && h * ncols <= L.max_nb && ncols <= L.max_cols;
  };
  // row-chunk height: largest h (halving) such that every single column fits
  int h = nrows;
  for (;;) {
    bool ok = true;
    for (int rc = r0; rc < r0 + nrows && ok; rc += h) {
      int hh = std::min(h, r0 + nrows - rc);
      for (int e = e_begin; e < e_end && ok; ++e) {
        int nu, nnz;
        if (!rect_fits(rc, hh, e, 1, &nu, &nnz)) ok = false;
      }
    }
    if (ok) break;
    if (h == 1)
      return set_error(MI_E_RANGE,
                       "a single bin (row %d) references more pixels or terms than one tile holds "
                       "(max %d pixels, %d terms); raise tile_pixels",
                       r0, L.max_u, L.max_nnz);
    h = (h + 1) / 2;
  }
  for (int rc = r0; rc < r0 + nrows; rc += h) {
    int hh = std::min(h, r0 + nrows - rc);
    int e = e_begin;
    while (e < e_end) {
      int ncols = 1, nu = 0, nnz = 0;
      rect_fits(rc, hh, e, 1, &nu, &nnz);
      while (e + ncols < e_end) {
        int nu2, nnz2;
        if (!rect_fits(rc, hh, e, ncols + 1, &nu2, &nnz2)) break;
        ++ncols;
        nu = nu2;
        nnz = nnz2;
      }
      tiles.push_back({rc, hh, e, ncols, nnz, nu});
      e += ncols;
    }
  }
  return MI_OK;
}

// normalisation factor and lineout weight of bin b (see mi_internal.h)
static inline void bin_scale(const HostCSR &csr, const Plan *p, int64_t b, float *scale, float *lw,
                             double *scale64 = nullptr) {
  const double an = csr.area_norm[b], ai = csr.area_in[b];
  double sc;
  if (p->semantics == MI_SEM_OMP)
    // IntegratorZarrOMP.c:1749-1753: a nonzero sum is divided by the area, whatever its size
    sc = p->normalize ? (an > 0.0 ? 1.0 / an : 0.0) : 1.0;
  else if (p->semantics != MI_SEM_PY)
    sc = an > kAreaThreshold ? (p->normalize ? 1.0 / an : 1.0) : 0.0;
  else
    sc = p->normalize ? (ai > kAreaThreshold ? 1.0 / ai : 0.0) : 1.0;
  // variance plans (integrate_with_variance, kernels.py:551-559; profile_1d_with_variance,
  // kernels.py:604-645): Var = sum w^2 var / A^2, lineout weight A^2
  if (p->variance) sc *= sc;
  if (scale64) *scale64 = sc;
  *scale = (float)sc;
  *lw = ai > kAreaThreshold ? (float)(p->variance ? ai * ai : ai) : 0.0f;
}

// staged pixel set of a tile (ascending), with lut[pixel] = local index
static std::vector<int32_t> tile_pixels(const HostCSR &csr, const mi_map_desc &m, const HostTile &t,
                                        std::vector<int32_t> &lut) {
  std::vector<int32_t> u;
  u.reserve(t.n_u);
  for (int r = t.r0; r < t.r0 + t.n_rows; ++r)
    for (int e = t.e0; e < t.e0 + t.n_cols; ++e) {
      const int64_t b = (int64_t)r * m.n_eta + e;
      for (int64_t j = csr.row_ptr[b]; j < csr.row_ptr[b + 1]; ++j) u.push_back(csr.col[j]);
    }
  std::sort(u.begin(), u.end());
  u.erase(std::unique(u.begin(), u.end()), u.end());
  for (size_t i = 0; i < u.size(); ++i) lut[u[i]] = (int32_t)i;
  return u;
}

static void csr_blob(const HostCSR &csr, const mi_map_desc &m, const Plan *p, const HostTile &t, int row_in_band,
                     std::vector<int32_t> &lut, std::vector<uint8_t> &out) {
  const int nb = t.n_rows * t.n_cols;
  uint32_t o_rp, o_sc, o_lw, o_up, o_lc, o_w, bytes;
  blob_layout(nb, t.nnz, t.n_u, &o_rp, &o_sc, &o_lw, &o_up, &o_lc, &o_w, &bytes);
  out.assign(bytes, 0);
  uint8_t *blob = out.data();
  TileHdr *h = (TileHdr *)blob;
  *h = TileHdr{nb, t.nnz, t.n_u, t.n_rows, t.n_cols, t.r0, t.e0, row_in_band};
  uint32_t *rowp = (uint32_t *)(blob + o_rp);
  double *scale = (double *)(blob + o_sc);
  float *lw = (float *)(blob + o_lw);
  uint32_t *upix = (uint32_t *)(blob + o_up);
  uint16_t *lcol = (uint16_t *)(blob + o_lc);
  float *wt = (float *)(blob + o_w);
  std::vector<int32_t> u = tile_pixels(csr, m, t, lut);
  for (size_t i = 0; i < u.size(); ++i) upix[i] = (uint32_t)u[i];
  uint32_t nz_o = 0;
  for (int r = t.r0; r < t.r0 + t.n_rows; ++r)
    for (int e = t.e0; e < t.e0 + t.n_cols; ++e) {
      const int64_t b = (int64_t)r * m.n_eta + e;
      const int lb = (r - t.r0) * t.n_cols + (e - t.e0);
      rowp[lb] = nz_o;
      for (int64_t j = csr.row_ptr[b]; j < csr.row_ptr[b + 1]; ++j) {
        lcol[nz_o] = (uint16_t)lut[csr.col[j]];
        wt[nz_o] = (float)csr.w[j];
        ++nz_o;
      }
      float sc32;
      bin_scale(csr, p, b, &sc32, lw + lb, scale + lb);
    }
  rowp[nb] = nz_o;
  for (int32_t v : u) lut[v] = -1;
}

struct RunRec {
  int rs, u;
  float w[8];
};

static void runs_blob(const HostCSR &csr, const mi_map_desc &m, const Plan *p, const HostTile &t, int row_in_band,
                      int G, int L, std::vector<int32_t> &lut, std::vector<uint8_t> &out) {
  const int nb = t.n_rows * t.n_cols, NRS = G - L + 2;
  std::vector<int32_t> u = tile_pixels(csr, m, t, lut);
  std::vector<uint16_t> rsp((size_t)t.n_cols * NRS, 0);
  std::vector<RunRec> all;
  struct Trip {
    int u, row;
    double w;
  };
  std::vector<Trip> trip;
  std::vector<RunRec> recs;
  for (int c = 0; c < t.n_cols; ++c) {
    trip.clear();
    for (int i = 0; i < t.n_rows; ++i) {
      const int64_t b = (int64_t)(t.r0 + i) * m.n_eta + t.e0 + c;
      for (int64_t j = csr.row_ptr[b]; j < csr.row_ptr[b + 1]; ++j) trip.push_back({lut[csr.col[j]], i, csr.w[j]});
    }
    std::sort(trip.begin(), trip.end(), [](const Trip &a, const Trip &b) {
      return a.u != b.u ? a.u < b.u : a.row < b.row;
    });
    recs.clear();
    for (size_t k = 0; k < trip.size();) {
      const int uu = trip[k].u;
      while (k < trip.size() && trip[k].u == uu) {
        RunRec r;
        r.rs = std::min(trip[k].row, G - L);
        r.u = uu;
        for (int q = 0; q < 8; ++q) r.w[q] = 0.0f;
        while (k < trip.size() && trip[k].u == uu && trip[k].row < r.rs + L) {
          r.w[trip[k].row - r.rs] = (float)trip[k].w;
          ++k;
        }
        recs.push_back(r);
      }
    }
    std::stable_sort(recs.begin(), recs.end(), [](const RunRec &a, const RunRec &b) { return a.rs < b.rs; });
    const size_t base = all.size();
    size_t k = 0;
    for (int q = 0; q < NRS; ++q) {
      while (k < recs.size() && recs[k].rs < q) ++k;
      rsp[(size_t)c * NRS + q] = (uint16_t)(base + (q == NRS - 1 ? recs.size() : k));
    }
    all.insert(all.end(), recs.begin(), recs.end());
  }
  const int n_rec = (int)all.size();
  uint32_t o_rsp, o_sc, o_lw, o_up, o_lc, o_w;
  const uint32_t bytes = runs_blob_layout(nb, t.n_cols, n_rec, t.n_u, G, L, &o_rsp, &o_sc, &o_lw, &o_up, &o_lc, &o_w);
  out.assign(bytes, 0);
  uint8_t *blob = out.data();
  *(TileHdr *)blob = TileHdr{nb, n_rec, t.n_u, t.n_rows, t.n_cols, t.r0, t.e0, row_in_band};
  // consumer units: every strip gets at least one; the rest go one by one to the strip with
  // the most records per unit; a strip's records are split evenly between its units
  {
    std::vector<int> cnt(t.n_cols), K(t.n_cols, 1);
    for (int c = 0; c < t.n_cols; ++c) cnt[c] = rsp[(size_t)c * NRS + NRS - 1] - rsp[(size_t)c * NRS];
    for (int left = kRunWarps - t.n_cols; left > 0; --left) {
      int best = 0;
      for (int c = 1; c < t.n_cols; ++c)
        if ((int64_t)cnt[c] * K[best] > (int64_t)cnt[best] * K[c]) best = c;
      ++K[best];
    }
    uint16_t *ut = (uint16_t *)(blob + kRunUnitsOff);
    uint16_t *st = ut + 4 * kRunWarps;
    int w = 0;
    for (int c = 0; c < t.n_cols; ++c) {
      const int j0 = rsp[(size_t)c * NRS];
      st[2 * c] = (uint16_t)w;
      st[2 * c + 1] = (uint16_t)K[c];
      for (int q = 0; q < K[c]; ++q, ++w) {
        ut[4 * w] = (uint16_t)c;
        ut[4 * w + 1] = (uint16_t)(j0 + (int)((int64_t)cnt[c] * q / K[c]));
        ut[4 * w + 2] = (uint16_t)(j0 + (int)((int64_t)cnt[c] * (q + 1) / K[c]));
        ut[4 * w + 3] = 0;
      }
    }
  }
  memcpy(blob + o_rsp, rsp.data(), rsp.size() * sizeof(uint16_t));
  double *scale = (double *)(blob + o_sc);
  float *lw = (float *)(blob + o_lw);
  for (int r = 0; r < t.n_rows; ++r)
    for (int c = 0; c < t.n_cols; ++c) {
      float sc32;
      bin_scale(csr, p, (int64_t)(t.r0 + r) * m.n_eta + t.e0 + c, &sc32, lw + r * t.n_cols + c,
                scale + r * t.n_cols + c);
    }
  uint32_t *upix = (uint32_t *)(blob + o_up);
  for (size_t i = 0; i < u.size(); ++i) upix[i] = (uint32_t)u[i];
  uint16_t *lcol = (uint16_t *)(blob + o_lc);
  float *w = (float *)(blob + o_w);
  for (int i = 0; i < n_rec; ++i) {
    lcol[i] = (uint16_t)all[i].u;
    for (int q = 0; q < L; ++q) w[(size_t)i * L + q] = all[i].w[q];
  }
  for (int32_t v : u) lut[v] = -1;
}

// Rows per record: the candidate (2, 4 or 8 <= G/2) with the least estimated work
// (records x (L + 6) instructions) over a sample of strips.
static int choose_run_len(const HostCSR &csr, const mi_map_desc &m, int rows, int G) {
  const int cands[3] = {2, 4, 8};
  double cost[3] = {0, 0, 0};
  std::vector<std::pair<int32_t, int>> pr;
  const int bands = (m.n_r + rows - 1) / rows;
  for (int band = 0; band < bands; band += std::max(1, bands / 24))
    for (int e = 0; e < m.n_eta; e += std::max(1, m.n_eta / 16)) {
      pr.clear();
      for (int i = 0; i < rows && band * rows + i < m.n_r; ++i) {
        const int64_t b = (int64_t)(band * rows + i) * m.n_eta + e;
        for (int64_t j = csr.row_ptr[b]; j < csr.row_ptr[b + 1]; ++j) pr.push_back({csr.col[j], i});
      }
      std::sort(pr.begin(), pr.end());
      for (int ci = 0; ci < 3; ++ci) {
        const int L = cands[ci];
        if (L > G / 2 || (G >= 16 && L == 2)) { cost[ci] = 1e300; continue; }
        int64_t nrec = 0;
        for (size_t k = 0; k < pr.size();) {
          const int32_t uu = pr[k].first;
          while (k < pr.size() && pr[k].first == uu) {
            const int rs = std::min(pr[k].second, G - L);
            while (k < pr.size() && pr[k].first == uu && pr[k].second < rs + L) ++k;
            ++nrec;
          }
        }
        cost[ci] += (double)nrec * (L + 6);
      }
    }
  int best = 1;
  for (int ci = 0; ci < 3; ++ci)
    if (cost[ci] < cost[best]) best = ci;
  return cands[best];
}

static int free_plan_mem(Plan *p) {
  cudaSetDevice(p->device);
  void *ptrs[] = {p->d_blobs, p->d_tiles, p->d_items, p->d_den_aw, p->d_cnt, p->d_partial,
                  p->d_dark, p->d_err, p->d_nmap, p->d_sorted, p->d_off, p->d_w, p->d_aw,
                  p->d_dr, p->d_py, p->d_pz, p->d_area_in, p->d_area_all, p->d_plain_img,
                  p->d_ctr, p->d_span_lo, p->d_row_off, p->d_xchunks, p->d_xc,
                  p->d_xc_pix, p->d_nan_bins};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  return MI_OK;
}

template <typename T>
static int upload(T **dst, const T *src, size_t n, size_t *acct) {
  size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
  MI_CUDA(cudaMalloc((void **)dst, bytes));
  *acct += bytes;
  if (n) MI_CUDA(copy_pieces(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return MI_OK;
}

// A weight of a tensor-core tile: signed fixed point relative to the bin's largest |w|,
// packed as four s8 digits (mma_digits).
static uint32_t mma_weight(double w, double wm) {
  double qd = wm > 0.0 ? (double)std::llround(w / wm * kMmaQMax) : 0.0;
  qd = std::min(std::max(qd, -kMmaQMax), kMmaQMax);
  return mma_digits((int64_t)qd);
}

// Within each K step, order the terms so that every 32 consecutive ones (the 32 lanes of one
// store of the B operand builders, which start at the step's first term) fall in distinct
// shared-memory banks as far as the step's terms allow: each group takes one term per bank,
// fullest banks first, and repeats banks only when fewer than 32 are left to draw from.
static void bank_order(std::vector<uint2> &terms, const std::vector<uint32_t> &sp, int n_k) {
  std::vector<uint2> bucket[32];
  int order[32];
  for (int st = 0; st < n_k; ++st) {
    for (auto &b : bucket) b.clear();
    for (uint32_t t = sp[st]; t < sp[st + 1]; ++t)
      bucket[mma_bank(terms[t].y >> 16, (terms[t].y & 0xFFFFu) % kMmaKStep)].push_back(terms[t]);
    uint32_t pos = sp[st];
    while (pos < sp[st + 1]) {
      for (int b = 0; b < 32; ++b) order[b] = b;
      std::stable_sort(order, order + 32, [&](int x, int y) { return bucket[x].size() > bucket[y].size(); });
      const uint32_t g_end = std::min(pos + 32u, sp[st + 1]);
      while (pos < g_end)
        for (int i = 0; i < 32 && pos < g_end; ++i)
          if (!bucket[order[i]].empty()) {
            terms[pos++] = bucket[order[i]].back();
            bucket[order[i]].pop_back();
          }
    }
  }
}

// ---- MMA encoding: tiles of up to kMmaRows x kMmaCols bins (see MmaHdr).  Each band of
// kMmaRows rows is cut into sub-bands of h rows (h = 12, 6, 3, 1: the largest whose tile
// blobs all fit the kernel's blob slots); a work item is a sub-band x item_cols columns,
// its tiles the item's groups of kMmaCols columns, all on the item's rows.
static int mma_tile_blob(const HostCSR &csr, const mi_map_desc &m, const std::vector<int32_t> &span_lo,
                         const std::vector<int32_t> &row_off, const std::vector<double> &wmax,
                         const std::vector<double> &fac, const std::vector<float> &lw, int r0, int nr, int box_rows,
                         int e0, int nc, std::vector<int32_t> &lut, std::vector<uint8_t> &blob, int *nnz_out,
                         int *nu_out) {
  std::vector<int32_t> pix;
  for (int i = 0; i < nr; ++i)
    for (int j = 0; j < nc; ++j) {
      const int64_t b = (int64_t)(r0 + i) * m.n_eta + e0 + j;
      for (int64_t t = csr.row_ptr[b]; t < csr.row_ptr[b + 1]; ++t)
        if (lut[csr.col[t]] < 0) {
          lut[csr.col[t]] = 0;
          pix.push_back(csr.col[t]);
        }
    }
  // K slots.  The tile's pixels form runs of consecutive compact indices (pieces of detector
  // rows); a run takes consecutive slots from a slot k with k % 8 == c % 8 (each staged row
  // carries its compact index's swizzle phase), so it is staged with one bulk copy per plane.
  // Runs are laid out in compact order, each after the previous one, skipping slots up to
  // its phase.  Before that, the run fills runs of such skipped slots below the end: a piece
  // of at least two of its pixels (or its last pixel) goes to the first skipped slot of its
  // phase with room, each piece staged with a bulk copy of its own.  The slots are a
  // summation index: any assignment serves as long as the weight planes use the same one.
  std::vector<std::pair<int64_t, int32_t>> cp(pix.size());
  for (size_t u = 0; u < pix.size(); ++u) {
    const int32_t z = pix[u] / m.ny, y = pix[u] - z * m.ny;
    cp[u] = {(int64_t)row_off[z] + y - span_lo[z], pix[u]};
  }
  std::sort(cp.begin(), cp.end());
  static_assert(kMmaKStep == 32, "one 32-bit occupancy mask per K step");
  std::vector<uint32_t> occ;   // per K step, one bit per slot in use
  int top = 0;                 // slots below are laid out (used or skipped)
  int lo_step = 0;             // steps before this one are full
  for (size_t u = 0; u < cp.size();) {
    size_t v = u + 1;
    while (v < cp.size() && cp[v].first == cp[v - 1].first + 1) ++v;
    const int len = (int)(v - u);
    auto put = [&](int i0, int n, int kpos) {
      for (int i = 0; i < n; ++i) {
        const int k = kpos + i, st = k / kMmaKStep;
        if (st >= (int)occ.size()) occ.resize(st + 1, 0u);
        occ[st] |= 1u << (k % kMmaKStep);
        lut[cp[u + i0 + i].second] = k;
      }
    };
    int i = 0;
    while (i < len) {
      // the first skipped slot of the next pixel's phase with room for a piece
      const int ph = (int)(cp[u + i].first & 7), want = std::min(MI_MMA_MIN_PIECE, len - i);
      const int s_end = std::min((int)occ.size(), top / kMmaKStep + 1);
      int kpos = -1, room = 0;
      for (int st = lo_step; st < s_end && kpos < 0; ++st)
        for (int k = ph; k < kMmaKStep && st * kMmaKStep + k < top; k += 8) {
          int h = 0;
          while (k + h < kMmaKStep && st * kMmaKStep + k + h < top && !(occ[st] >> (k + h) & 1u)) ++h;
          if (h >= want) {
            kpos = st * kMmaKStep + k;
            room = h;
            break;
          }
        }
      if (kpos < 0) break;
      const int n = std::min(room, len - i);
      put(i, n, kpos);
      i += n;
    }
    if (i < len) {
      const int ph = (int)(cp[u + i].first & 7);
      const int kpos = top + ((ph - (top & 7) + 8) & 7);
      put(i, len - i, kpos);
      top = kpos + len - i;
    }
    while (lo_step < (int)occ.size() && occ[lo_step] == 0xFFFFFFFFu) ++lo_step;
    u = v;
  }
  const int n_k = std::max(1, (top + kMmaKStep - 1) / kMmaKStep);
  if (n_k * kMmaKStep > 65535) {
    for (int32_t q : pix) lut[q] = -1;
    return set_error(MI_E_RANGE, "MMA tile at row %d, column %d stages more than 65535 pixel slots", r0, e0);
  }
  std::vector<uint32_t> xrow((size_t)n_k * kMmaKStep, kMmaEmpty);
  for (auto &e : cp) xrow[lut[e.second]] = (uint32_t)e.first;
  // runs: consecutive slots of one step holding consecutive compact indices
  std::vector<uint2> runs;
  std::vector<uint32_t> rptr(n_k + 1, 0);
  for (int s = 0; s < n_k; ++s) {
    rptr[s] = (uint32_t)runs.size();
    for (int k = 0; k < kMmaKStep;) {
      const uint32_t c = xrow[s * kMmaKStep + k];
      if (c == kMmaEmpty) { ++k; continue; }
      int len = 1;
      while (k + len < kMmaKStep && xrow[s * kMmaKStep + k + len] == c + (uint32_t)len) ++len;
      runs.push_back(make_uint2(c, (uint32_t)k | ((uint32_t)len << 8)));
      k += len;
    }
  }
  rptr[n_k] = (uint32_t)runs.size();
  std::vector<uint2> terms;
  double bfac[kMmaN] = {0}, bdk[kMmaN] = {0};
  float blw[kMmaN] = {0};
  for (int i = 0; i < nr; ++i)
    for (int j = 0; j < nc; ++j) {
      const int64_t b = (int64_t)(r0 + i) * m.n_eta + e0 + j;
      const uint32_t n = (uint32_t)(i * kMmaCols + j);
      bfac[n] = fac[b];
      blw[n] = lw[b];
      const double wm = wmax[b];
      for (int64_t t = csr.row_ptr[b]; t < csr.row_ptr[b + 1]; ++t) {
        terms.push_back(make_uint2(mma_weight(csr.w[t], wm), (uint32_t)lut[csr.col[t]] | (n << 16)));
      }
    }
  // words: a bin's terms in four consecutive slots 4w .. 4w+3 of a step, one 32-bit word per
  // digit plane (the B operand's K-major rows hold those four bytes side by side), so the
  // stage builders store a word where they would store up to four bytes; words in step order
  // (by slot), then bank-ordered within each step like the terms they replace
  std::stable_sort(terms.begin(), terms.end(), [](const uint2 &x, const uint2 &y) {
    const uint32_t kx = (x.y & 0xFFFFu) / 4, ky = (y.y & 0xFFFFu) / 4;
    return kx != ky ? kx < ky : (x.y >> 16) < (y.y >> 16);
  });
  std::vector<uint4> wpl;
  std::vector<uint2> wkey;   // {word index, (k / 4) | n << 16} for bank ordering
  for (size_t t = 0; t < terms.size();) {
    const uint32_t kq = (terms[t].y & 0xFFFFu) / 4, n = terms[t].y >> 16;
    uint4 wv = make_uint4(0u, 0u, 0u, 0u);
    size_t u = t;
    for (; u < terms.size() && (terms[u].y & 0xFFFFu) / 4 == kq && (terms[u].y >> 16) == n; ++u) {
      const uint32_t b = (terms[u].y & 0xFFFFu) % 4, d = terms[u].x;
      wv.x |= (d & 0xFFu) << (8 * b);
      wv.y |= ((d >> 8) & 0xFFu) << (8 * b);
      wv.z |= ((d >> 16) & 0xFFu) << (8 * b);
      wv.w |= (d >> 24) << (8 * b);
    }
    wkey.push_back(make_uint2((uint32_t)wpl.size(), (kq * 4) | (n << 16)));
    wpl.push_back(wv);
    t = u;
  }
  std::vector<uint32_t> sp(n_k + 1, 0);
  for (const uint2 &k : wkey) ++sp[(k.y & 0xFFFFu) / kMmaKStep + 1];
  for (int s = 0; s < n_k; ++s) sp[s + 1] += sp[s];
  bank_order(wkey, sp, n_k);
  std::vector<uint4> wpl_o(wpl.size());
  std::vector<uint16_t> widx(wpl.size());
  for (size_t i = 0; i < wkey.size(); ++i) {
    wpl_o[i] = wpl[wkey[i].x];
    const uint32_t k = wkey[i].y & 0xFFFFu, n = wkey[i].y >> 16;
    widx[i] = (uint16_t)(((k % kMmaKStep) / 4) | (n << 3));
  }
  for (int32_t q : pix) lut[q] = -1;
  const MmaBlob L = mma_blob_layout(n_k, (int)runs.size(), (int)wpl_o.size());
  blob.assign(L.bytes, 0);
  MmaHdr h{nr, nc, r0, e0, n_k, (int32_t)wpl_o.size(), box_rows, (int32_t)runs.size()};
  memcpy(blob.data(), &h, sizeof(h));
  memcpy(blob.data() + kMmaBinsOff, bfac, sizeof(bfac));
  memcpy(blob.data() + kMmaBinsOff + sizeof(bfac), bdk, sizeof(bdk));
  memcpy(blob.data() + kMmaBinsOff + sizeof(bfac) + sizeof(bdk), blw, sizeof(blw));
  if (!runs.empty()) memcpy(blob.data() + L.runs, runs.data(), runs.size() * 8);
  memcpy(blob.data() + L.run_ptr, rptr.data(), rptr.size() * 4);
  memcpy(blob.data() + L.step_ptr, sp.data(), sp.size() * 4);
  if (!wpl_o.empty()) {
    memcpy(blob.data() + L.wpl, wpl_o.data(), wpl_o.size() * 16);
    memcpy(blob.data() + L.widx, widx.data(), widx.size() * 2);
  }
  *nnz_out = (int)terms.size();
  *nu_out = (int)pix.size();
  return MI_OK;
}

// ---- Direct MMA encoding (see MmadBlob): the tile's pixels covered by 8-pixel row granules
// in (row, column) order, four granules per K step; pixel (z, y) of granule g sits in slot
// 8 g + (y - y0).  Weights as in the MMA encoding (mma_weight).
static int mmad_tile_blob(const HostCSR &csr, const mi_map_desc &m, const std::vector<double> &wmax,
                          const std::vector<double> &fac, const std::vector<float> &lw, int r0, int nr, int box_rows,
                          int e0, int nc, std::vector<int32_t> &lut, std::vector<uint8_t> &blob, int *nnz_out,
                          int *nu_out) {
  std::vector<int32_t> pix;
  for (int i = 0; i < nr; ++i)
    for (int j = 0; j < nc; ++j) {
      const int64_t b = (int64_t)(r0 + i) * m.n_eta + e0 + j;
      for (int64_t t = csr.row_ptr[b]; t < csr.row_ptr[b + 1]; ++t)
        if (lut[csr.col[t]] < 0) {
          lut[csr.col[t]] = 0;
          pix.push_back(csr.col[t]);
        }
    }
  std::sort(pix.begin(), pix.end());
  // granules in ascending flat order = (row, column) order
  std::vector<uint32_t> gran;
  int64_t last = -1;
  for (int32_t q : pix) {
    const int32_t z = q / m.ny, y = q - z * m.ny, y0 = y & ~(kMmadGranPx - 1);
    const int64_t key = (int64_t)z * m.ny + y0;
    if (key != last) {
      gran.push_back((uint32_t)z | ((uint32_t)y0 << 16));
      last = key;
    }
    lut[q] = (int32_t)((gran.size() - 1) * kMmadGranPx + (y - y0));
  }
  const int n_k = std::max(1, (int)((gran.size() + kMmadGran - 1) / kMmadGran));
  if ((int64_t)n_k * kMmaKStep > 65535) {
    for (int32_t q : pix) lut[q] = -1;
    return set_error(MI_E_RANGE, "MMA tile at row %d, column %d stages more than 65535 pixel slots", r0, e0);
  }
  gran.resize((size_t)n_k * kMmadGran, kMmadEmpty);
  std::vector<uint2> terms;
  double bfac[kMmaN] = {0}, bdk[kMmaN] = {0};
  float blw[kMmaN] = {0};
  for (int i = 0; i < nr; ++i)
    for (int j = 0; j < nc; ++j) {
      const int64_t b = (int64_t)(r0 + i) * m.n_eta + e0 + j;
      const uint32_t n = (uint32_t)(i * kMmaCols + j);
      bfac[n] = fac[b];
      blw[n] = lw[b];
      const double wm = wmax[b];
      for (int64_t t = csr.row_ptr[b]; t < csr.row_ptr[b + 1]; ++t) {
        terms.push_back(make_uint2(mma_weight(csr.w[t], wm), (uint32_t)lut[csr.col[t]] | (n << 16)));
      }
    }
  std::stable_sort(terms.begin(), terms.end(),
                   [](const uint2 &x, const uint2 &y) { return (x.y & 0xFFFFu) < (y.y & 0xFFFFu); });
  std::vector<uint32_t> sp(n_k + 1, 0);
  for (const uint2 &t : terms) ++sp[(t.y & 0xFFFFu) / kMmaKStep + 1];
  for (int s2 = 0; s2 < n_k; ++s2) sp[s2 + 1] += sp[s2];
  bank_order(terms, sp, n_k);
  for (int32_t q : pix) lut[q] = -1;
  const MmadBlob L = mmad_blob_layout(n_k, (int)terms.size());
  blob.assign(L.bytes, 0);
  MmaHdr h{nr, nc, r0, e0, n_k, (int32_t)terms.size(), box_rows, 0};
  memcpy(blob.data(), &h, sizeof(h));
  memcpy(blob.data() + kMmaBinsOff, bfac, sizeof(bfac));
  memcpy(blob.data() + kMmaBinsOff + sizeof(bfac), bdk, sizeof(bdk));
  memcpy(blob.data() + kMmaBinsOff + sizeof(bfac) + sizeof(bdk), blw, sizeof(blw));
  memcpy(blob.data() + L.gran, gran.data(), gran.size() * 4);
  memcpy(blob.data() + L.step_ptr, sp.data(), sp.size() * 4);
  if (!terms.empty()) memcpy(blob.data() + L.terms, terms.data(), terms.size() * 8);
  *nnz_out = (int)terms.size();
  *nu_out = (int)pix.size();
  return MI_OK;
}

static int build_mma_tiles(const HostCSR &csr, const mi_map_desc &m, Plan *p, const std::vector<int32_t> &span_lo,
                           const std::vector<int32_t> &row_off, bool direct, int *n_slots_out,
                           std::vector<TileRef> *tiles_out, std::vector<WorkItem> *items_out,
                           std::vector<uint8_t> *blobs_out) {
  const int64_t n_bins = (int64_t)m.n_r * m.n_eta, n_pix = (int64_t)m.ny * m.nz;
  std::vector<double> wmax(n_bins, 0.0), fac(n_bins, 0.0);
  std::vector<float> lw(n_bins, 0.0f);
  for (int64_t b = 0; b < n_bins; ++b) {
    if (csr.row_ptr[b + 1] - csr.row_ptr[b] > kMmaMaxBinTerms)
      return set_error(MI_E_RANGE, "bin %lld has more than %d terms: use the run encoding", (long long)b,
                       kMmaMaxBinTerms);
    double wm = 0.0;
    for (int64_t t = csr.row_ptr[b]; t < csr.row_ptr[b + 1]; ++t) wm = std::max(wm, std::fabs(csr.w[t]));
    wmax[b] = wm;
    float sc32;
    double sc;
    bin_scale(csr, p, b, &sc32, &lw[b], &sc);
    fac[b] = wm / kMmaQMax * sc;
  }
  // items of about 12 per band, on 8-column (32-byte) cake boundaries when there are enough
  // columns, always on kMmaCols boundaries
  int item_cols = std::max(1, (m.n_eta + 11) / 12);
  item_cols = m.n_eta >= 96 ? (item_cols + 7) & ~7 : (item_cols + kMmaCols - 1) / kMmaCols * kMmaCols;
  const int n_slots = (m.n_eta + item_cols - 1) / item_cols;
  const int n_bands = (m.n_r + kMmaRows - 1) / kMmaRows;
  struct BandOut {
    std::vector<WorkItem> items;
    std::vector<std::vector<uint8_t>> blobs;
    std::vector<int> nu;
  };
  std::vector<BandOut> bands(n_bands);
  int err = MI_OK;
  const int nthr = std::min(omp_get_max_threads(), 16);
#pragma omp parallel num_threads(nthr)
  {
    std::vector<int32_t> lut(n_pix, -1);
#pragma omp for schedule(dynamic, 1)
    for (int bi = 0; bi < n_bands; ++bi) {
      BandOut &bo = bands[bi];
      const int br0 = bi * kMmaRows, bnr = std::min(kMmaRows, m.n_r - br0);
      for (int h : {kMmaRows, 6, 3, 1}) {
        bo.items.clear();
        bo.blobs.clear();
        bo.nu.clear();
        bool fits = true;
        for (int r0 = br0; r0 < br0 + bnr && fits; r0 += h) {
          const int nr = std::min(h, br0 + bnr - r0);
          for (int sl = 0; sl < n_slots && fits; ++sl) {
            WorkItem w{};
            w.tile_begin = (int)bo.blobs.size();
            w.r0 = r0;
            w.n_rows = nr;
            w.slot = sl;
            const int e_end = std::min(m.n_eta, (sl + 1) * item_cols);
            for (int e0 = sl * item_cols; e0 < e_end; e0 += kMmaCols) {
              bo.blobs.emplace_back();
              int nnz = 0, nu = 0;
              const int e =
                  direct ? mmad_tile_blob(csr, m, wmax, fac, lw, r0, nr, h, e0, std::min(kMmaCols, e_end - e0), lut,
                                          bo.blobs.back(), &nnz, &nu)
                         : mma_tile_blob(csr, m, span_lo, row_off, wmax, fac, lw, r0, nr, h, e0,
                                         std::min(kMmaCols, e_end - e0), lut, bo.blobs.back(), &nnz, &nu);
              if (e) {
#pragma omp critical
                err = e;
                fits = false;
                break;
              }
              if (bo.blobs.back().size() > kMmaBlobCap) {
                fits = false;
                break;
              }
              w.nnz += nnz;
              bo.nu.push_back(nu);
            }
            w.tile_end = (int)bo.blobs.size();
            bo.items.push_back(w);
          }
        }
        if (fits || err) break;
        if (h == 1) {
#pragma omp critical
          err = set_error(MI_E_RANGE, "an MMA tile of one row at row %d exceeds %u B; use the run encoding", br0,
                          kMmaBlobCap);
          break;
        }
      }
    }
  }
  if (err) return err;
  // arena
  std::vector<TileRef> &tiles = *tiles_out;
  std::vector<WorkItem> &items = *items_out;
  tiles.clear();
  items.clear();
  uint64_t arena = 0;
  uint32_t max_blob = 0;
  int max_u = 0;
  int64_t staged = 0;
  for (BandOut &bo : bands)
    for (WorkItem w : bo.items) {
      const int tb = (int)tiles.size();
      for (int k = w.tile_begin; k < w.tile_end; ++k) {
        const uint32_t bytes = (uint32_t)bo.blobs[k].size();
        tiles.push_back({arena, bytes, 0});
        arena += bytes;
        max_blob = std::max(max_blob, bytes);
        max_u = std::max(max_u, bo.nu[k]);
        staged += bo.nu[k];
      }
      w.tile_end = (int)tiles.size();
      w.tile_begin = tb;
      items.push_back(w);
    }
  blobs_out->assign(arena, 0);
  size_t ti = 0;
  for (BandOut &bo : bands)
    for (WorkItem w : bo.items)
      for (int k = w.tile_begin; k < w.tile_end; ++k, ++ti) {
        memcpy(blobs_out->data() + tiles[ti].off, bo.blobs[k].data(), bo.blobs[k].size());
        std::vector<uint8_t>().swap(bo.blobs[k]);
      }
  p->n_tiles = (int)tiles.size();
  p->max_blob = max_blob;
  p->max_u = max_u;
  p->max_nb = kMmaN;
  p->staged_pixels = staged;
  p->n_slots = n_slots;
  p->lim.rows = kMmaRows;
  p->lim.max_u = max_u;
  p->lim.item_cols = item_cols;
  *n_slots_out = n_slots;
  return MI_OK;
}

// Caps the OpenMP threads of the calling thread's parallel regions for a scope (the
// host_threads plan option); the previous setting is restored on exit.
struct HostThreads {
  int prev = 0;
  explicit HostThreads(int n) {
    if (n > 0) {
      prev = omp_get_max_threads();
      omp_set_num_threads(n);
    }
  }
  ~HostThreads() {
    if (prev > 0) omp_set_num_threads(prev);
  }
};

// Build a plan.  `pre` (optional) is the weight list already built for the whole detector
// (panel plans: the panels' lists merged over the virtual detector); `m` then describes the
// virtual detector and carries no records, and the plain path is not built.
static int build_plan(const mi_map_desc &m, const mi_plan_opts &o, Plan *p, HostCSR *pre = nullptr) {
  p->mode = o.mode;
  p->normalize = o.normalize ? 1 : 0;
  p->semantics = o.semantics;
  p->n_r = m.n_r;
  p->n_eta = m.n_eta;
  p->ny = m.ny;
  p->nz = m.nz;
  p->bc_y = m.bc_y;
  p->bc_z = m.bc_z;
  p->n_bins = (int64_t)m.n_r * m.n_eta;
  p->n_records = m.n_records;
  const int64_t n_pix = (int64_t)m.ny * m.nz;

  HostCSR csr;
  int rc = MI_OK;
  if (pre) csr = std::move(*pre);
  else if ((rc = build_host_csr(m, o.mode, o.semantics, &csr))) return rc;
  p->variance = o.variance ? 1 : 0;
  if (p->variance)
    for (double &x : csr.w) x *= x;   // _square_csr (kernels.py:378-400) of the coalesced weights
  if (p->panels.empty()) p->panels.push_back({m.ny, m.nz, 0, 0, 0});
  p->nnz = (int64_t)csr.col.size();
  p->oob = csr.oob;

  // ---- encoding and limits
  const int enc = (o.encoding == MI_ENC_CSR || o.encoding == MI_ENC_MMA || o.encoding == MI_ENC_MMAD) ? o.encoding
                                                                                                    : MI_ENC_RUNS;
  if (o.encoding < 0 || o.encoding > 4) return set_error(MI_E_ARG, "unknown encoding %d", o.encoding);
  if (enc == MI_ENC_MMAD && (m.ny > 65535 || m.nz > 65535))
    return set_error(MI_E_UNSUPPORTED, "the direct MMA encoding takes detectors up to 65535 x 65535 pixels");
  p->encoding = enc;
  int fpl = o.frames_per_lane > 0 ? o.frames_per_lane : 1;
  if (fpl != 1 && fpl != 2 && fpl != 4) return set_error(MI_E_ARG, "frames_per_lane must be 1, 2 or 4");
  p->frames_per_lane = fpl;
  TileLimits L;
  L.rows = o.tile_rows > 0 ? o.tile_rows : 16;
  if (L.rows > (enc == MI_ENC_RUNS ? 32 : 64))
    return set_error(MI_E_RANGE, "tile_rows %d > %d", L.rows, enc == MI_ENC_RUNS ? 32 : 64);
  L.max_u = o.tile_pixels > 0 ? o.tile_pixels
                              : (enc == MI_ENC_RUNS ? 1024 : (fpl == 1 ? 640 : (fpl == 2 ? 320 : 160)));
  if (L.max_u > 65535) return set_error(MI_E_RANGE, "tile_pixels %d > 65535", L.max_u);
  L.max_nb = 256;
  L.max_nnz = enc == MI_ENC_RUNS ? 12288 : 4096;
  L.max_cols = enc == MI_ENC_RUNS ? kRunWarps : 1 << 30;
  // about 12 items per band; item boundaries on 8-column (32-byte) boundaries of the cake
  // rows when there are enough columns, so no cake sector is written by two items
  L.item_cols = std::max(1, (m.n_eta + 11) / 12);
  if (m.n_eta >= 96) L.item_cols = (L.item_cols + 7) & ~7;
  int G = 0, RL = 0;
  if (enc == MI_ENC_RUNS) {
    G = L.rows <= 8 ? 8 : (L.rows <= 16 ? 16 : 32);
    RL = o.run_len > 0 ? o.run_len : choose_run_len(csr, m, L.rows, G);
    if (!(RL == 2 || RL == 4 || RL == 8) || RL > G / 2 || (G == 32 && RL == 2) || (G == 16 && RL == 2))
      return set_error(MI_E_ARG, "run_len %d not supported with %d rows per strip", RL, G);
  }
  p->run_g = G;
  p->run_l = RL;
  int dev_smem = 0;
  MI_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, p->device));
  if (enc == MI_ENC_RUNS) {
    // budget for kRunCtasPerSm resident CTAs per SM (1 KB per CTA is reserved by the runtime)
    int sm_smem = 0;
    MI_CUDA(cudaDeviceGetAttribute(&sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, p->device));
    dev_smem = std::min(dev_smem, sm_smem / kRunCtasPerSm - 1024);
  }

  // distinct referenced pixels, and their row spans for pixel-major staging
  std::vector<int32_t> span_lo(m.nz, 0), row_off(m.nz, 0);
  std::vector<XcChunk> xchunks;
  int64_t n_xc = 0;
  {
    std::vector<uint8_t> seen(n_pix, 0);
    int64_t n = 0;
    int64_t cmin = n_pix, cmax = -1;
    for (int32_t c : csr.col) {
      if (!seen[c]) { seen[c] = 1; ++n; }
      cmin = std::min<int64_t>(cmin, c);
      cmax = std::max<int64_t>(cmax, c);
    }
    p->ref_pixels = n;
    p->ref_row_lo = cmax >= 0 ? (int)(cmin / m.ny) : 0;
    p->ref_row_hi = cmax >= 0 ? (int)(cmax / m.ny) + 1 : 0;
    if (p->panels.size() == 1) {
      for (int z0 = p->ref_row_lo; z0 < p->ref_row_hi; z0 += kUploadRows) {
        const int z1 = std::min(z0 + kUploadRows, p->ref_row_hi);
        int lo = m.ny, hi = 0;
        for (int z = z0; z < z1; ++z) {
          const uint8_t *row = seen.data() + (int64_t)z * m.ny;
          int a = 0, b = m.ny;
          while (a < m.ny && !row[a]) ++a;
          while (b > a && !row[b - 1]) --b;
          if (b > a) { lo = std::min(lo, a); hi = std::max(hi, b); }
        }
        if (hi > lo) p->upload_groups.push_back(make_int4(z0, z1, lo & ~7, std::min(m.ny, (hi + 7) & ~7)));
      }
    }
    if ((p->encoding == MI_ENC_RUNS && runs_frames_per_group(2, p->run_g) == kXcFrames) ||
        p->encoding == MI_ENC_MMA) {
      size_t pi = 0;
      for (int z = 0; z < m.nz; ++z) {
        // chunks are made row by row, so each panel's chunks are one contiguous range
        while (pi + 1 < p->panels.size() && z >= p->panels[pi + 1].z_off) ++pi;
        if (z == p->panels[pi].z_off) p->panels[pi].chunk_begin = (int)xchunks.size();
        const uint8_t *row = seen.data() + (int64_t)z * m.ny;
        int lo = 0, hi = m.ny;
        while (lo < m.ny && !row[lo]) ++lo;
        while (hi > lo && !row[hi - 1]) --hi;
        lo &= ~7;
        // the panel's own width bounds the span: the transpose reads the panel's frame rows
        if (hi > lo) hi = std::min(p->panels[pi].ny, (hi + 7) & ~7);
        else hi = lo;
        span_lo[z] = lo;
        row_off[z] = (int32_t)n_xc;
        for (int y = lo; y < hi; y += kXcChunk)
          xchunks.push_back({z, y, std::min(kXcChunk, hi - y), (int32_t)(n_xc + (y - lo))});
        n_xc += hi - lo;
        p->panels[pi].chunk_end = (int)xchunks.size();
      }
    }
  }
  int n_slots = 0, n_items = 0;
  std::vector<TileRef> tiles;
  std::vector<WorkItem> items;
  std::vector<uint8_t> blobs;
  if (enc == MI_ENC_MMA || enc == MI_ENC_MMAD) {
    if ((rc = build_mma_tiles(csr, m, p, span_lo, row_off, enc == MI_ENC_MMAD, &n_slots, &tiles, &items, &blobs)))
      return rc;
    n_items = (int)items.size();
  } else {
    // ---- items and tiles; shrink the tile limits until the kernel's shared memory fits
    const int n_bands = (m.n_r + L.rows - 1) / L.rows;
    n_slots = (m.n_eta + L.item_cols - 1) / L.item_cols;
    p->n_slots = n_slots;
    n_items = n_bands * n_slots;
    std::vector<std::vector<HostTile>> item_tiles(n_items);
    std::vector<std::vector<std::vector<uint8_t>>> item_blobs(n_items);
    for (int attempt = 0;; ++attempt) {
      int err = MI_OK;
      int nthr = std::min(omp_get_max_threads(), 16);
  #pragma omp parallel num_threads(nthr)
      {
        std::vector<int32_t> stamp(n_pix, 0), lut(n_pix, -1);
        int32_t sid = 0;
  #pragma omp for schedule(dynamic, 1)
        for (int it = 0; it < n_items; ++it) {
          item_tiles[it].clear();
          item_blobs[it].clear();
          int band = it / n_slots, slot = it % n_slots;
          int r0 = band * L.rows, nr = std::min(L.rows, m.n_r - r0);
          int e0 = slot * L.item_cols, e1 = std::min(m.n_eta, e0 + L.item_cols);
          int e = tile_item(Builder(csr, m.n_r, m.n_eta, n_pix, L), r0, nr, e0, e1, stamp, sid,
                            item_tiles[it]);
          if (e) {
  #pragma omp critical
            err = e;
            continue;
          }
          for (const HostTile &t : item_tiles[it]) {
            item_blobs[it].emplace_back();
            if (enc == MI_ENC_RUNS)
              runs_blob(csr, m, p, t, t.r0 - r0, G, RL, lut, item_blobs[it].back());
            else
              csr_blob(csr, m, p, t, t.r0 - r0, lut, item_blobs[it].back());
          }
        }
      }
      if (err) return err;
      uint32_t mb = 0;
      int mu = 1, mnb = 1;
      for (int it = 0; it < n_items; ++it)
        for (size_t k = 0; k < item_tiles[it].size(); ++k) {
          mb = std::max(mb, (uint32_t)item_blobs[it][k].size());
          mu = std::max(mu, item_tiles[it][k].n_u);
          mnb = std::max(mnb, item_tiles[it][k].n_rows * item_tiles[it][k].n_cols);
        }
      const uint32_t cap = (mb + 15u) & ~15u;
      const uint32_t need = enc == MI_ENC_RUNS
                                ? runs_smem_layout(cap, mu, mnb | 1, L.rows, G, runs_frames_per_group(2, G), nullptr,
                                                   nullptr, nullptr, nullptr, nullptr)
                                : cake_smem_layout(fpl, cap, mu, mnb | 1, L.rows, nullptr, nullptr, nullptr, nullptr);
      if (need + 1024u <= (uint32_t)dev_smem) break;
      if (attempt >= 12 || L.max_u <= 32)
        return set_error(MI_E_RANGE, "tiles need %u B of shared memory (device allows %d); lower tile_rows",
                         need, dev_smem);
      L.max_u = std::max(32, L.max_u * 4 / 5);
      L.max_nnz = std::max(256, L.max_nnz * 4 / 5);
      L.max_nb = std::max(16, L.max_nb * 4 / 5);
    }
    p->lim = L;

    // ---- blob arena
    items.assign(n_items, WorkItem{});
    uint64_t arena = 0;
    uint32_t max_blob = 0;
    int max_u = 0, max_nb = 0;
    int64_t staged = 0;
    for (int it = 0; it < n_items; ++it) {
      int band = it / n_slots, slot = it % n_slots;
      WorkItem &w = items[it];
      w.tile_begin = (int)tiles.size();
      w.r0 = band * L.rows;
      w.n_rows = std::min(L.rows, m.n_r - w.r0);
      w.slot = slot;
      w.nnz = 0;
      for (size_t k = 0; k < item_tiles[it].size(); ++k) {
        const HostTile &t = item_tiles[it][k];
        const uint32_t bytes = (uint32_t)item_blobs[it][k].size();
        tiles.push_back({arena, bytes, 0});
        arena += bytes;
        max_blob = std::max(max_blob, bytes);
        max_u = std::max(max_u, t.n_u);
        max_nb = std::max(max_nb, t.n_rows * t.n_cols);
        staged += t.n_u;
        w.nnz += t.nnz;
      }
      w.tile_end = (int)tiles.size();
    }
    p->n_tiles = (int)tiles.size();
    p->max_blob = max_blob;
    p->max_u = max_u;
    p->max_nb = max_nb;
    p->staged_pixels = staged;
    blobs.assign(arena, 0);
    for (int it = 0, ti = 0; it < n_items; ++it)
      for (size_t k = 0; k < item_blobs[it].size(); ++k, ++ti) {
        memcpy(blobs.data() + tiles[ti].off, item_blobs[it][k].data(), item_blobs[it][k].size());
        std::vector<uint8_t>().swap(item_blobs[it][k]);
      }
  }

  // heaviest-first launch order
  std::vector<int> order(n_items);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return items[a].nnz > items[b].nnz; });
  std::vector<WorkItem> items_sorted(n_items);
  for (int i = 0; i < n_items; ++i) items_sorted[i] = items[order[i]];
  p->n_items = n_items;

  // lineout denominators (variance plans: squared, kernels.py:625-640)
  std::vector<double> den(m.n_r, 0.0), cnt(m.n_r, 0.0);
  for (int r = 0; r < m.n_r; ++r) {
    for (int e = 0; e < m.n_eta; ++e) {
      double a = csr.area_in[(int64_t)r * m.n_eta + e];
      if (a > kAreaThreshold) { den[r] += a; cnt[r] += 1.0; }
    }
    if (p->variance) {
      den[r] = den[r] > kAreaThreshold ? den[r] * den[r] : 0.0;
      cnt[r] *= cnt[r];
    }
  }
  p->area_gs = csr.area_gs;

  size_t acct = 0;
  MI_CUDA(cudaSetDevice(p->device));
  if ((rc = upload(&p->d_blobs, blobs.data(), blobs.size(), &acct))) return rc;
  p->blob_bytes = blobs.size();
  if ((rc = upload(&p->d_tiles, tiles.data(), tiles.size(), &acct))) return rc;
  if ((rc = upload(&p->d_items, items_sorted.data(), items_sorted.size(), &acct))) return rc;
  if ((rc = upload(&p->d_den_aw, den.data(), den.size(), &acct))) return rc;
  if ((rc = upload(&p->d_cnt, cnt.data(), cnt.size(), &acct))) return rc;

  {
    size_t bytes = (size_t)kMaxFramesPerLaunch * m.n_r * n_slots * 2 * sizeof(double);
    MI_CUDA(cudaMalloc((void **)&p->d_partial, bytes));
    acct += bytes;
  }
  MI_CUDA(cudaMalloc((void **)&p->d_dark, n_pix * sizeof(float)));
  MI_CUDA(cudaMemset(p->d_dark, 0, n_pix * sizeof(float)));
  acct += n_pix * sizeof(float);
  MI_CUDA(cudaMalloc((void **)&p->d_err, sizeof(int)));
  MI_CUDA(cudaMemset(p->d_err, 0, sizeof(int)));
  MI_CUDA(cudaMalloc((void **)&p->d_ctr, sizeof(int)));
  MI_CUDA(cudaDeviceGetAttribute(&p->n_sms, cudaDevAttrMultiProcessorCount, p->device));
  if (n_xc > 0) {
    if ((rc = upload(&p->d_span_lo, span_lo.data(), span_lo.size(), &acct))) return rc;
    if ((rc = upload(&p->d_row_off, row_off.data(), row_off.size(), &acct))) return rc;
    if ((rc = upload(&p->d_xchunks, xchunks.data(), xchunks.size(), &acct))) return rc;
    if (enc == MI_ENC_MMA) {
      std::vector<int32_t> xpix(n_xc);
      for (int z = 0; z < m.nz; ++z) {
        const int64_t c1 = z + 1 < m.nz ? row_off[z + 1] : n_xc;
        for (int64_t c = row_off[z]; c < c1; ++c) xpix[c] = (int32_t)((int64_t)z * m.ny + span_lo[z] + (c - row_off[z]));
      }
      if ((rc = upload(&p->d_xc_pix, xpix.data(), xpix.size(), &acct))) return rc;
    }
    const size_t bytes = (size_t)n_xc * kXcFrames * kXcGroups * sizeof(uint16_t);
    MI_CUDA(cudaMalloc((void **)&p->d_xc, bytes));
    acct += bytes;
    p->n_xc = n_xc;
    p->n_xchunks = (int)xchunks.size();
  }

  if ((rc = upload(&p->d_area_in, csr.area_in.data(), csr.area_in.size(), &acct))) return rc;
  // ---- plain path: reference SoA layout (PrecomputeOffsets_kernel, …Stream.cu:901-924)
  if (!pre) {
    const int64_t nrec = m.n_records;
    std::vector<int32_t> off(nrec);
    std::vector<float> w(nrec), aw(nrec), dr(nrec), py(nrec), pz(nrec);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nrec; ++i) {
      const mi_map_record &r = m.records[i];
      long long zz = (long long)r.z;
      float s = (float)(zz * (long long)m.ny) + r.y;
      long long o2 = (long long)s;
      const int64_t ty = (int64_t)r.y, tz = (int64_t)r.z;
      const bool inb = ty >= 0 && ty < m.ny && tz >= 0 && tz < m.nz;
      if (p->semantics == MI_SEM_PY) o2 = inb ? (long long)(tz * m.ny + ty) : -1;
      else if (o2 < 0 || o2 >= (long long)m.ny * m.nz) o2 = -1;
      off[i] = (int32_t)o2;
      w[i] = (float)r.frac;
      aw[i] = r.areaWeight;
      dr[i] = r.deltaR;
      py[i] = r.y;
      pz[i] = r.z;
    }
    std::vector<int32_t> sorted(p->n_bins);
    std::iota(sorted.begin(), sorted.end(), 0);
    std::stable_sort(sorted.begin(), sorted.end(),
                     [&](int32_t a, int32_t b) { return m.nmap[2 * a] > m.nmap[2 * b]; });
    std::vector<double> area_all(p->n_bins, 0.0);
    for (int64_t b = 0; b < p->n_bins; ++b) {
      double s = 0;
      for (int32_t k = 0; k < m.nmap[2 * b]; ++k) s += m.records[(int64_t)m.nmap[2 * b + 1] + k].areaWeight;
      area_all[b] = s;
    }
    if ((rc = upload(&p->d_nmap, m.nmap, (size_t)(2 * p->n_bins), &acct))) return rc;
    if ((rc = upload(&p->d_sorted, sorted.data(), sorted.size(), &acct))) return rc;
    if ((rc = upload(&p->d_off, off.data(), off.size(), &acct))) return rc;
    if ((rc = upload(&p->d_w, w.data(), w.size(), &acct))) return rc;
    if ((rc = upload(&p->d_aw, aw.data(), aw.size(), &acct))) return rc;
    if ((rc = upload(&p->d_dr, dr.data(), dr.size(), &acct))) return rc;
    if ((rc = upload(&p->d_py, py.data(), py.size(), &acct))) return rc;
    if ((rc = upload(&p->d_pz, pz.data(), pz.size(), &acct))) return rc;
    if ((rc = upload(&p->d_area_all, area_all.data(), area_all.size(), &acct))) return rc;
    MI_CUDA(cudaMalloc((void **)&p->d_plain_img, n_pix * sizeof(float)));
    acct += n_pix * sizeof(float);
  }
  p->device_bytes = acct;
  return MI_OK;
}

}  // namespace mi

using namespace mi;

// ---------------------------------------------------------------------------
// Fused multi-shift maps (build_fused_geometry, packages/midas_integrate/midas_integrate/
// fused_csr.py:139-296): N maps whose R edges are shifted by k / N of a bin, each
// area-normalised (1 / area_in where it exceeds the area threshold, else 0: D_k), moved
// onto shift 0's R axis by linear interpolation in R (P_k, fused_csr.py:63-104: at most two
// source rows per target row, identity in eta) and averaged:
//   M = 1/N sum_k P_k D_k M_k,  every bin's area 1 (the normalisation is in the weights).
// ---------------------------------------------------------------------------
namespace mi {
static void interp_row(const double *src, int n_src, double r, int *j, double *wl, double *wh) {
  if (r <= src[0]) {
    *j = 0; *wl = 1.0; *wh = 0.0;
  } else if (r >= src[n_src - 1]) {
    *j = n_src - 2; *wl = 0.0; *wh = 1.0;
  } else {
    int jj = (int)(std::upper_bound(src, src + n_src, r) - src) - 1;
    jj = std::max(0, std::min(jj, n_src - 2));
    const double den = src[jj + 1] - src[jj];
    const double t = den > 0.0 ? (r - src[jj]) / den : 0.0;
    *j = jj; *wl = 1.0 - t; *wh = t;
  }
}

int build_fused_csr(const mi_map_desc *maps, int n_shifts, const double *const *r_axes, int mode, HostCSR *out) {
  if (!maps || !r_axes || n_shifts < 1) return set_error(MI_E_ARG, "fused map: null argument or no shifts");
  if (mode != MI_MODE_BILINEAR && mode != MI_MODE_GRADIENT)
    return set_error(MI_E_ARG, "fused map: mode must be bilinear or gradient");
  const mi_map_desc &m0 = maps[0];
  for (int k = 0; k < n_shifts; ++k) {
    const mi_map_desc &m = maps[k];
    if (m.n_eta != m0.n_eta || m.ny != m0.ny || m.nz != m0.nz)
      return set_error(MI_E_ARG, "fused map: shift %d has another eta binning or detector shape", k);
    if (m.n_r < 2 || m.n_eta <= 0 || m.ny < 2 || m.nz < 2 || !m.nmap || (m.n_records > 0 && !m.records) ||
        !r_axes[k])
      return set_error(MI_E_ARG, "fused map: shift %d has a bad shape or null arrays (two R bins at least)", k);
  }
  const int n_eta = m0.n_eta, n_r0 = m0.n_r;
  const int64_t n_bins = (int64_t)n_r0 * n_eta;
  std::vector<HostCSR> part(n_shifts);
  std::vector<std::vector<double>> inv_a(n_shifts);
  std::vector<int> jlo((size_t)n_shifts * n_r0);
  std::vector<double> wlo((size_t)n_shifts * n_r0), whi((size_t)n_shifts * n_r0);
  int64_t oob = 0;
  for (int k = 0; k < n_shifts; ++k) {
    int rc = build_host_csr(maps[k], mode, MI_SEM_PY, &part[k]);
    if (rc) return rc;
    oob += part[k].oob;
    inv_a[k].resize(part[k].area_in.size());
    for (size_t b = 0; b < inv_a[k].size(); ++b) {
      const double a = part[k].area_in[b];
      inv_a[k][b] = a > kAreaThreshold ? 1.0 / std::max(a, kAreaThreshold) : 0.0;
    }
    for (int i = 0; i < n_r0; ++i)
      interp_row(r_axes[k], maps[k].n_r, r_axes[0][i], &jlo[(size_t)k * n_r0 + i], &wlo[(size_t)k * n_r0 + i],
                 &whi[(size_t)k * n_r0 + i]);
  }
  const double inv_n = 1.0 / n_shifts;
  auto gather = [&](int64_t b, std::vector<Term> &t) {
    t.clear();
    const int i = (int)(b / n_eta), e = (int)(b % n_eta);
    for (int k = 0; k < n_shifts; ++k) {
      const size_t q = (size_t)k * n_r0 + i;
      const int js[2] = {jlo[q], jlo[q] + 1};
      const double ws[2] = {wlo[q], whi[q]};
      for (int h = 0; h < 2; ++h) {
        if (ws[h] == 0.0) continue;
        const int64_t bs = (int64_t)js[h] * n_eta + e;
        const double f = ws[h] * inv_a[k][bs] * inv_n;
        if (f == 0.0) continue;
        for (int64_t x = part[k].row_ptr[bs]; x < part[k].row_ptr[bs + 1]; ++x)
          t.push_back({part[k].col[x], part[k].w[x] * f});
      }
    }
    std::stable_sort(t.begin(), t.end(), [](const Term &a, const Term &c) { return a.col < c.col; });
    size_t o = 0;
    for (size_t x = 0; x < t.size();) {
      size_t y = x;
      double sum = 0.0;
      while (y < t.size() && t[y].col == t[x].col) sum += t[y++].w;
      if (sum != 0.0) t[o++] = {t[x].col, sum};
      x = y;
    }
    t.resize(o);
  };
  std::vector<int64_t> counts(n_bins + 1, 0);
#pragma omp parallel
  {
    std::vector<Term> t;
#pragma omp for schedule(dynamic, 256)
    for (int64_t b = 0; b < n_bins; ++b) {
      gather(b, t);
      counts[b + 1] = (int64_t)t.size();
    }
  }
  out->row_ptr.assign(n_bins + 1, 0);
  for (int64_t b = 0; b < n_bins; ++b) out->row_ptr[b + 1] = out->row_ptr[b] + counts[b + 1];
  out->col.resize(out->row_ptr[n_bins]);
  out->w.resize(out->row_ptr[n_bins]);
#pragma omp parallel
  {
    std::vector<Term> t;
#pragma omp for schedule(dynamic, 256)
    for (int64_t b = 0; b < n_bins; ++b) {
      gather(b, t);
      int64_t o = out->row_ptr[b];
      for (const Term &x : t) {
        out->col[o] = x.col;
        out->w[o++] = x.w;
      }
    }
  }
  out->area_in.assign(n_bins, 1.0);
  out->area_norm.assign(n_bins, 1.0);
  out->area_gs.assign(n_bins, 1.0);
  out->oob = oob;
  return MI_OK;
}
}  // namespace mi

struct mi_plan : public mi::Plan {};

extern "C" {

const char *mi_last_error(void) { return mi::g_err; }
const char *mi_version(void) { return "midas_b200 0.1.0 (sm_100a)"; }

int mi_plan_create(const mi_map_desc *map, const mi_plan_opts *opts, int device, mi_plan **out) {
  if (!map || !out) return set_error(MI_E_ARG, "mi_plan_create: null argument");
  *out = nullptr;
  if (map->n_r <= 0 || map->n_eta <= 0 || map->ny < 2 || map->nz < 2)
    return set_error(MI_E_ARG, "mi_plan_create: bad shape n_r=%d n_eta=%d ny=%d nz=%d", map->n_r,
                     map->n_eta, map->ny, map->nz);
  if (!map->nmap || (map->n_records > 0 && !map->records))
    return set_error(MI_E_ARG, "mi_plan_create: null map arrays");
  if ((int64_t)map->ny * map->nz > (int64_t)INT32_MAX)
    return set_error(MI_E_RANGE, "mi_plan_create: detector larger than 2^31 pixels");
  mi_plan_opts o{};
  if (opts) o = *opts;
  else { o.mode = MI_MODE_FLOOR; o.normalize = 1; o.semantics = MI_SEM_PY; }
  if (o.mode < 0 || o.mode > 2) return set_error(MI_E_ARG, "mi_plan_create: unknown mode %d", o.mode);
  if (o.semantics < 0 || o.semantics > 3)
    return set_error(MI_E_ARG, "mi_plan_create: unknown semantics %d", o.semantics);
  if ((o.semantics == MI_SEM_IC || o.semantics == MI_SEM_OMP) && o.mode == MI_MODE_FLOOR)
    return set_error(MI_E_ARG, "mi_plan_create: IntegrationCore semantics has no floor mode "
                               "(integration_apply_map always interpolates)");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_error(MI_E_CUDA, "mi_plan_create: no CUDA device available");
  if (device < 0 || device >= ndev) return set_error(MI_E_ARG, "mi_plan_create: bad device %d", device);
  mi_plan *p = new (std::nothrow) mi_plan();
  if (!p) return set_error(MI_E_OOM, "mi_plan_create: host allocation failed");
  p->device = device;
  int prev = 0;
  cudaGetDevice(&prev);
  HostThreads ht(o.host_threads);
  int rc = build_plan(*map, o, p);
  cudaSetDevice(prev);
  if (rc) {
    free_plan_mem(p);
    delete p;
    return rc;
  }
  *out = p;
  return MI_OK;
}

int mi_plan_create_panels(const mi_map_desc *maps, int n_panels, const mi_plan_opts *opts, int device,
                          mi_plan **out) {
  if (!maps || !out || n_panels < 1) return set_error(MI_E_ARG, "mi_plan_create_panels: null argument or no panels");
  *out = nullptr;
  int ny_v = 0;
  int64_t nz_v = 0, n_rec = 0;
  for (int i = 0; i < n_panels; ++i) {
    const mi_map_desc &m = maps[i];
    if (m.n_r != maps[0].n_r || m.n_eta != maps[0].n_eta)
      return set_error(MI_E_ARG, "mi_plan_create_panels: panel %d has %d x %d bins, panel 0 %d x %d", i, m.n_r,
                       m.n_eta, maps[0].n_r, maps[0].n_eta);
    if (m.n_r <= 0 || m.n_eta <= 0 || m.ny < 2 || m.nz < 2)
      return set_error(MI_E_ARG, "mi_plan_create_panels: panel %d has a bad shape", i);
    if (!m.nmap || (m.n_records > 0 && !m.records))
      return set_error(MI_E_ARG, "mi_plan_create_panels: panel %d has null map arrays", i);
    ny_v = std::max(ny_v, m.ny);
    nz_v += m.nz;
    n_rec += m.n_records;
  }
  if ((int64_t)ny_v * nz_v > (int64_t)INT32_MAX)
    return set_error(MI_E_RANGE, "mi_plan_create_panels: panels hold more than 2^31 pixels");
  mi_plan_opts o{};
  if (opts) o = *opts;
  else { o.mode = MI_MODE_FLOOR; o.normalize = 1; o.semantics = MI_SEM_PY; }
  HostThreads ht(o.host_threads);
  if (o.mode < 0 || o.mode > 2 || o.semantics < 0 || o.semantics > 2 ||
      (o.semantics == MI_SEM_IC && o.mode == MI_MODE_FLOOR))
    return set_error(MI_E_ARG, "mi_plan_create_panels: bad mode %d / semantics %d", o.mode, o.semantics);
  if (o.encoding == MI_ENC_CSR || o.encoding == MI_ENC_MMAD || (o.encoding != MI_ENC_MMA && o.tile_rows > 16))
    return set_error(MI_E_UNSUPPORTED,
                     "mi_plan_create_panels: panel plans use the run encoding with tile_rows <= 16 or the MMA encoding");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_error(MI_E_CUDA, "mi_plan_create_panels: no CUDA device available");
  if (device < 0 || device >= ndev) return set_error(MI_E_ARG, "mi_plan_create_panels: bad device %d", device);
  // each panel's weights with its own geometry, then merged over the virtual detector:
  // panel i's pixel (z, y) is virtual pixel (z_off_i + z) * ny_v + y; a bin's terms are
  // panel 0's, then panel 1's, ... (ascending virtual index); areas add up
  const int64_t n_bins = (int64_t)maps[0].n_r * maps[0].n_eta;
  std::vector<HostCSR> part(n_panels);
  std::vector<Plan::Panel> geo(n_panels);
  int z_off = 0;
  for (int i = 0; i < n_panels; ++i) {
    int rc = build_host_csr(maps[i], o.mode, o.semantics, &part[i]);
    if (rc) return rc;
    geo[i] = {maps[i].ny, maps[i].nz, z_off, 0, 0};
    z_off += maps[i].nz;
  }
  HostCSR csr;
  csr.row_ptr.assign(n_bins + 1, 0);
  csr.area_in.assign(n_bins, 0.0);
  csr.area_norm.assign(n_bins, 0.0);
  csr.area_gs.assign(n_bins, 0.0);
  for (int64_t b = 0; b < n_bins; ++b) {
    int64_t c = 0;
    for (int i = 0; i < n_panels; ++i) {
      c += part[i].row_ptr[b + 1] - part[i].row_ptr[b];
      csr.area_in[b] += part[i].area_in[b];
      csr.area_norm[b] += part[i].area_norm[b];
      csr.area_gs[b] += part[i].area_gs[b];
    }
    csr.row_ptr[b + 1] = csr.row_ptr[b] + c;
  }
  csr.col.resize(csr.row_ptr[n_bins]);
  csr.w.resize(csr.row_ptr[n_bins]);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t b = 0; b < n_bins; ++b) {
    int64_t o2 = csr.row_ptr[b];
    for (int i = 0; i < n_panels; ++i)
      for (int64_t j = part[i].row_ptr[b]; j < part[i].row_ptr[b + 1]; ++j, ++o2) {
        const int32_t c = part[i].col[j];
        const int32_t z = c / geo[i].ny, y = c - z * geo[i].ny;
        csr.col[o2] = (int32_t)((int64_t)(geo[i].z_off + z) * ny_v + y);
        csr.w[o2] = part[i].w[j];
      }
  }
  for (int i = 0; i < n_panels; ++i) csr.oob += part[i].oob;
  std::vector<HostCSR>().swap(part);
  mi_map_desc vm{};
  vm.records = nullptr;
  vm.n_records = n_rec;
  vm.nmap = nullptr;
  vm.n_r = maps[0].n_r;
  vm.n_eta = maps[0].n_eta;
  vm.ny = ny_v;
  vm.nz = (int32_t)nz_v;
  mi_plan *p = new (std::nothrow) mi_plan();
  if (!p) return set_error(MI_E_OOM, "mi_plan_create_panels: host allocation failed");
  p->device = device;
  p->panels = geo;
  int prev = 0;
  cudaGetDevice(&prev);
  int rc = build_plan(vm, o, p, &csr);
  cudaSetDevice(prev);
  if (rc == MI_OK && p->n_xc == 0)
    rc = set_error(MI_E_UNSUPPORTED, "mi_plan_create_panels: the plan has no pixel-major staging");
  if (rc) {
    free_plan_mem(p);
    delete p;
    return rc;
  }
  *out = p;
  return MI_OK;
}

int mi_fused_csr(const mi_map_desc *maps, int n_shifts, const double *const *r_axes, int mode, int64_t *row_ptr,
                 int32_t *col, double *w, int64_t capacity, int64_t *nnz) {
  if (!nnz) return set_error(MI_E_ARG, "mi_fused_csr: null nnz");
  HostCSR csr;
  int rc = build_fused_csr(maps, n_shifts, r_axes, mode, &csr);
  if (rc) return rc;
  const int64_t n = (int64_t)csr.col.size();
  *nnz = n;
  if (row_ptr) memcpy(row_ptr, csr.row_ptr.data(), csr.row_ptr.size() * sizeof(int64_t));
  if (col || w) {
    if (!col || !w) return set_error(MI_E_ARG, "mi_fused_csr: col and w go together");
    if (capacity < n) return set_error(MI_E_RANGE, "mi_fused_csr: %lld terms, capacity %lld", (long long)n,
                                       (long long)capacity);
    if (n) {
      memcpy(col, csr.col.data(), n * sizeof(int32_t));
      memcpy(w, csr.w.data(), n * sizeof(double));
    }
  }
  return MI_OK;
}

int mi_plan_create_fused(const mi_map_desc *maps, int n_shifts, const double *const *r_axes, const mi_plan_opts *opts,
                         int device, mi_plan **out) {
  if (!out) return set_error(MI_E_ARG, "mi_plan_create_fused: null argument");
  *out = nullptr;
  mi_plan_opts o{};
  if (opts) o = *opts;
  else { o.mode = MI_MODE_GRADIENT; o.normalize = 1; o.semantics = MI_SEM_PY; }
  if (o.semantics != MI_SEM_PY || o.variance)
    return set_error(MI_E_UNSUPPORTED, "mi_plan_create_fused: fused maps are midas_integrate CSR geometries "
                                       "(py semantics, no variance plan)");
  if (!maps || n_shifts < 1) return set_error(MI_E_ARG, "mi_plan_create_fused: null argument or no shifts");
  if ((int64_t)maps[0].ny * maps[0].nz > (int64_t)INT32_MAX)
    return set_error(MI_E_RANGE, "mi_plan_create_fused: detector larger than 2^31 pixels");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_error(MI_E_CUDA, "mi_plan_create_fused: no CUDA device available");
  if (device < 0 || device >= ndev) return set_error(MI_E_ARG, "mi_plan_create_fused: bad device %d", device);
  HostThreads ht(o.host_threads);
  HostCSR csr;
  int rc = build_fused_csr(maps, n_shifts, r_axes, o.mode, &csr);
  if (rc) return rc;
  mi_map_desc vm = maps[0];
  vm.records = nullptr;
  vm.nmap = nullptr;
  vm.n_records = 0;
  for (int k = 0; k < n_shifts; ++k) vm.n_records += maps[k].n_records;
  mi_plan *p = new (std::nothrow) mi_plan();
  if (!p) return set_error(MI_E_OOM, "mi_plan_create_fused: host allocation failed");
  p->device = device;
  int prev = 0;
  cudaGetDevice(&prev);
  rc = build_plan(vm, o, p, &csr);
  cudaSetDevice(prev);
  if (rc) {
    free_plan_mem(p);
    delete p;
    return rc;
  }
  *out = p;
  return MI_OK;
}

int mi_plan_set_dark_panels(mi_plan *p, const float *const *darks) {
  if (!p || !darks) return set_error(MI_E_ARG, "mi_plan_set_dark_panels: null argument");
  std::vector<float> v((size_t)p->ny * p->nz, 0.0f);
  for (size_t i = 0; i < p->panels.size(); ++i) {
    const Plan::Panel &pn = p->panels[i];
    if (!darks[i]) continue;
    for (int z = 0; z < pn.nz; ++z)
      memcpy(v.data() + (size_t)(pn.z_off + z) * p->ny, darks[i] + (size_t)z * pn.ny, pn.ny * sizeof(float));
  }
  return mi_plan_set_dark(p, v.data());
}

int mi_plan_set_dark(mi_plan *p, const float *dark) {
  if (!p) return set_error(MI_E_ARG, "mi_plan_set_dark: null plan");
  const size_t n = (size_t)p->ny * p->nz;
  int prev = 0;
  cudaGetDevice(&prev);
  MI_CUDA(cudaSetDevice(p->device));
  if (dark) MI_CUDA(copy_pieces(p->d_dark, dark, n * sizeof(float), cudaMemcpyHostToDevice));
  else MI_CUDA(cudaMemset(p->d_dark, 0, n * sizeof(float)));
  p->has_dark = dark ? 1 : 0;
  int rc = MI_OK;
  if (p->encoding == MI_ENC_MMA || p->encoding == MI_ENC_MMAD) {
    // the per-bin dark terms, computed once per dark on the legacy stream; waiting for that
    // stream alone leaves other threads' streams running
    rc = p->encoding == MI_ENC_MMA ? launch_mma_dark(p, nullptr) : launch_mmad_dark(p, nullptr);
    if (rc == MI_OK) MI_CUDA(cudaStreamSynchronize(nullptr));
  }
  cudaSetDevice(prev);
  return rc;
}

int mi_plan_set_mma_pipeline(mi_plan *p, int stages, int producers) {
  if (!p) return set_error(MI_E_ARG, "mi_plan_set_mma_pipeline: null plan");
  if (p->encoding != MI_ENC_MMA)
    return set_error(MI_E_UNSUPPORTED, "mi_plan_set_mma_pipeline: the plan does not use the MMA encoding");
  if (!mma_pipeline_supported(stages, producers))
    return set_error(MI_E_UNSUPPORTED, "mi_plan_set_mma_pipeline: no kernel for %d stages and %d producers "
                                       "(8/6, 7/6, 6/6, 5/5, 7/7, 4/4)", stages, producers);
  p->mma_stages = stages;
  p->mma_producers = producers;
  return MI_OK;
}

int mi_plan_set_bin_mask(mi_plan *p, const uint8_t *mask) {
  if (!p) return set_error(MI_E_ARG, "mi_plan_set_bin_mask: null plan");
  if (p->semantics != MI_SEM_OMP)
    return set_error(MI_E_ARG, "mi_plan_set_bin_mask: only MI_SEM_OMP plans write masked bins as NaN");
  std::vector<int32_t> bins;
  if (mask)
    for (int64_t b = 0; b < p->n_bins; ++b)
      if (mask[b]) bins.push_back((int32_t)b);
  int prev = 0;
  cudaGetDevice(&prev);
  MI_CUDA(cudaSetDevice(p->device));
  MI_CUDA(cudaDeviceSynchronize());
  cudaFree(p->d_nan_bins);
  p->d_nan_bins = nullptr;
  p->n_nan_bins = 0;
  int rc = MI_OK;
  if (!bins.empty()) {
    size_t acct = 0;
    rc = upload(&p->d_nan_bins, bins.data(), bins.size(), &acct);
    if (rc == MI_OK) p->n_nan_bins = (int)bins.size();
  }
  cudaSetDevice(prev);
  return rc;
}

int mi_plan_get_info(const mi_plan *p, mi_plan_info *info) {
  if (!p || !info) return set_error(MI_E_ARG, "mi_plan_get_info: null argument");
  info->n_bins = p->n_bins;
  info->n_r = p->n_r;
  info->n_eta = p->n_eta;
  info->nnz = p->nnz;
  info->n_records = p->n_records;
  info->n_tiles = p->n_tiles;
  info->n_items = p->n_items;
  info->staged_pixels = p->staged_pixels;
  info->ref_pixels = p->ref_pixels;
  info->map_bytes = (int64_t)p->blob_bytes;
  info->device_bytes = (int64_t)p->device_bytes;
  info->oob_records = p->oob;
  info->tile_rows = p->lim.rows;
  info->tile_pixels = p->lim.max_u;
  info->frames_per_lane = p->frames_per_lane;
  info->run_len = p->run_l;
  info->xc_pixels = p->n_xc;
  info->ref_row_lo = p->ref_row_lo;
  info->ref_row_hi = p->ref_row_hi;
  info->upload_pixels = 0;
  for (const int4 &g : p->upload_groups) info->upload_pixels += (int64_t)(g.y - g.x) * (g.w - g.z);
  return MI_OK;
}

int mi_plan_status(mi_plan *p, int *status) {
  if (!p || !status) return set_error(MI_E_ARG, "mi_plan_status: null argument");
  int prev = 0;
  cudaGetDevice(&prev);
  MI_CUDA(cudaSetDevice(p->device));
  MI_CUDA(cudaDeviceSynchronize());
  MI_CUDA(cudaMemcpy(status, p->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  MI_CUDA(cudaMemset(p->d_err, 0, sizeof(int)));
  cudaSetDevice(prev);
  return MI_OK;
}

int mi_plan_bytes(const mi_plan *p, size_t *bytes) {
  if (!p || !bytes) return set_error(MI_E_ARG, "mi_plan_bytes: null argument");
  *bytes = p->device_bytes;
  return MI_OK;
}

void mi_plan_destroy(mi_plan *p) {
  if (!p) return;
  int prev = 0;
  cudaGetDevice(&prev);
  free_plan_mem(p);
  cudaSetDevice(prev);
  delete p;
}

int mi_integrate_batch(mi_plan *p, const void *frames, int dtype, int n_frames, int64_t stride,
                       float *cake, double *lo_aw, double *lo_sm, void *stream) {
  if (!p || !frames) return set_error(MI_E_ARG, "mi_integrate_batch: null argument");
  if (p->panels.size() > 1)
    return set_error(MI_E_ARG, "mi_integrate_batch: a panel plan takes its frames per panel: use mi_integrate_panels");
  if (n_frames < 0) return set_error(MI_E_ARG, "mi_integrate_batch: n_frames < 0");
  if (dtype_size(dtype) == 0) return set_error(MI_E_ARG, "mi_integrate_batch: unknown dtype code %d", dtype);
  if (stride < (int64_t)p->ny * p->nz)
    return set_error(MI_E_ARG, "mi_integrate_batch: frame_stride %lld < ny*nz", (long long)stride);
  if (n_frames == 0) return MI_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != p->device) MI_CUDA(cudaSetDevice(p->device));
  int rc = MI_OK;
  const size_t es = dtype_size(dtype);
  for (int f0 = 0; f0 < n_frames && rc == MI_OK; f0 += kMaxFramesPerLaunch) {
    int nf = std::min(kMaxFramesPerLaunch, n_frames - f0);
    rc = launch_cake(p, (const uint8_t *)frames + (size_t)f0 * stride * es, dtype, nf, stride,
                     cake ? cake + (size_t)f0 * p->n_bins : nullptr,
                     lo_aw ? lo_aw + (size_t)f0 * p->n_r : nullptr,
                     lo_sm ? lo_sm + (size_t)f0 * p->n_r : nullptr, p->d_partial, (cudaStream_t)stream);
  }
  if (prev != p->device) cudaSetDevice(prev);
  return rc;
}

int mi_integrate_panels(mi_plan *p, const void *const *frames, const int *dtypes, const int64_t *strides,
                        int n_frames, float *cake, double *lo_aw, double *lo_sm, void *stream) {
  if (!p || !frames || !dtypes || !strides) return set_error(MI_E_ARG, "mi_integrate_panels: null argument");
  if (n_frames < 0) return set_error(MI_E_ARG, "mi_integrate_panels: n_frames < 0");
  if (p->n_xc == 0)
    return set_error(MI_E_UNSUPPORTED, "mi_integrate_panels: the plan has no pixel-major staging");
  const int np = (int)p->panels.size();
  bool as_f32 = false;
  for (int i = 0; i < np; ++i) {
    if (!frames[i] && n_frames > 0) return set_error(MI_E_ARG, "mi_integrate_panels: panel %d has no frames", i);
    if (dtype_size(dtypes[i]) == 0)
      return set_error(MI_E_ARG, "mi_integrate_panels: panel %d: unknown dtype code %d", i, dtypes[i]);
    if (strides[i] < (int64_t)p->panels[i].ny * p->panels[i].nz)
      return set_error(MI_E_ARG, "mi_integrate_panels: panel %d: frame_stride %lld < ny*nz", i,
                       (long long)strides[i]);
    if (!(dtypes[i] == MI_DT_U16 || dtypes[i] == MI_DT_U8)) as_f32 = true;
  }
  if (n_frames == 0 || (!cake && !lo_aw && !lo_sm)) return MI_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != p->device) MI_CUDA(cudaSetDevice(p->device));
  const cudaStream_t s = (cudaStream_t)stream;
  const bool want_lo = lo_aw || lo_sm;
  if (as_f32 && p->encoding == MI_ENC_MMA)
    return set_error(MI_E_UNSUPPORTED, "mi_integrate_panels: MMA plans take 8/16-bit frames only");
  const int chunk = as_f32 ? kXcFramesF * kXcGroupsF : kXcFrames * kXcGroups;
  int rc = MI_OK;
  for (int g0 = 0; g0 < n_frames && rc == MI_OK; g0 += kMaxFramesPerLaunch) {
    const int ng = std::min(kMaxFramesPerLaunch, n_frames - g0);
    for (int f0 = 0; f0 < ng && rc == MI_OK; f0 += chunk) {
      const int nf = std::min(chunk, ng - f0);
      for (int i = 0; i < np && rc == MI_OK; ++i)
        rc = launch_xc(p, i, (const uint8_t *)frames[i] + (size_t)(g0 + f0) * strides[i] * dtype_size(dtypes[i]),
                       dtypes[i], nf, strides[i], as_f32, s);
      if (rc == MI_OK && p->encoding == MI_ENC_MMA)
        rc = launch_mma(p, nf, cake ? cake + (size_t)(g0 + f0) * p->n_bins : nullptr,
                        p->d_partial + (size_t)f0 * p->n_r * p->n_slots * 2, want_lo, s);
      else if (rc == MI_OK)
        rc = launch_runs_staged(p, as_f32, nf, cake ? cake + (size_t)(g0 + f0) * p->n_bins : nullptr,
                                p->d_partial + (size_t)f0 * p->n_r * p->n_slots * 2, want_lo, s);
    }
    if (rc == MI_OK && want_lo)
      rc = launch_lineout(p, p->d_partial, ng, lo_aw ? lo_aw + (size_t)g0 * p->n_r : nullptr,
                          lo_sm ? lo_sm + (size_t)g0 * p->n_r : nullptr, s);
  }
  if (prev != p->device) cudaSetDevice(prev);
  return rc;
}

int mi_stage_host_frames(const mi_plan *p, const void *src, int dtype, int n_frames, int64_t src_stride, void *dst,
                         int64_t dst_stride) {
  if (!p || !src || !dst) return set_error(MI_E_ARG, "mi_stage_host_frames: null argument");
  if (p->panels.size() > 1) return set_error(MI_E_ARG, "mi_stage_host_frames: a panel plan has one band per panel");
  const size_t es = dtype_size(dtype);
  if (es == 0) return set_error(MI_E_ARG, "mi_stage_host_frames: unknown dtype code %d", dtype);
  const int64_t npix = (int64_t)p->ny * p->nz;
  if (n_frames < 0 || src_stride < npix || dst_stride < npix)
    return set_error(MI_E_ARG, "mi_stage_host_frames: bad frame count or stride");
  for (int f = 0; f < n_frames; ++f) {
    const uint8_t *s = (const uint8_t *)src + (size_t)f * src_stride * es;
    uint8_t *d = (uint8_t *)dst + (size_t)f * dst_stride * es;
    for (const int4 &g : p->upload_groups)
      for (int z = g.x; z < g.y; ++z) {
        const size_t o = ((size_t)z * p->ny + g.z) * es;
        memcpy(d + o, s + o, (size_t)(g.w - g.z) * es);
      }
  }
  return MI_OK;
}

int mi_upload_frames(const mi_plan *p, const void *host, int dtype, int n_frames, int64_t host_stride,
                     void *device_frames, int64_t device_stride, void *stream) {
  if (!p || !host || !device_frames) return set_error(MI_E_ARG, "mi_upload_frames: null argument");
  if (p->panels.size() > 1) return set_error(MI_E_ARG, "mi_upload_frames: a panel plan has one band per panel");
  const size_t es = dtype_size(dtype);
  if (es == 0) return set_error(MI_E_ARG, "mi_upload_frames: unknown dtype code %d", dtype);
  const int64_t npix = (int64_t)p->ny * p->nz;
  if (n_frames < 0 || host_stride < npix || device_stride < npix)
    return set_error(MI_E_ARG, "mi_upload_frames: bad frame count or stride");
  if (n_frames == 0 || p->ref_row_hi <= p->ref_row_lo) return MI_OK;
  if (!p->upload_groups.empty() && host_stride % p->ny == 0 && device_stride % p->ny == 0) {
    // one 3-D copy per row group: its referenced columns x its rows x the frames, so only
    // the referenced part of each row crosses PCIe (a frame is host_stride / ny rows deep)
    const size_t pitch = (size_t)p->ny * es;
    for (const int4 &g : p->upload_groups) {
      cudaMemcpy3DParms c = {};
      c.srcPtr = make_cudaPitchedPtr(const_cast<void *>(host), pitch, pitch, (size_t)(host_stride / p->ny));
      c.dstPtr = make_cudaPitchedPtr(device_frames, pitch, pitch, (size_t)(device_stride / p->ny));
      c.srcPos = make_cudaPos((size_t)g.z * es, (size_t)g.x, 0);
      c.dstPos = c.srcPos;
      c.extent = make_cudaExtent((size_t)(g.w - g.z) * es, (size_t)(g.y - g.x), (size_t)n_frames);
      c.kind = cudaMemcpyHostToDevice;
      MI_CUDA(cudaMemcpy3DAsync(&c, (cudaStream_t)stream));
    }
    return MI_OK;
  }
  const size_t off = (size_t)p->ref_row_lo * p->ny * es;
  const size_t width = (size_t)(p->ref_row_hi - p->ref_row_lo) * p->ny * es;
  MI_CUDA(cudaMemcpy2DAsync((uint8_t *)device_frames + off, (size_t)device_stride * es, (const uint8_t *)host + off,
                            (size_t)host_stride * es, width, (size_t)n_frames, cudaMemcpyHostToDevice,
                            (cudaStream_t)stream));
  return MI_OK;
}

int mi_integrate_plain(mi_plan *p, const void *frame, int dtype, double *cake, double *lo_aw,
                       double *lo_sm, void *stream) {
  if (!p || !frame) return set_error(MI_E_ARG, "mi_integrate_plain: null argument");
  if (p->panels.size() > 1 || !p->d_plain_img)
    return set_error(MI_E_UNSUPPORTED, "mi_integrate_plain: a panel plan has no one-frame path");
  if (dtype_size(dtype) == 0) return set_error(MI_E_ARG, "mi_integrate_plain: unknown dtype code %d", dtype);
  if (p->semantics == MI_SEM_IC || p->semantics == MI_SEM_OMP)
    return set_error(MI_E_UNSUPPORTED, "mi_integrate_plain: the one-frame GPU kernel follows the GPU stream "
                                       "or midas_integrate semantics, not IntegrationCore's");
  if (p->variance)
    return set_error(MI_E_UNSUPPORTED, "mi_integrate_plain: variance plans are caked by mi_integrate_batch");
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != p->device) MI_CUDA(cudaSetDevice(p->device));
  int rc = launch_plain(p, frame, dtype, cake, lo_aw, lo_sm, (cudaStream_t)stream);
  if (prev != p->device) cudaSetDevice(prev);
  return rc;
}

int mi_profile_batch(mi_plan *p, const void *cake, int cake_dtype, int n_frames, double *lo_aw, double *lo_sm,
                     void *stream) {
  if (!p || !cake) return set_error(MI_E_ARG, "mi_profile_batch: null argument");
  if (n_frames < 0) return set_error(MI_E_ARG, "mi_profile_batch: n_frames < 0");
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != p->device) MI_CUDA(cudaSetDevice(p->device));
  int rc = launch_profile(p, cake, cake_dtype, n_frames, lo_aw, lo_sm, (cudaStream_t)stream);
  if (prev != p->device) cudaSetDevice(prev);
  return rc;
}

int mi_sum_cake(mi_plan *p, const float *cake, int n_frames, double *sum, void *stream) {
  if (!p || !sum || (n_frames > 0 && !cake)) return set_error(MI_E_ARG, "mi_sum_cake: null argument");
  if (n_frames < 0) return set_error(MI_E_ARG, "mi_sum_cake: n_frames < 0");
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != p->device) MI_CUDA(cudaSetDevice(p->device));
  int rc = launch_sum_cake(p, cake, n_frames, sum, (cudaStream_t)stream);
  if (prev != p->device) cudaSetDevice(prev);
  return rc;
}

int mi_plan_bin_table(const mi_plan *p, const double *r_lo, const double *r_hi, const double *eta_lo,
                      const double *eta_hi, double px_um, double lsd_um, double wavelength_a, double *table) {
  if (!p || !r_lo || !r_hi || !eta_lo || !eta_hi || !table) return set_error(MI_E_ARG, "mi_plan_bin_table: null argument");
  if (lsd_um == 0.0) return set_error(MI_E_ARG, "mi_plan_bin_table: Lsd must be non-zero");
  // initialize_PerFrameArr_Area_kernel (IntegratorFitPeaksGPUStream.cu:817-899)
  const double rad2deg = 180.0 / M_PI;
  for (int r = 0; r < p->n_r; ++r)
    for (int e = 0; e < p->n_eta; ++e) {
      const int64_t b = (int64_t)r * p->n_eta + e;
      const double rm = (r_lo[r] + r_hi[r]) * 0.5, em = (eta_lo[e] + eta_hi[e]) * 0.5;
      const double tth = atan(rm * px_um / lsd_um);
      double *t = table + b * MI_BIN_NCOL;
      t[0] = rm;
      t[1] = rad2deg * tth;
      t[2] = em;
      t[3] = p->area_gs[b];
      t[4] = wavelength_a > 0 ? (4.0 * M_PI / wavelength_a) * sin(tth / 2.0) : 0.0;
    }
  return MI_OK;
}

int mi_cast_dark(const void *frames, int dtype, int64_t n_pixels, int n_frames, const float *dark,
                 float *out, void *stream) {
  if (!frames || !out) return set_error(MI_E_ARG, "mi_cast_dark: null argument");
  if (dtype_size(dtype) == 0) return set_error(MI_E_ARG, "mi_cast_dark: unknown dtype code %d", dtype);
  if (n_pixels < 0 || n_frames < 0) return set_error(MI_E_ARG, "mi_cast_dark: negative size");
  if (n_pixels == 0 || n_frames == 0) return MI_OK;
  return launch_cast(frames, dtype, n_pixels, n_frames, dark, out, (cudaStream_t)stream);
}

}  // extern "C"
