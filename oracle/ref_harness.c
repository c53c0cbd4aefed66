/*
 * ref_harness.c -- drives the reference's own C implementation, compiled unmodified
 * from the MIDAS sources by oracle/Makefile into oracle/_ref/libmidas_ref.so.
 *
 * TEST AND BASELINE INFRASTRUCTURE ONLY (the checker and the timed CPU baseline).
 *
 *   ref_build_map  -> mapper_build_map (FF_HEDM/src/MapperCore.c:45), serialised
 *                     bin-major exactly as DetectorMapper does (DetectorMapper.c:813-834)
 *   ref_integrate  -> integration_apply_map (FF_HEDM/src/IntegrationCore.c:14),
 *                     split over R-row chunks with OpenMP (the same per-bin math as the
 *                     OpenMP loop of IntegratorZarrOMP.c:1709-1778, which needs HDF5,
 *                     blosc2 and libzip and cannot be built here).
 */
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "IntegrationCore.h"
#include "MapperCore.h"

long long ref_build_map(int ny, int nz, double px, double lsd, double bcy, double bcz, double tx, double ty,
                        double tz, double rhod, const double *p /*15*/, double parallax, int sa, int pol,
                        double polf, int spl, double spw, const double *rlo, const double *rhi,
                        const double *elo, const double *ehi, int nr, int neta, int nthreads,
                        struct MapPixelData **recs_out, int **nmap_out, int **binmask_out) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  struct MapPixelData ***pxList = malloc(nr * sizeof(*pxList));
  int **nPx = malloc(nr * sizeof(*nPx));
  int **maxn = malloc(nr * sizeof(*maxn));
  for (int i = 0; i < nr; i++) {
    pxList[i] = calloc(neta, sizeof(*pxList[i]));
    nPx[i] = calloc(neta, sizeof(*nPx[i]));
    maxn[i] = calloc(neta, sizeof(*maxn[i]));
  }
  long long nb = (long long)nr * neta;
  int *mask_flag = calloc(nb, sizeof(int));
  double *dmy = calloc((size_t)ny * nz, sizeof(double));
  double *dmz = calloc((size_t)ny * nz, sizeof(double));
  omp_lock_t *locks = malloc(MAPPER_N_BIN_LOCKS * sizeof(omp_lock_t));
  for (int i = 0; i < MAPPER_N_BIN_LOCKS; i++) omp_init_lock(&locks[i]);
  int trans[10] = {0};
  long long tot = mapper_build_map(tx, ty, tz, ny, nz, px, px, bcy, bcz, lsd, rhod, p[0], p[1], p[2], p[3], p[4],
                                   p[5], p[6], p[7], p[8], p[9], p[10], p[11], p[12], p[13], p[14], (double *)elo,
                                   (double *)ehi, (double *)rlo, (double *)rhi, nr, neta, pxList, nPx, maxn, NULL,
                                   mask_flag, 0, trans, locks, spl, spw, parallax, sa, pol, polf, dmy, dmz, NULL, 0,
                                   NULL);
  for (int i = 0; i < MAPPER_N_BIN_LOCKS; i++) omp_destroy_lock(&locks[i]);
  free(locks);
  struct MapPixelData *recs = malloc((tot > 0 ? tot : 1) * sizeof(*recs));
  int *nmap = malloc(nb * 2 * sizeof(int));
  long long cur = 0;
  for (int i = 0; i < nr; i++)
    for (int j = 0; j < neta; j++) {
      long long pos = (long long)i * neta + j;
      nmap[2 * pos] = nPx[i][j];
      nmap[2 * pos + 1] = (int)cur;
      if (nPx[i][j]) memcpy(recs + cur, pxList[i][j], nPx[i][j] * sizeof(*recs));
      cur += nPx[i][j];
      free(pxList[i][j]);
    }
  for (int i = 0; i < nr; i++) {
    free(pxList[i]);
    free(nPx[i]);
    free(maxn[i]);
  }
  free(pxList);
  free(nPx);
  free(maxn);
  free(dmy);
  free(dmz);
  *recs_out = recs;
  *nmap_out = nmap;
  *binmask_out = mask_flag;
  return cur;
}

void ref_free(void *p) { free(p); }

/* R rows are split into chunks processed in parallel; each chunk calls the reference
 * integration_apply_map on its own rows (pointer-table views into the same map). */
int ref_integrate(const struct MapPixelData *recs, const int *nmap, int nr, int neta, const double *image, int ny,
                  int nz, const double *dark, double bcy, double bcz, int gradient, int nthreads, int chunk_rows,
                  double *profiles, double *norm) {
  struct MapPixelData ***px = malloc(nr * sizeof(*px));
  int **npx = malloc(nr * sizeof(*npx));
  for (int r = 0; r < nr; r++) {
    px[r] = malloc(neta * sizeof(*px[r]));
    npx[r] = malloc(neta * sizeof(*npx[r]));
    for (int e = 0; e < neta; e++) {
      long long b = (long long)r * neta + e;
      npx[r][e] = nmap[2 * b];
      px[r][e] = (struct MapPixelData *)(recs + nmap[2 * b + 1]);
    }
  }
  if (chunk_rows < 1) chunk_rows = 8;
  int nchunks = (nr + chunk_rows - 1) / chunk_rows;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nchunks; c++) {
    int r0 = c * chunk_rows;
    int n = nr - r0 < chunk_rows ? nr - r0 : chunk_rows;
    long long o = (long long)r0 * neta;
    integration_apply_map(px + r0, npx + r0, n, neta, image, ny, nz, dark, bcy, bcz, gradient, profiles + o,
                          norm + o);
  }
  for (int r = 0; r < nr; r++) {
    free(px[r]);
    free(npx[r]);
  }
  free(px);
  free(npx);
  return 0;
}

int ref_max_threads(void) { return omp_get_max_threads(); }
