/*
 * midas_b200.h -- C ABI of the B200-native radial-integration ("caking") engine.
 *
 * This is the drop-in boundary for the MIDAS caking hot path.  Every entry point
 * takes plain pointers and sizes; no PyTorch or CUDA C++ types cross it (a CUDA
 * stream is passed as an opaque `void*`, NULL meaning the legacy default stream).
 *
 * Reference interfaces replaced (paths inside the MIDAS repository):
 *   mi_plan_create       <- build_csr()                packages/midas_integrate/midas_integrate/kernels.py:242
 *                           + ReadBins/PrecomputeOffsets FF_HEDM/src/IntegratorFitPeaksGPUStream.cu:742,901
 *                           + initialize_PerFrameArr_Area_kernel  IntegratorFitPeaksGPUStream.cu:817
 *   mi_plan_set_dark     <- dark upload (average of dark frames) IntegratorFitPeaksGPUStream.cu:2191-2238
 *   mi_integrate_batch   <- integrate() + profile_1d()  kernels.py:416,567 (one frame per call there;
 *                           here F frames per launch), and the submit path of the GPU stream,
 *                           IntegratorFitPeaksGPUStream.cu:2806-2870
 *   mi_integrate_plain   <- ProcessImageGPU + integrate_noMapMask + calculate_1D_profile_kernel(s),
 *                           IntegratorFitPeaksGPUStream.cu:1633,975,1162,1256 (one frame per launch,
 *                           thread per sorted bin: the reference's own GPU algorithm)
 *   mi_cast_dark         <- process_direct_kernel<T>   IntegratorFitPeaksGPUStream.cu:1148
 *   mi_fit_batch         <- fitPeaks()                 FF_HEDM/src/PeakFit.c:275 (called per frame at
 *                           IntegratorFitPeaksGPUStream.cu:2630-2702) and fit_peaks()
 *                           packages/midas_integrate/midas_integrate/peakfit.py:334
 *   mi_fit_plan_*        <- fitPeaks() job construction and joint fits, PeakFit.c:292-545, and the
 *                           per-eta fits of FF_HEDM/src/IntegratorZarrOMP.c:1902-2030
 *   mi_plan_create_fused <- build_fused_geometry()     packages/midas_integrate/midas_integrate/fused_csr.py:139
 *   mi_map_build         <- mapper_build_map()         FF_HEDM/src/MapperCore.c:45 (DetectorMapper)
 *   mi_last_error        <- (new) the reference aborts the process on any CUDA error
 *                           (gpuAssert, IntegratorFitPeaksGPUStream.cu:299-308); this library
 *                           returns a status code and keeps a thread-local message instead.
 *
 * Status codes: 0 = ok, negative = error (see MI_E_*).  No entry point ever calls exit().
 */
#ifndef MIDAS_B200_H
#define MIDAS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define MI_OK 0
#define MI_E_ARG (-1)        /* bad argument (null pointer, size, unknown code)          */
#define MI_E_MAP (-2)        /* malformed map: negative count, offset past end of Map.bin */
#define MI_E_OOM (-3)        /* device or host allocation failed                         */
#define MI_E_CUDA (-4)       /* CUDA runtime error (message has the CUDA error string)   */
#define MI_E_TIMEOUT (-5)    /* a bounded device wait expired                            */
#define MI_E_UNSUPPORTED (-6)/* valid request this build does not implement              */
#define MI_E_RANGE (-7)      /* size beyond a documented maximum                         */

/* ---- integration modes (MI/kernels.py module docstring) ----------------- */
#define MI_MODE_FLOOR 0      /* truncated (y,z) lookup, 1 term per Map.bin record        */
#define MI_MODE_BILINEAR 1   /* bilinear sample at (y,z), 4 corner terms, coalesced      */
#define MI_MODE_GRADIENT 2   /* bilinear at (y,z) shifted by -deltaR along the radius    */

/* ---- semantics: the reference's three integrators differ in rounding and normaliser -- */
#define MI_SEM_PY 0          /* midas_integrate kernels.py: normaliser = sum of in-bounds
                                areaWeight; invalid bins -> 0 when normalising, raw sum
                                otherwise (kernels.py:311-318, 461-471)                  */
#define MI_SEM_GPUSTREAM 1   /* IntegratorFitPeaksGPUStream.cu:1038-1049: normaliser = sum
                                of ALL areaWeight of the bin; bins with area <= 1e-9 -> 0 */
#define MI_SEM_IC 2          /* IntegrationCore.c:integration_apply_map (:14-82), the CPU
                                integrator: bilinear at (y,z) (gradient: shifted by
                                -deltaR*d/R in FP64 when deltaR != 0 and R > 1), base pixel
                                = floorf() of the position rounded to float, clamp under
                                then over; normaliser = sum of ALL areaWeight (<= 1e-9 ->
                                0). It has no floor mode: MI_MODE_FLOOR is rejected, and
                                mi_integrate_plain does not take this semantics.          */
#define MI_SEM_OMP 3         /* IntegratorZarrOMP.c:1709-1778 (the OpenMP integrator): the
                                sums of MI_SEM_IC; a nonzero sum is divided by the sum of
                                ALL areaWeight of the bin (no validity threshold; a bin with
                                a nonzero sum and zero area gives 0 here, +-inf there); bins
                                flagged by mi_plan_set_bin_mask are NaN; lineout_sm is the
                                mean of the row's nonzero, non-NaN bins (:1829-1843) and
                                lineout_aw the area-weighted mean over its valid, non-NaN
                                bins, both computed from the cake, which must be requested
                                with them.  No floor mode; single-detector plans only.    */

/* ---- frame dtype codes: the socket protocol's codes (MI/image.py:24-30) -- */
#define MI_DT_U8 0
#define MI_DT_U16 1
#define MI_DT_U32 2
#define MI_DT_I64 3
#define MI_DT_F32 4
#define MI_DT_F64 5
#define MI_DT_HYBRID 6       /* u16 base + int64 overflow patch: decoded by mi_decode_hybrid */
#define MI_DT_I32 7          /* extension: PILATUS-style signed 32-bit frames            */

/* ---- maps ---------------------------------------------------------------- */
/* One Map.bin record, 24 bytes, layout of struct data / MapPixelData
 * (IntegratorFitPeaksGPUStream.cu:234-240, FF_HEDM/src/MapperCore.h:19-25). */
typedef struct {
  float y;           /* pixel column (+ sub-pixel centroid offset)            */
  float z;           /* pixel row                                             */
  double frac;       /* corrected weight = area / (solid angle x polarisation) */
  float deltaR;      /* R(sub-pixel centre) - R(bin centre), px               */
  float areaWeight;  /* geometric pixel-bin overlap area                      */
} mi_map_record;

typedef struct {
  const mi_map_record *records; /* host pointer: Map.bin data (header skipped)          */
  int64_t n_records;
  const int32_t *nmap;          /* host pointer: nMap.bin {count, offset} pairs, n_bins */
  int32_t n_r, n_eta;           /* bins are R-major: bin = r * n_eta + eta              */
  int32_t ny, nz;               /* NrPixelsY, NrPixelsZ; flat pixel = z * ny + y        */
  double bc_y, bc_z;            /* beam centre (px), used by MI_MODE_GRADIENT           */
} mi_map_desc;

typedef struct {
  int32_t mode;            /* MI_MODE_*                                              */
  int32_t normalize;       /* Normalize key (1 = divide by bin area)                  */
  int32_t semantics;       /* MI_SEM_*                                               */
  int32_t tile_rows;       /* rows (R bins) per tile strip; 0 = autotune              */
  int32_t tile_pixels;     /* max staged pixels per tile; 0 = autotune                */
  int32_t frames_per_lane; /* CSR encoding only: 1, 2 or 4 frames per thread; 0 = auto */
  int32_t encoding;        /* MI_ENC_*: tile encoding of the map                      */
  int32_t run_len;         /* run encoding: rows per record (2, 4 or 8); 0 = auto      */
  int32_t variance;        /* 1 = variance plan: the cake of a variance map (per-pixel
                              variances, dark already subtracted) under squared weights,
                              integrate_with_variance (MI/kernels.py:474-536): bin
                              variance = sum(w^2 var) / A^2 (normalised) or sum(w^2 var);
                              lineouts are the propagated variances of profile_1d
                              (kernels.py:567-628): sum(A^2 var) / (sum A)^2 and
                              sum(var) / N^2.  mi_integrate_plain rejects such plans.  */
  int32_t host_threads;    /* host threads building the plan (0 = all): a server that
                              admits a stream while serving others leaves cores to them */
} mi_plan_opts;

#define MI_ENC_AUTO 0      /* runs                                                       */
#define MI_ENC_CSR 1       /* per-bin term lists, one warp per bin, lane = frame         */
#define MI_ENC_RUNS 2      /* per-pixel radial runs: one staged value feeds run_len bins */
#define MI_ENC_MMA 3       /* tensor cores (8/16-bit frames only): 12 x 4-bin tiles as dense
                              int8 MMAs, frames split into two u8 byte planes and weights into
                              signed fixed point (four s8 digits, relative to the bin's largest
                              |weight|), exact int32 accumulation, FP64 recombination; other
                              frame types get
                              MI_E_UNSUPPORTED                                            */
#define MI_ENC_MMAD 4      /* tensor cores reading the frames in place (u16/u8 frames): the
                              tiles of MI_ENC_MMA, pixels in 8-pixel row granules loaded per
                              frame into tensor memory (one vector load per granule when rows
                              are a multiple of 8 pixels and frames and strides 16-byte
                              aligned), the same signed weight digits, five int32 accumulators;
                              no pixel-major staging pass                                 */

typedef struct {
  int64_t n_bins, n_r, n_eta;
  int64_t nnz;             /* terms of the selected mode after coalescing             */
  int64_t n_records;       /* Map.bin records read                                   */
  int64_t n_tiles, n_items;/* staging tiles, scheduled work items                     */
  int64_t staged_pixels;   /* sum over tiles of staged pixels (halo included)          */
  int64_t ref_pixels;      /* distinct pixels the map references                       */
  int64_t map_bytes;       /* device bytes of the tiled map read per batch             */
  int64_t device_bytes;    /* all device memory the plan holds                        */
  int64_t oob_records;     /* records whose truncated (y,z) is off the detector        */
  int32_t tile_rows, tile_pixels, frames_per_lane;
  int32_t run_len;         /* register-run length of the tile encoding                 */
  int64_t xc_pixels;       /* pixels of the pixel-major staging spans (run encoding with
                              tile_rows <= 16); 0: frames are gathered frame-major     */
  int32_t ref_row_lo, ref_row_hi; /* detector rows [lo, hi) holding referenced pixels  */
  int64_t upload_pixels;   /* pixels of one frame mi_upload_frames copies: per group of 16
                              rows of the band, the columns any of them references       */
} mi_plan_info;

typedef struct mi_plan mi_plan; /* opaque, immutable after creation except for the dark */

/* Build a device-resident plan for one (map, binning, mode).  Validates the map
 * (counts >= 0, offset + count <= n_records) like build_csr (kernels.py:288-301). */
int mi_plan_create(const mi_map_desc *map, const mi_plan_opts *opts, int device,
                   mi_plan **out);
/* Set (or clear, dark == NULL) the per-pixel dark (ny*nz floats, host pointer).
 * The reference subtracts (float)raw - dark[pixel] (IntegratorFitPeaksGPUStream.cu:1156). */
int mi_plan_set_dark(mi_plan *plan, const float *dark_host);
int mi_plan_get_info(const mi_plan *plan, mi_plan_info *info);

/* ---- panels: several detectors, one binning, one merged cake ---------------------------
 * Replaces the per-panel integrate-then-merge of multi-detector setups (one
 * integrate() + profile_1d() per detector, packages/midas_integrate/midas_integrate/
 * kernels.py:416,567, and one IntegratorFitPeaksGPUStream per detector).  Each panel has
 * its own map (geometry, beam centre, mask, dtype) over the SAME n_r x n_eta bins (R or
 * Q binning).  A bin of the merged cake is the sum of all panels' weighted pixels over
 * the sum of their areas: one concatenated weight list, as if the panels were one
 * detector.  The panels' rows are stacked into a virtual detector as wide as the widest
 * panel (panel i: rows z_off_i .. z_off_i + nz_i - 1, z_off_i = nz_0 + .. + nz_{i-1}).
 * The plan uses the run encoding (tile_rows <= 16).  mi_integrate_batch and
 * mi_integrate_plain reject panel plans.                                              */
int mi_plan_create_panels(const mi_map_desc *maps, int n_panels, const mi_plan_opts *opts,
                          int device, mi_plan **out);
/* One dark per panel (ny_i*nz_i floats, host pointers; NULL entries = no dark). */
int mi_plan_set_dark_panels(mi_plan *plan, const float *const *darks_host);
/* F frames of every panel (device pointers, panel i frame f at frames[i] + f*strides[i]
 * elements of dtypes[i]; types may differ between panels) -> merged cake [F][n_r][n_eta]
 * and lineouts, like mi_integrate_batch.  Kernel (a) transposes each panel's frames into
 * the plan's pixel-major buffer, then one launch of kernel (b) cakes all panels. */
int mi_integrate_panels(mi_plan *plan, const void *const *frames, const int *dtypes,
                        const int64_t *strides, int n_frames, float *cake, double *lineout_aw,
                        double *lineout_sm, void *stream);
/* ---- fused multi-shift maps ------------------------------------------------------------
 * Replaces build_fused_geometry (packages/midas_integrate/midas_integrate/fused_csr.py:139):
 * n_shifts maps of one detector whose R edges are shifted by k / n_shifts of a bin
 * (RMin + k/N x RBinSize), r_axes[k] the n_r of map k's R bin centres.  Each shift's
 * bilinear or gradient weights (py semantics) are divided by the bin's in-bounds area
 * (bins at or under 1e-9: 0), moved onto shift 0's R axis by linear interpolation in R
 * (at most two source rows per row, fused_csr.py:63-104: clamped to the first / last pair
 * outside the axis), summed over the shifts and divided by n_shifts.  The cake of the
 * fused plan is the average of the shifts' normalised cakes, interpolated onto shift 0's
 * axis, in one pass; every bin's area is 1, so `normalize` changes nothing and the
 * lineouts weigh every bin of a row alike.  Shifts share n_eta and the detector shape;
 * n_r may differ (at least 2).  opts: mode bilinear or gradient, semantics MI_SEM_PY, no
 * variance; any encoding.                                                              */
int mi_plan_create_fused(const mi_map_desc *maps, int n_shifts, const double *const *r_axes,
                         const mi_plan_opts *opts, int device, mi_plan **out);
/* The fused weights themselves, on the host (no device needed): row_ptr (n_bins + 1, or
 * NULL), then col / w (both NULL to ask for *nnz only, else `capacity` entries). */
int mi_fused_csr(const mi_map_desc *maps, int n_shifts, const double *const *r_axes, int mode,
                 int64_t *row_ptr, int32_t *col, double *w, int64_t capacity, int64_t *nnz);

/* Failure-detection self test (no counterpart in the reference, which aborts on errors):
 * one mbarrier wait bounded to `polls` polls, as every wait in this library's kernels is,
 * on a barrier that nothing completes (arrive = 0) or that its thread completed first
 * (arrive = 1).  *status receives MI_E_TIMEOUT when the limit ran out, MI_OK when the wait
 * succeeded; the device context stays usable either way. */
int mi_selftest_wait(uint32_t polls, int arrive, int device, int *status);

/* Per-bin mask of a MI_SEM_OMP plan (host, n_bins bytes, nonzero = the bin holds a masked
 * pixel, DetectorMapper's bin mask): those bins of every cake are NaN, as the OpenMP
 * integrator writes them (IntegratorZarrOMP.c:1766-1767).  NULL clears it. */
int mi_plan_set_bin_mask(mi_plan *plan, const uint8_t *bin_mask);
/* Pipeline depth of the MMA encoding's kernel (no counterpart in the reference): stage
 * slots and producer warps, one of the compiled pairs 8/6 (the default), 7/6, 6/6, 5/5,
 * 7/7, 4/4; MI_E_UNSUPPORTED for other pairs or plans of other encodings.  Results are the same
 * bit for bit; only the time differs (the autotuner times them per map). */
int mi_plan_set_mma_pipeline(mi_plan *plan, int stages, int producers);

/* Device-side status of the plan's launches so far: the plan's error word (MI_E_TIMEOUT
 * when a bounded in-kernel wait expired, else 0), which is then cleared.  Synchronises
 * the plan's device. */
int mi_plan_status(mi_plan *plan, int *device_status);
int mi_plan_bytes(const mi_plan *plan, size_t *bytes);
void mi_plan_destroy(mi_plan *plan);

/* Host -> device copy of F frames for this plan: only the pixels the map can read cross
 * PCIe.  Per group of 16 detector rows of the referenced band (ref_row_lo .. ref_row_hi-1)
 * the columns any row of the group references (rounded out to 8 pixels), all F frames in one
 * 3-D copy on `stream` (upload_pixels of mi_plan_info per frame); when a stride is not a
 * whole number of rows, the band's full rows in one 2-D copy.  The other pixels of the
 * device frames are left as they are, and no kernel reads them.  The reference copies every
 * whole frame (IntegratorFitPeaksGPUStream.cu:1633-1683).  `host` should be page-locked for
 * the copy to be asynchronous. */
int mi_upload_frames(const mi_plan *plan, const void *host, int dtype, int n_frames,
                     int64_t host_stride, void *device_frames, int64_t device_stride,
                     void *stream);
/* Host -> host copy of F frames (e.g. into the page-locked buffer mi_upload_frames then
 * sends) of exactly the pixels mi_upload_frames copies (upload_pixels of mi_plan_info per
 * frame); the destination's other pixels are left as they are.  No device work.  A
 * server stages a caller's frame with it instead of copying the whole frame. */
int mi_stage_host_frames(const mi_plan *plan, const void *src, int dtype, int n_frames,
                         int64_t src_stride, void *dst, int64_t dst_stride);

/* Cake F frames in one launch.
 *   frames:      device pointer, F frames of ny*nz pixels, frame f at frames + f*frame_stride
 *                elements (frame_stride >= ny*nz)
 *   cake:        device [F][n_r][n_eta] float32, or NULL to skip the 2D output
 *   lineout_aw:  device [F][n_r] float64, area-weighted eta average (calculate_1D_profile_kernel,
 *                IntegratorFitPeaksGPUStream.cu:1162), or NULL
 *   lineout_sm:  device [F][n_r] float64, simple mean over valid bins (…_simple_mean_kernel,
 *                IntegratorFitPeaksGPUStream.cu:1256), or NULL
 *   stream:      cudaStream_t or NULL
 * Results for a frame do not depend on F or on the other frames in the batch. */
int mi_integrate_batch(mi_plan *plan, const void *frames, int dtype, int n_frames,
                       int64_t frame_stride, float *cake, double *lineout_aw,
                       double *lineout_sm, void *stream);

/* mi_integrate_batch that allocates nothing (no counterpart in the reference).
 * For callers that cannot have device memory allocated for them once running -- a
 * detector front-end that reserves the device's whole memory budget at start-up and
 * hands the library only its own buffers -- the batched kernels keep their only scratch, the
 * per-row lineout partial sums, in a fixed 8 MiB array inside the library (held on every
 * GPU that loads it until exit).  Same arguments and results as mi_integrate_batch;
 * frames are processed in chunks that fit the array; a plan needing more than the array
 * for one frame (n_r x 12 x 2 doubles > 1,048,576) gets MI_E_RANGE.  The first call on a
 * device looks up the array's address: make it before any stream capture.  Calls that
 * overlap on the GPU share the array and race.  A device reset while the library is loaded
 * is not supported (the looked-up address is kept).  On a tensor-core (MMA) plan the chunk
 * is bounded by the array (11 frames per launch for 3960 x 360 bins), which costs speed. */
int mi_integrate_batch_static(mi_plan *plan, const void *frames, int dtype, int n_frames,
                              int64_t frame_stride, float *cake, double *lineout_aw,
                              double *lineout_sm, void *stream);

/* The reference's own GPU algorithm, one frame per launch: cast/dark kernel, one thread per
 * bin in heaviest-first order with FP32 accumulation and on-the-fly bilinear sampling in
 * gradient mode, FP64 cake, then the two profile kernels.  This is the plain baseline. */
int mi_integrate_plain(mi_plan *plan, const void *frame, int dtype, double *cake,
                       double *lineout_aw, double *lineout_sm, void *stream);

/* SumImages (IntegratorFitPeaksGPUStream.cu:1043-1046, the running dSumMatrix of
 * :2141-2144): sum[b] += cake[f][b] for the F frames of a float32 [F][n_r][n_eta] device
 * cake, in FP64 and frame order; NaN bins add nothing.  sum: n_r*n_eta doubles on the
 * device, zeroed by the caller before the first batch; stream-ordered like the caking. */
int mi_sum_cake(mi_plan *plan, const float *cake, int n_frames, double *sum, void *stream);

/* Kernel (c) on a cake the caller already holds: area-weighted and simple-mean eta
 * reductions of F frames of a [F][n_r][n_eta] cake (float32 with cake_dtype = MI_DT_F32,
 * float64 with MI_DT_F64), with the plan's in-bounds bin areas (profile_1d,
 * packages/midas_integrate/midas_integrate/kernels.py:567). */
int mi_profile_batch(mi_plan *plan, const void *cake, int cake_dtype, int n_frames,
                     double *lineout_aw, double *lineout_sm, void *stream);

/* Kernel (a) on its own: out[f][p] = (float)frames[f][p] - dark[p] (dark may be NULL),
 * 128-bit vector loads.  frames and out are device pointers. */
int mi_cast_dark(const void *frames, int dtype, int64_t n_pixels, int n_frames,
                 const float *dark, float *out, void *stream);

/* Per-pixel mean of k frames, accumulated in FP64 and stored as float: the dark
 * average of the stream server's start-up (IntegratorFitPeaksGPUStream.cu:2191-2238,
 * average_dark_frames, MI/image.py:161-184), on the device.  frames: device pointer,
 * frame f at frames + f*frame_stride elements of dtype (not MI_DT_HYBRID); out: device
 * [n_pixels] float.  The result can be passed to mi_plan_set_dark after a copy to the host,
 * or used on the device directly. */
int mi_average_frames(const void *frames, int dtype, int64_t n_pixels, int n_frames,
                      int64_t frame_stride, float *out, void *stream);

/* Decode one hybrid (dtype code 6) socket payload into a float frame of raw counts on
 * the device.  payload: host bytes as received, [u32 C][u16 base, ny*nz][i32 index, C]
 * [i64 value, C] (ProcessImageGPU_Hybrid_Impl, IntegratorFitPeaksGPUStream.cu:1497-1560;
 * decode_hybrid_payload, MI/image.py:83-123), best page-locked.  It crosses PCIe in one
 * copy into device_staging (>= payload_bytes + 4 bytes, 16-byte aligned, owned by the
 * caller; reused once the stream has passed the decode), out[p] = (float)base[p], then
 * out[index[i]] = (float)value[i].  The frame holds raw counts: cake it with dtype
 * MI_DT_F32 and the plan's dark, which gives (float)raw - dark like the reference.
 * A payload whose size does not match C and ny*nz is rejected on the host (MI_E_ARG);
 * an index outside the frame is skipped and sets *device_status (device int) to
 * MI_E_RANGE. */
int mi_decode_hybrid(const void *payload, size_t payload_bytes, int ny, int nz,
                     void *device_staging, float *out, int *device_status, void *stream);

/* Per-bin axis table of a plan, host doubles [n_r*n_eta][MI_BIN_NCOL], bin = r*n_eta + eta:
 *   R mean (px), 2-theta (deg) = atan(R * px / Lsd), eta mean (deg), bin area (sum of the
 *   map's areaWeight, float sums like the reference), Q (1/A) = 4 pi / lambda sin(theta)
 * (the caked output header of IntegratorFitPeaksGPUStream.cu:817-899).  r_lo/r_hi and
 * eta_lo/eta_hi are the bin edges (host, n_r and n_eta).  Panel plans sum the panels'
 * areas. */
#define MI_BIN_NCOL 5
int mi_plan_bin_table(const mi_plan *plan, const double *r_lo, const double *r_hi,
                      const double *eta_lo, const double *eta_hi, double px_um,
                      double lsd_um, double wavelength_a, double *table);

/* ---- peak fitting ----------------------------------------------------------
 * One warp per (frame, peak) window; Levenberg-Marquardt in FP32 with an FP64
 * normal-equation Cholesky solve.  Models:
 *   MI_FIT_PV  : I(x) = bg0 + bg1*xn + h*[eta*L(x) + (1-eta)*G(x)], FWHM shared, 6 params
 *                (center, height, fwhm, eta, bg0, bg1); xn = 2(x-x_lo)/(x_hi-x_lo)-1
 *   MI_FIT_TCH : area-normalised TCH pseudo-Voigt + 2-term Chebyshev background,
 *                params (area, center, sig, gam, bg0, bg1) as pf_calculate_model
 *                (FF_HEDM/src/PeakFit.c:50-92)
 * Output per (frame, peak): MI_FIT_NOUT doubles
 *   [area, center, sig, gam, fwhm, eta, chi2_dof, height, bg0, bg1, two_theta_deg]
 * (first seven exactly the PF_PARAMS_PER_PEAK layout of PeakFit.h). */
#define MI_FIT_PV 0
#define MI_FIT_TCH 1
#define MI_FIT_NOUT 11

typedef struct {
  int32_t model;        /* MI_FIT_*                                       */
  int32_t half_window;  /* samples each side of the peak bin (FitROIPadding) */
  int32_t max_iter;     /* LM iteration cap                                */
  double x_bin;         /* x bin size (same units as x)                    */
  double px_um;         /* pixel size (um) for the 2-theta conversion; 0 = skip */
  double lsd_um;        /* sample-detector distance (um)                   */
} mi_fit_opts;

/* x: device [n_x] (R bin centres), lineouts: device [F][n_x], peaks: device [n_peaks]
 * target x positions; out: device [F][n_peaks][MI_FIT_NOUT]; iters: device [F][n_peaks]
 * int32 (negative = rejected window).  */
int mi_fit_batch(const double *x, const double *lineouts, int n_frames, int n_x,
                 const double *peaks, int n_peaks, const mi_fit_opts *opts,
                 double *out, int32_t *iters, void *stream);

/* ---- fit plans: multi-peak fit jobs ---------------------------------------
 * A fit plan fixes the reference's fit jobs once per (x axis, peak list, options) and
 * fits every job of every series of a batch in one launch (one warp per series;
 * Levenberg-Marquardt with the step projected onto the reference's box bounds, FP32
 * model and Jacobian, FP64 normal equations and Cholesky solve).
 *   MI_FIT_KIND_PEAKS <- fitPeaks()  FF_HEDM/src/PeakFit.c:275-545 and fit_peaks()
 *                        packages/midas_integrate/midas_integrate/peakfit.py:334: nearest
 *                        bin per peak (kept when closer than 2 x_bin), ROI = bin +-
 *                        half_window, overlapping ROIs merged into one joint job (at most
 *                        MI_FIT_JOB_MAX_PEAKS peaks; a longer overlapping run starts a new
 *                        job), area-normalised TCH pseudo-Voigt per peak + bg0 + bg1 * xn.
 *   MI_FIT_KIND_ETA   <- the per-eta-bin fits of FF_HEDM/src/IntegratorZarrOMP.c:1902-2030
 *                        (pf_fit_single_peak / pf_fit_doublet_peak, PeakFit.c:1174-1195, PV
 *                        mode): series with fewer than 5 nonzero samples are skipped; each
 *                        peak, or each pair of adjacent peaks closer than doublet_sep, is
 *                        fit on the bins whose centre lies within half_window bins of it;
 *                        height-normalised pseudo-Voigt, one mixing, flat background.
 * Output rows: MI_FIT_NOUT doubles per (series, peak), in the caller's peak order:
 *   PEAKS: [area, center, sig, gam, fwhm, eta, chi2_dof, height, bg0, bg1, two_theta_deg]
 *   ETA:   [0, center, 0, 0, 0, 0, snr, height, bg, 0, two_theta_deg] when snr > 1 (the
 *          reference's per-eta row), else zeros
 * iters per (series, peak): iterations of its job, -1 peak not fit (no nearest bin within
 * 2 x_bin, or no ROI), -2 job with no more samples than parameters, -3 series skipped. */
#define MI_FIT_KIND_PEAKS 0
#define MI_FIT_KIND_ETA 1
#define MI_FIT_JOB_MAX_PEAKS 8

typedef struct {
  int32_t kind;         /* MI_FIT_KIND_*                                              */
  int32_t half_window;  /* ROI padding in bins (FitROIPadding)                        */
  int32_t max_iter;     /* LM iteration cap per job (<= 0: 200)                       */
  int32_t pad;
  double x_bin;         /* bin size of the x axis                                     */
  double doublet_sep;   /* KIND_ETA: adjacent peaks closer than this are one job; 0 = none */
  double px_um;         /* pixel size (um) for the 2-theta column; 0 = skip           */
  double lsd_um;        /* sample-detector distance (um)                              */
} mi_fit_job_opts;

typedef struct mi_fit_plan mi_fit_plan;

/* x: host [n_x] bin centres (ascending), peaks: host [n_peaks] positions.  device < 0 makes
 * a host-only plan (its job table for mi_fit_plan_info / mi_fit_plan_jobs; it cannot run). */
int mi_fit_plan_create(const double *x, int n_x, const double *peaks, int n_peaks,
                       const mi_fit_job_opts *opts, int device, mi_fit_plan **out);
/* jobs formed, peaks placed in a job, most peaks in one job */
int mi_fit_plan_info(const mi_fit_plan *plan, int *n_jobs, int *n_valid, int *max_job_peaks);
/* The job table: jobs [n_jobs][4] = {first sample, last sample, peaks, first entry}, and
 * peak_ids [n_valid] = the caller's index of each entry (either pointer may be NULL). */
int mi_fit_plan_jobs(const mi_fit_plan *plan, int32_t *jobs, int32_t *peak_ids);
/* Fit n_series x n_sub series: sample i of series (f, e) at
 * src + f*ld_series + e*ld_sub + i*ld_x elements (src_dtype MI_DT_F32 or MI_DT_F64, device
 * memory).  Lineouts [F][n_x]: n_sub 1, ld_series n_x, ld_x 1.  Eta columns of a cake
 * [F][n_r][n_eta]: n_sub n_eta, ld_series n_r*n_eta, ld_sub 1, ld_x n_eta.
 * out: device [n_series*n_sub][n_peaks][MI_FIT_NOUT]; iters: device [n_series*n_sub][n_peaks]. */
int mi_fit_plan_run(const mi_fit_plan *plan, const void *src, int src_dtype, int n_series, int n_sub,
                    int64_t ld_series, int64_t ld_sub, int64_t ld_x, double *out, int32_t *iters,
                    void *stream);
void mi_fit_plan_destroy(mi_fit_plan *plan);

/* Automatic peak detection and fit of each lineout: fitPeaksAutoDetect (FF_HEDM/src/
 * PeakFit.c:549-877; the GPU stream's AutoDetectPeaks mode, IntegratorFitPeaksGPUStream.cu:
 * 2606-2629).  SNIP background (snip_iter passes; 0 = none), Savitzky-Golay-smoothed
 * negative second difference, the most prominent candidates at least max(3, 3 x_bin / bin
 * width) bins apart (up to 3 max_peaks), fitPeaks jobs on the background-subtracted profile
 * (TCH, +-roi_padding bins, overlapping ROIs joint), then the reference's quality filter.
 * x: device [n_x] bin centres; lineouts: device [F][n_x]; out: device [F][max_peaks]
 * [MI_FIT_NOUT] (first n_found[f] rows filled, in position order, the rest zero);
 * n_found: device [F] int32.  One block per lineout. */
int mi_fit_autodetect(const double *x, const double *lineouts, int n_frames, int n_x, int max_peaks,
                      double x_bin, int roi_padding, int snip_iter, double px_um, double lsd_um,
                      double *out, int32_t *n_found, void *stream);

/* ---- map building (DetectorMapper on the device) -------------------------- */
typedef struct {
  int32_t ny, nz;
  double px_um;                 /* pixel size (um), square pixels              */
  double lsd_um;                /* sample-detector distance (um)               */
  double bc_y, bc_z;            /* beam centre (px)                            */
  double tx, ty, tz;            /* tilts (deg)                                 */
  double rho_d;                 /* distortion normalisation radius (um)        */
  double p[15];                 /* p0..p14 distortion coefficients             */
  double parallax_um;           /* Parallax key                                */
  int32_t solid_angle;          /* SolidAngleCorrection                        */
  int32_t polarization;         /* PolarizationCorrection                      */
  double pol_fraction;          /* PolarizationFraction                        */
  int32_t sub_pixel_level;      /* SubPixelLevel (1 = no splitting)            */
  double sub_pixel_cardinal_width; /* SubPixelCardinalWidth (deg)              */
  const uint8_t *mask_host;     /* optional ny*nz mask (1 = masked) or NULL    */
} mi_geometry;

typedef struct {
  int32_t n_r, n_eta;
  const double *r_lo, *r_hi;    /* host, n_r R-bin edges (px)                  */
  const double *eta_lo, *eta_hi;/* host, n_eta eta-bin edges (deg)             */
} mi_binning;

typedef struct mi_map mi_map;   /* built map held on the host                  */

/* device >= 0: build on that GPU; device == -1: build on the host cores (OpenMP),
 * same code, used to cross-check the device build.  Entries of a bin are ordered by
 * pixel (y outer, z inner), the serial loop order of mapper_build_map. */
int mi_map_build(const mi_geometry *geom, const mi_binning *bins, int device,
                 mi_map **out);
int mi_map_sizes(const mi_map *map, int64_t *n_records, int64_t *n_bins);
/* Copy out Map.bin records and nMap.bin pairs (host buffers sized by mi_map_sizes). */
int mi_map_copy(const mi_map *map, mi_map_record *records, int32_t *nmap,
                int32_t *bin_mask);
void mi_map_destroy(mi_map *map);

/* ---- synthetic detector frames (test and benchmark input) ------------------ */
typedef struct {
  int32_t ny, nz;
  double bc_y, bc_z;            /* beam centre (px)                                */
  double lsd_um, px_um;         /* geometry used for the ring radii                */
  double ty, tz;                /* tilts (deg) applied to the ring model           */
  int32_t n_rings;
  double ring_r_px[32];         /* ring radii (px)                                 */
  double ring_amp[32];          /* peak heights (counts)                           */
  double fwhm_px, mix_eta;      /* radial pseudo-Voigt shape                       */
  double texture;               /* cos(2 eta) modulation amplitude (0.3 = +-30 %)  */
  double background;            /* flat background (counts)                        */
  double amp_drift;             /* per-frame uniform amplitude drift (0.2 = +-20 %) */
  int32_t n_spots;              /* Gaussian single-crystal spots per frame         */
  double spot_sigma, spot_amp;
  double dark_mean, dark_sigma; /* dark = dark_mean + N(0, dark_sigma)             */
  uint64_t seed;
  int32_t poisson;              /* 1 = Poisson counts, 0 = expected value rounded  */
} mi_synth_desc;

/* Frames first_frame .. first_frame+n_frames-1 of the seeded sweep, written as
 * u16 (dtype MI_DT_U16) or i32 (MI_DT_I32) to a device buffer with frame_stride
 * elements between frames.  Counts include the dark (raw = dark + signal). */
int mi_synth_frames(const mi_synth_desc *desc, int64_t first_frame, int n_frames,
                    int dtype, void *out, int64_t frame_stride, void *stream);
/* The sweep's dark (float, ny*nz), device pointer. */
int mi_synth_dark(const mi_synth_desc *desc, float *out, void *stream);

/* ---- errors ---------------------------------------------------------------- */
/* Message of the last failing call on this thread ("" if none). */
const char *mi_last_error(void);
/* Library version string. */
const char *mi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* MIDAS_B200_H */
