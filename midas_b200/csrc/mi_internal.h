// mi_internal.h -- shared internals of libmidas_b200 (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/midas_b200.h"

namespace mi {

// Bins whose normalising area is at or below this are invalid
// (AREA_THRESHOLD, IntegratorFitPeaksGPUStream.cu and kernels.py:44).
constexpr double kAreaThreshold = 1e-9;

// Largest number of frames one launch of the batched kernel processes; larger
// batches are split into several launches inside mi_integrate_batch.
constexpr int kMaxFramesPerLaunch = 256;

int set_error(int code, const char *fmt, ...);
// cudaMemcpy of a large buffer in 4 MB pieces (pageable host memory on either side).
cudaError_t copy_pieces(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind);
int cuda_error(cudaError_t e, const char *what, const char *file, int line);

#define MI_CUDA(call)                                                         \
  do {                                                                        \
    cudaError_t mi_e_ = (call);                                               \
    if (mi_e_ != cudaSuccess)                                                 \
      return ::mi::cuda_error(mi_e_, #call, __FILE__, __LINE__);              \
  } while (0)

// ---------------------------------------------------------------------------
// Tiled map encoding used by the batched caking kernel.
//
// Bins are R-major (bin = r * n_eta + e).  Rows are grouped into bands of
// `tile_rows` R bins; a band is split along eta into work items (one CTA
// each); an item is covered by staging tiles (rectangles of rows x eta
// columns) whose union of referenced pixels fits in shared memory.
// Each tile is one contiguous, 16-byte aligned blob in device memory that the
// kernel copies to shared memory with one bulk (TMA) copy:
//
//   TileHdr                        32 B
//   uint32 row_ptr[nb + 1]         term offsets per bin (bins row-major in tile)
//   double scale[nb]               result = sum * scale (1/area, 1 or 0)
//   float  lw[nb]                  lineout weight: in-bounds area if > 1e-9 else 0
//   uint32 upix[n_u]               staged pixels (flat detector index), ascending
//   uint16 lcol[nnz]               term -> index into upix
//   float  w[nnz]                  term weight (fp32)
// every array starts on a 16-byte boundary; the blob size is a multiple of 16.
struct TileHdr {
  int32_t nb, nnz, n_u, n_rows, n_cols, r0, e0, row_in_band;
};
static_assert(sizeof(TileHdr) == 32, "TileHdr layout");

struct TileRef {
  uint64_t off;    // byte offset of the blob in the blob arena
  uint32_t bytes;  // blob size (multiple of 16)
  uint32_t pad;
};

struct WorkItem {
  int32_t tile_begin, tile_end;  // tiles [begin, end) in the tile table
  int32_t r0, n_rows;            // rows of the band this item covers
  int32_t slot;                  // lineout partial slot (item index inside band)
  int32_t nnz;                   // total terms (for scheduling)
  int32_t pad0, pad1;
};

struct BlobLayout {
  uint32_t o_rowptr, o_scale, o_lw, o_upix, o_lcol, o_w, bytes;
};

inline uint32_t align16(uint32_t x) { return (x + 15u) & ~15u; }

__host__ __device__ inline void blob_layout(int nb, int nnz, int n_u, uint32_t *o_rowptr,
                                            uint32_t *o_scale, uint32_t *o_lw,
                                            uint32_t *o_upix, uint32_t *o_lcol,
                                            uint32_t *o_w, uint32_t *bytes) {
  auto a16 = [](uint32_t x) { return (x + 15u) & ~15u; };
  uint32_t o = 32;
  *o_rowptr = o; o = a16(o + 4u * (uint32_t)(nb + 1));
  *o_scale = o;  o = a16(o + 8u * (uint32_t)nb);
  *o_lw = o;     o = a16(o + 4u * (uint32_t)nb);
  *o_upix = o;   o = a16(o + 4u * (uint32_t)n_u);
  *o_lcol = o;   o = a16(o + 2u * (uint32_t)nnz);
  *o_w = o;      o = a16(o + 4u * (uint32_t)nnz);
  *bytes = o;
}

constexpr int kRunWarps = 8;          // consumer (compute) warps per CTA of the run kernel
constexpr uint32_t kRunUnitsOff = 32;  // unit and strip tables follow the tile header
constexpr uint32_t kRunUnitsBytes = kRunWarps * 8 + kRunWarps * 4;

// ---------------------------------------------------------------------------
// Run encoding (MI_ENC_RUNS).  A tile is split into strips, one per eta column,
// each strip being the tile's G rows of that column.  Every staged pixel that
// feeds a strip contributes one or more records: a record holds the pixel's
// weights for L consecutive rows starting at row rs (zero where the pixel has no
// term), so one staged value per frame feeds L accumulators held in registers.
// Records of a strip are sorted by rs; rs_ptr[strip][q] is the first record with
// rs >= q (q = 0 .. G-L+1, the last entry being the strip's end).
//
//   TileHdr                          32 B  (nnz field = number of records)
//   uint16 units[kRunWarps][4]       {strip, first record, end record, 0}: the record range
//                                    of each consumer warp; units of a strip are consecutive
//                                    and split the strip's records evenly
//   uint16 strips[kRunWarps][2]      {first unit, number of units} of each strip
//   uint16 rs_ptr[n_cols][G-L+2]
//   double scale[nb]; float lw[nb]   nb = n_rows * n_cols, row-major
//   uint32 upix[n_u]
//   uint16 lcol[n_rec]
//   float  w[n_rec][L]
// every array 16-byte aligned; the blob size is a multiple of 16.
__host__ __device__ inline uint32_t runs_blob_layout(int nb, int n_cols, int n_rec, int n_u, int G, int L,
                                                     uint32_t *o_rsp, uint32_t *o_sc, uint32_t *o_lw,
                                                     uint32_t *o_up, uint32_t *o_lc, uint32_t *o_w) {
  auto a16 = [](uint32_t x) { return (x + 15u) & ~15u; };
  uint32_t o = kRunUnitsOff + kRunUnitsBytes;
  *o_rsp = o; o = a16(o + 2u * (uint32_t)n_cols * (uint32_t)(G - L + 2));
  *o_sc = o;  o = a16(o + 8u * (uint32_t)nb);
  *o_lw = o;  o = a16(o + 4u * (uint32_t)nb);
  *o_up = o;  o = a16(o + 4u * (uint32_t)n_u);
  *o_lc = o;  o = a16(o + 2u * (uint32_t)n_rec);
  *o_w = o;   o = a16(o + 4u * (uint32_t)n_rec * (uint32_t)L);
  return o;
}

constexpr int kRunProducerWarps = 6; // producer (gather) warps per CTA, frame-major staging
constexpr int kRunProducersXc = 2;   // producer warps issuing the copies of pixel-major staging
constexpr int kRunCtasPerSm = 1;
constexpr int kRunPitch = 144;       // bytes per staged pixel: 64 x u16 or 32 x f32, then (u16
                                     // staging) the pixel's dark as f32 at byte 128, pad

// Frames per group of the run kernel: 8/16-bit frames are staged as u16 and, with G <= 16,
// computed two frames per lane (64 per group); otherwise one frame per lane (32).
__host__ __device__ constexpr int runs_frames_per_group(int sizeof_t, int G) {
  return (sizeof_t <= 2 && G <= 16) ? 64 : 32;
}

// Shared memory of the run kernel (two pipeline slots b = 0, 1):
//   [blob b: blob_cap][staging b: u_cap x kRunPitch; after the record loop, the bin
//    results fg x nbp floats]  x 2
//   [unit partials: kRunWarps x G x fg floats][lineout partials: rows x fg x 2 doubles]
//   [4 mbarriers: blob b, staging b]
// Offsets of slot 1 are those of slot 0 plus *slot_bytes.
__host__ __device__ inline uint32_t runs_smem_layout(uint32_t blob_cap, int u_cap, int nbp, int rows, int G, int fg,
                                                     uint32_t *off_val, uint32_t *slot_bytes, uint32_t *off_part,
                                                     uint32_t *off_lo, uint32_t *off_bar) {
  auto a16 = [](uint32_t x) { return (x + 15u) & ~15u; };
  const uint32_t ov = a16(blob_cap);                        // staging area of slot 0
  uint32_t stage = (uint32_t)u_cap * (uint32_t)kRunPitch;
  const uint32_t outb = (uint32_t)fg * (uint32_t)nbp * 4u;
  if (outb > stage) stage = outb;
  const uint32_t slot = a16(ov + stage);                    // [blob | staging] of one slot
  const uint32_t op = 2u * slot;
  const uint32_t ol = a16(op + (uint32_t)kRunWarps * (uint32_t)G * (uint32_t)fg * 4u);
  const uint32_t ob = a16(ol + (uint32_t)fg * (uint32_t)rows * 2u * 8u);
  if (off_val) *off_val = ov;
  if (slot_bytes) *slot_bytes = slot;
  if (off_part) *off_part = op;
  if (off_lo) *off_lo = ol;
  if (off_bar) *off_bar = ob;
  return ob + 32u;
}

// Shared-memory layout of the batched kernel for `fpl` frames per lane:
// [2 blob buffers][staged values: u_cap x 33*fpl floats][bin results: 32*fpl x nbp floats]
// [lineout partials: 32*fpl x rows x 2 doubles][2 mbarriers]; returns the total bytes.
__host__ __device__ inline uint32_t cake_smem_layout(int fpl, uint32_t blob_cap, int u_cap, int nbp,
                                                     int rows, uint32_t *off_val, uint32_t *off_out,
                                                     uint32_t *off_lo, uint32_t *off_bar) {
  auto a16 = [](uint32_t x) { return (x + 15u) & ~15u; };
  const uint32_t ov = a16(2u * blob_cap);
  const uint32_t oo = a16(ov + (uint32_t)u_cap * 33u * (uint32_t)fpl * 4u);
  const uint32_t ol = a16(oo + 32u * (uint32_t)fpl * (uint32_t)nbp * 4u);
  const uint32_t ob = a16(ol + 32u * (uint32_t)fpl * (uint32_t)rows * 2u * 8u);
  if (off_val) *off_val = ov;
  if (off_out) *off_out = oo;
  if (off_lo) *off_lo = ol;
  if (off_bar) *off_bar = ob;
  return ob + 16u;
}

// Host-side CSR of one integration mode: rows = bins, cols = flat pixels.
struct HostCSR {
  std::vector<int64_t> row_ptr;  // n_bins + 1
  std::vector<int32_t> col;
  std::vector<double> w;
  std::vector<double> area_norm;  // normaliser per bin (semantics dependent)
  std::vector<double> area_in;    // in-bounds area per bin (profile weights)
  std::vector<double> area_gs;    // area of records with 0 <= y < ny, 0 <= z < nz (as floats)
  int64_t oob = 0;
};

struct TileLimits {
  int rows;      // rows per band
  int max_u;     // max staged pixels per tile
  int max_nb;    // max bins per tile
  int max_nnz;   // max terms per tile
  int max_cols;  // max eta columns per tile
  int item_cols; // eta columns per work item
};

// Pixel-major staging for the run kernel.  The referenced pixels of each detector row
// are covered by one span [span_lo, span_lo + len) with both ends on 8-pixel boundaries
// (len may end at ny when ny is not a multiple of 8); the spans, concatenated row by row,
// give the compact pixel index c.  Kernel (a) writes kXcRowBytes per compact pixel:
// 8/16-bit frames as u16 (128 frames, groups of 64), other frame types as fp32 with the
// dark already subtracted (64 frames, groups of 32), so a tile stages each of its pixels,
// one frame group at a time, with one 128-byte bulk copy.  Transpose work is cut into
// chunks of <= kXcChunk pixels of one span.
constexpr int kXcFrames = 64;      // u16 frames of one group (one 128-byte staged row)
constexpr int kXcGroups = 2;       // u16 groups held per launch
constexpr int kXcFramesF = 32;     // fp32 frames of one group
constexpr int kXcGroupsF = 2;      // fp32 groups held per launch
constexpr int kXcRowBytes = 256;   // bytes per compact pixel
constexpr int kXcChunk = 256;
constexpr int kUploadRows = 16;   // detector rows per column range of mi_upload_frames
struct XcChunk {
  int32_t z, y0, n, c0;  // detector row, first column, pixels, compact index of the first
};

// ---------------------------------------------------------------------------
// MMA encoding (MI_ENC_MMA, kernel k_mma of mi_mma.cu): caking of 8/16-bit frames on the
// tensor cores with exact integer arithmetic.  A tile is kMmaRows x kMmaCols bins (bin
// n = row * kMmaCols + col) and its staged pixels in K slots; a frame batch is the M = 128
// rows of the MMA.  Frames are split into two u8 byte planes (lo, hi), weights into four
// s8 digit planes of a signed fixed-point value q = round(w / max|w|(bin) * kMmaQMax) (see
// mma_digits); the eight u8 x s8 products accumulate exactly in int32 (five accumulators,
// one per byte shift 0..4), and the epilogue recombines them in FP64:
//   cake = fac * sum_k 2^(8k) acc_k - dk,  fac = max|w| / kMmaQMax * scale,
//   dk = fac * sum q * dark (the dark term of the bin, set with the dark).
// The pixel-major buffer of an MMA plan holds two byte planes, [lo: n_xc x 128][hi: n_xc x
// 128]: row c of a plane is compact pixel c's byte of 128 frames, its 16-byte granule g
// (frames 16g .. 16g+15) at position g ^ (c % 8).
// Blob of a tile (16-byte aligned arrays):
//   MmaHdr                              32 B
//   double fac[48], dk[48]; float lw[48]  per bin n of the tile (zeros for bins outside it);
//                                       dk is written by the dark kernel when a dark is set
//   uint2  runs[n_runs]                 {c, k0 | len << 8}: len consecutive K slots k0.. of a
//                                       step staged from pixel-major rows c.. (one bulk copy
//                                       per byte plane); slot k holds a pixel with
//                                       c % 8 == k % 8 (the swizzle phase of its row)
//   uint32 run_ptr[n_k + 1]             runs of K step s: [run_ptr[s], run_ptr[s+1])
//   uint32 step_ptr[n_k + 1]            words of K step s
//   uint4  wpl[n_words]                 a bin's weights in four consecutive K slots 4w .. 4w+3
//                                       of a step: one 32-bit word per digit plane (plane j
//                                       in .x/.y/.z/.w, slot 4w + b in byte b; 0 where the bin
//                                       has no term)
//   uint16 widx[n_words]                w (0..7, within the step) | n << 3, words sorted by
//                                       step (n_terms of the header counts the words)
struct MmaHdr {
  int32_t n_rows, n_cols, r0, e0, n_k, n_terms;
  int32_t box_rows;   // rows of the item's sub-band (12, 6, 3 or 1): the cake store's box height
  int32_t n_runs;
};
static_assert(sizeof(MmaHdr) == 32, "MmaHdr layout");
constexpr int kMmaRows = 12;           // R rows per tile
constexpr int kMmaCols = 4;            // eta columns per tile (one 16-byte cake segment)
constexpr int kMmaN = kMmaRows * kMmaCols;  // 48 bins: the N of every MMA
constexpr int kMmaFrames = 128;        // frames per launch: the M of every MMA
constexpr int kMmaKStep = 32;          // K slots (staged pixels) per MMA step
constexpr uint32_t kMmaEmpty = 0xFFFFFFFFu;
constexpr int kMmaDarkWarps = 8;       // warps of the dark-term kernels (48 bins: 6 per warp)
constexpr int kMmaMaxBinTerms = 16000; // int32 accumulators: 2 x 255 x 128 per term
// Tensor-core weights: q = round(w / max|w|(bin) x kMmaQMax), |q| <= kMmaQMax, written as four
// balanced base-256 digits d_k in [-128, 127] (q = sum_k 256^k d_k), one s8 byte plane each:
// bilinear weights of the IntegrationCore semantics can be negative.  127 x (1 + 2^8 + 2^16 +
// 2^24) is the largest magnitude the four digits hold either way.
constexpr double kMmaQMax = 2139062143.0;
// the digits packed one per byte (two's complement), plane k in byte k
__host__ __device__ inline uint32_t mma_digits(int64_t q) {
  uint32_t packed = 0;
  for (int k = 0; k < 4; ++k) {
    const int64_t d = ((q % 256) + 384) % 256 - 128;   // q - d divisible by 256, d in [-128, 127]
    packed |= (uint32_t)(uint8_t)(int8_t)d << (8 * k);
    q = (q - d) / 256;
  }
  return packed;
}
// Shared-memory bank of a term's byte in the B operand of one K step (byte (n, k) at
// (n % 8) * 16 + (n / 8) * 256 + (k % 16) + (k / 16) * 128, the plane offsets multiples of 128)
__host__ __device__ inline int mma_bank(uint32_t n, uint32_t kk) {
  return (int)((n & 7u) * 4u + ((kk & 15u) >> 2));
}
__host__ __device__ inline int64_t mma_digits_value(uint32_t packed) {
  int64_t q = 0;
  for (int k = 3; k >= 0; --k) q = q * 256 + (int8_t)(uint8_t)(packed >> (8 * k));
  return q;
}
constexpr uint32_t kMmaBlobCap = 28 * 1024;  // largest tile blob (blob slots in shared memory)
constexpr uint32_t kMmaBinsOff = 32;   // fac, dk, lw after the header
constexpr uint32_t kMmaBinsBytes = kMmaN * (8 + 8 + 4);

struct MmaBlob {
  uint32_t runs, run_ptr, step_ptr, wpl, widx, bytes;
};
__host__ __device__ inline MmaBlob mma_blob_layout(int n_k, int n_runs, int n_words) {
  auto a16 = [](uint32_t x) { return (x + 15u) & ~15u; };
  MmaBlob b;
  uint32_t o = a16(kMmaBinsOff + kMmaBinsBytes);
  b.runs = o;     o = a16(o + 8u * (uint32_t)n_runs);
  b.run_ptr = o;  o = a16(o + 4u * (uint32_t)(n_k + 1));
  b.step_ptr = o; o = a16(o + 4u * (uint32_t)(n_k + 1));
  b.wpl = o;      o = a16(o + 16u * (uint32_t)n_words);
  b.widx = o;     o = a16(o + 2u * (uint32_t)n_words);
  b.bytes = o;
  return b;
}

// Direct MMA encoding (MI_ENC_MMAD, kernel k_mmad of mi_mmad.cu): the tiles, bins and
// epilogue of the MMA encoding, with the frames read by the kernel straight from their
// frame-major layout (no pixel-major buffer).  A tile's pixels are covered by 8-pixel
// granules (8 consecutive pixels of one detector row, the first at a multiple of 8); a K
// step of 32 slots is four granules, slot k holding pixel k % 8 of granule k / 8.  The
// producer warps load a frame's granule with one 16-byte load per frame (u16 frames), split
// it into its low and high byte planes and store both into tensor memory, where they are
// the A operand of the MMAs.  Weights are the MMA encoding's signed fixed point (kMmaQMax),
// four s8 digit planes (the B operand, N = 192), so five int32 accumulators (byte shifts
// 0..4) hold the exact products:
//   cake = fac * sum_k 2^(8k) acc_k - dk,  fac = max|w| / kMmaQMax * scale.
// Blob of a tile (16-byte aligned arrays):
//   MmaHdr                       32 B (n_runs: 0)
//   double fac[48], dk[48]; float lw[48]
//   uint32 gran[n_k][4]          granule z | y0 << 16 (kMmadEmpty: none)
//   uint32 step_ptr[n_k + 1]     terms of K step s
//   uint2  terms[n_terms]        {mma_digits(q), k | n << 16}, sorted by slot k (k / 32 = K step)
constexpr int kMmadGran = 4;           // granules per K step
constexpr int kMmadGranPx = 8;         // pixels per granule
constexpr uint32_t kMmadEmpty = 0xFFFFFFFFu;

struct MmadBlob {
  uint32_t gran, step_ptr, terms, bytes;
};
__host__ __device__ inline MmadBlob mmad_blob_layout(int n_k, int n_terms) {
  auto a16 = [](uint32_t x) { return (x + 15u) & ~15u; };
  MmadBlob b;
  uint32_t o = a16(kMmaBinsOff + kMmaBinsBytes);
  b.gran = o;     o = a16(o + 4u * kMmadGran * (uint32_t)n_k);
  b.step_ptr = o; o = a16(o + 4u * (uint32_t)(n_k + 1));
  b.terms = o;    o = a16(o + 8u * (uint32_t)n_terms);
  b.bytes = o;
  return b;
}

struct Plan {
  int device = 0;
  int mode = 0, normalize = 1, semantics = 0;
  int variance = 0;              // squared weights, area^2 normalisation, variance lineouts
  std::vector<double> area_gs;   // per bin, for mi_plan_bin_table
  int n_r = 0, n_eta = 0, ny = 0, nz = 0;
  double bc_y = 0, bc_z = 0;
  int64_t n_bins = 0, nnz = 0, n_records = 0, oob = 0;
  int frames_per_lane = 1;
  int encoding = MI_ENC_RUNS;
  int run_g = 0, run_l = 0;      // run encoding: rows per strip (8/16/32), rows per record
  TileLimits lim{};
  int64_t staged_pixels = 0, ref_pixels = 0;
  int ref_row_lo = 0, ref_row_hi = 0;   // detector rows holding referenced pixels
  // host -> device upload of frames (mi_upload_frames): per group of kUploadRows detector
  // rows, the columns any of its rows references, rounded out to 8 pixels as the transpose
  // reads them: {first row, end row, first column, end column}
  std::vector<int4> upload_groups;

  // batched path
  uint8_t *d_blobs = nullptr;
  size_t blob_bytes = 0;
  TileRef *d_tiles = nullptr;
  int n_tiles = 0;
  WorkItem *d_items = nullptr;   // in launch order (heaviest first)
  int n_items = 0;
  int n_slots = 0;               // work items per band
  uint32_t max_blob = 0;         // largest blob (bytes)
  int max_u = 0, max_nb = 0;     // realised maxima over tiles
  double *d_den_aw = nullptr;    // per R row: sum of valid in-bounds area
  double *d_cnt = nullptr;       // per R row: number of valid bins
  double *d_partial = nullptr;   // [kMaxFramesPerLaunch][n_r][n_slots][2]
  int32_t *d_nan_bins = nullptr; // MI_SEM_OMP: bins written as NaN (the plan's bin mask)
  int n_nan_bins = 0;
  float *d_dark = nullptr;       // ny*nz (zeros when no dark is set)
  int has_dark = 0;
  int *d_err = nullptr;          // device error word (bounded waits)
  int *d_ctr = nullptr;          // work-item counter of the persistent run kernel
  int n_sms = 0;
  int mma_stages = 8, mma_producers = 6;   // pipeline of the MMA kernel (mi_plan_set_mma_pipeline)

  // pixel-major staging (run encoding with 64-frame groups)
  int64_t n_xc = 0;              // compact pixels (0: not built)
  int32_t *d_span_lo = nullptr;  // per detector row: first column of its span
  int32_t *d_row_off = nullptr;  // per detector row: compact index of the span start
  XcChunk *d_xchunks = nullptr;
  int n_xchunks = 0;
  uint8_t *d_xc = nullptr;       // [n_xc][kXcRowBytes]
  int32_t *d_xc_pix = nullptr;   // MMA encoding: virtual pixel of each compact index

  // panels (a plan over several detectors sharing one binning): panel p's rows are rows
  // [z_off, z_off + nz) of a virtual detector ny pixels wide (ny = the widest panel)
  struct Panel {
    int ny, nz, z_off;
    int chunk_begin, chunk_end;  // its transpose chunks
  };
  std::vector<Panel> panels;     // one entry for an ordinary plan

  // plain (reference-layout) path
  int32_t *d_nmap = nullptr;     // {count, offset} per bin
  int32_t *d_sorted = nullptr;   // bins, heaviest first
  int32_t *d_off = nullptr;      // per record: flat pixel offset (floor mode)
  float *d_w = nullptr, *d_aw = nullptr, *d_dr = nullptr, *d_py = nullptr, *d_pz = nullptr;
  double *d_area_in = nullptr;   // per bin in-bounds area
  double *d_area_all = nullptr;  // per bin sum of all areaWeight
  float *d_plain_img = nullptr;  // one cast frame
  size_t device_bytes = 0;
};

// Builders (mi_plan.cu)
int build_host_csr(const mi_map_desc &m, int mode, int semantics, HostCSR *out);

// Launchers (mi_cake.cu, mi_plain.cu)
// `partial` is the lineout scratch, [n_frames][n_r][n_slots][2] doubles (the plan's d_partial,
// or a caller-provided array of that size)
int launch_cake(Plan *p, const void *frames, int dtype, int n_frames, int64_t stride,
                float *cake, double *lo_aw, double *lo_sm, double *partial, cudaStream_t s);
int launch_runs(Plan *p, const void *frames, int dtype, int n_frames, int64_t stride, float *cake, double *partial,
                bool want_lo, cudaStream_t s);
// true when launch_runs stages this dtype through the pixel-major buffer
bool runs_uses_xc(const Plan *p, int dtype);
// Transpose frames [0, F) of panel `panel` into the pixel-major buffer: u16 rows when
// `as_f32` is false (8/16-bit frames, F <= 128), else fp32 rows minus the dark (F <= 64).
int launch_xc(Plan *p, int panel, const void *frames, int dtype, int F, int64_t stride, bool as_f32,
              cudaStream_t s);
// Caking of frames [0, F) (F <= 128 u16 / 64 fp32) already staged pixel-major.
int launch_runs_staged(Plan *p, bool as_f32, int F, float *cake, double *partial, bool want_lo, cudaStream_t s);
// MMA encoding (mi_mma.cu): caking of frames [0, F) (F <= 128) staged as byte planes, and
// the per-bin dark terms (after a dark is set)
int launch_mma(Plan *p, int F, float *cake, double *partial, bool want_lo, cudaStream_t s);
bool mma_pipeline_supported(int stages, int producers);
int launch_mma_dark(Plan *p, cudaStream_t s);
// Direct MMA encoding (mi_mmad.cu): caking of frames [0, F) (F <= 128, u16 or u8) read in
// place at frames + f * stride, and the per-bin dark terms
int launch_mmad(Plan *p, const void *frames, int dtype, int F, int64_t stride, float *cake, double *partial,
                bool want_lo, cudaStream_t s);
int launch_mmad_dark(Plan *p, cudaStream_t s);
// kernel (c): lineouts of frames [0, n_frames) from the partial sums in `partial`
int launch_lineout(Plan *p, const double *partial, int n_frames, double *lo_aw, double *lo_sm, cudaStream_t s);
int launch_plain(Plan *p, const void *frame, int dtype, double *cake, double *lo_aw,
                 double *lo_sm, cudaStream_t s);
int launch_cast(const void *frames, int dtype, int64_t n_pixels, int n_frames,
                const float *dark, float *out, cudaStream_t s);
int launch_profile(Plan *p, const void *cake, int cake_dtype, int n_frames, double *lo_aw,
                   double *lo_sm, cudaStream_t s);
// MI_SEM_OMP plans: NaN into the masked bins of F cakes
int launch_nan_bins(Plan *p, float *cake, int n_frames, cudaStream_t s);
int launch_sum_cake(Plan *p, const float *cake, int n_frames, double *sum, cudaStream_t s);

size_t dtype_size(int dtype);

}  // namespace mi
