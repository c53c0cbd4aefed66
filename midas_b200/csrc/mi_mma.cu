// mi_mma.cu -- kernel (b), MMA encoding: batched caking on the tensor cores (tcgen05, int8).
//
// Same contract as the run kernel (integrate() of packages/midas_integrate/midas_integrate/
// kernels.py:416-473, integrate_noMapMask of FF_HEDM/src/IntegratorFitPeaksGPUStream.cu:
// 975-1050): cake = diag(scale) W (frames - dark) plus the eta partial sums of both
// lineouts, here for batches of up to 128 frames of 8/16-bit pixels.
//
// A tile (kMmaRows x kMmaCols = 48 bins) is a dense int8 product on the tensor cores:
//   D[frame][bin] (int32, TMEM) += A[frame][pixel] (a byte plane of the frames)
//                                  x B[pixel][bin] (a byte plane of the weights q)
// two frame planes x four weight planes, issued as two tcgen05.mma of N = 192 per K step of
// 32 staged pixels, into five int32 accumulators (one per byte shift 0..4).  Every product and sum is exact;
// the epilogue forms sum_k 2^(8k) acc_k in FP64, subtracts the bin's dark term and scales:
// cake = fac * value - dk.  The only approximation is the signed fixed-point weight (four s8
// digits, a step of 2^-31 of the bin's largest |w|); the reference's fp32 (raw - dark) and
// fp32 sums are replaced by exact integer sums, so the result is closer to the FP64 one.
//
// Operands in shared memory, per pipeline stage (kMmaStepsPerStage K steps of 32 pixel slots):
//   A (frames): MN-major, 128B swizzle; slot k of the stage is the 128-byte row
//     (k % 8) * 128 + (k / 8) * 1024 holding the pixel's 128 frame bytes, 16-byte granule g
//     at position g ^ (k % 8).  Kernel (a) writes each pixel-major row with its granules
//     already in that order for phase c % 8, and the tiler puts pixel c in a slot with
//     k % 8 == c % 8, so a slot is filled by one plain 128-byte bulk copy per plane.
//   B (weights): K-major, no swizzle, the four s8 digit planes as rows n' = 48 j + n; byte
//     (n', k) at (n' % 8) * 16 + (n' / 8) * kMmaBSbo + (k % 16) + (k / 16) * 128, zeroed and
//     then scattered from the stage's terms (the tiler orders a step's terms so that each
//     32 consecutive ones fall in distinct banks where the step allows: mma_bank).
//
// Roles (one persistent CTA per SM, 16 warps with the default 6 producers):
//   warp 0          TMEM allocation (512 columns: two accumulator sets of 5 x 48) and, on one
//                   lane, the MMA issue: 2 MMAs per K step, a commit that frees the stage, and
//                   at a tile's last step a commit that hands the accumulators to the epilogue
//   warp 1          loader: claims work items (heaviest first) and brings each tile's blob
//                   into one of its blob slots with one bulk copy
//   warps 2,3,12.. producers: stage g (counted over the CTA's tiles) is built by producer
//                   g % producers into stage slot g % stages
//   warps 4-11      epilogue: warp w reads TMEM lanes 32 (w % 4) + 0..31 (= frames) and half
//                   of the tile's bins (8 bins x 5 accumulators at a time), recombines, puts the
//                   cake values into a shared-memory image holding two adjacent tiles of the
//                   item (8 columns: 32-byte rows, whole sectors) that one TMA tensor store
//                   writes to the [F][n_r][n_eta] cake, and accumulates the lineout
//                   partial sums of the item's rows in registers (a frame's result does not
//                   depend on the rest of its batch)
// Every wait is an mbarrier poll with an iteration limit; on expiry the kernel sets the
// plan's error word (MI_E_TIMEOUT) and the role leaves its loop.
#include <cuda.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>

#include "mi_internal.h"
#include "mi_tc.cuh"

namespace mi {

// Pipeline depth: the kernel is compiled for a few (stages, producer warps) pairs, chosen per
// plan at launch (mi_plan_set_mma_pipeline; the autotuner times them); 8 stages and 6
// producers by default.  A producer waits for its stage slot by the parity of the slot's
// empty barrier, which is sound only while the barrier is at most one phase behind the
// waiter.  The producer of stage g has seen stage g - producers - stages consumed; stage
// g - 2 stages must be: producers <= stages.
constexpr int kMmaStepsPerStage = 1;   // K steps (32 pixel slots each) per stage
constexpr int kMmaEpiWarps = 8;
__host__ __device__ constexpr int mma_threads(int producers) { return (2 + producers + kMmaEpiWarps) * 32; }
// per stage: A lo 4096 | A hi 4096 | B 6144 per K step
constexpr uint32_t kMmaStageBytes = 14336u * kMmaStepsPerStage;
constexpr uint32_t kMmaAHi = 4096u * kMmaStepsPerStage, kMmaB = 8192u * kMmaStepsPerStage;
constexpr uint32_t kMmaBPlane = 1536u * kMmaStepsPerStage;   // 48 rows of the K-major weight operand
constexpr uint32_t kMmaBSbo = 256u * kMmaStepsPerStage;      // bytes per 8-row group of that operand
constexpr int kMmaBlobSlotsMax = 4;
constexpr int kMmaFacSlots = 6;             // ring of the tiles' per-bin factors (epilogue)
constexpr uint32_t kMmaFacBytes = 1024;      // one ring entry: fac, dk, lw of 48 bins (960 B)
constexpr int kMmaTmemCols = 512;
constexpr int kMmaAccCols = 256;            // columns per accumulator set (5 x 48 used)
constexpr uint32_t kMmaOutBytes = kMmaFrames * kMmaN * 4;   // one cake tile: [128][rows][4] floats
// The epilogue stores two adjacent tiles of an item (8 columns) with one box: 32-byte rows

struct MmaArgs {
  CUtensorMap tmap[kCakeBoxes];  // the call's cake as (n_eta, F, n_r) floats (encode_cake_boxes)
  const WorkItem *items;
  const TileRef *tiles;
  const uint8_t *blobs;
  const uint8_t *xc_lo, *xc_hi;   // pixel-major byte planes, 128 bytes per compact pixel
  float *cake;
  double *partial;          // [F][n_r][n_slots][2]
  int F, n_r, n_eta, n_slots;
  int64_t n_bins;
  int want_cake, want_lo, use_tma;
  int n_items;
  int *counter;
  int *err;
  uint32_t blob_cap;
  int n_blob;               // blob slots (2 to 4, as shared memory allows)
};

// Per-slot and per-stage tags passed between the roles through shared memory.
struct MmaTag {
  int32_t end, tile, step, n_k;     // end of work; tile sequence number of the CTA; stage of the
                                    // tile; K steps of the tile (the MMA lane reads these 16 B)
  int32_t slot, first, last, box;   // item's lineout slot; first/last tile of item; box rows
  int32_t r0, n_rows, e0, n_cols;   // the tile's bins
  int32_t pos, pad0, pad1, pad2;    // index of the tile in its item
};

struct MmaSmem {
  uint32_t off_out, off_blob, off_fac, off_shdr, off_btag, off_atag, off_bar, off_tmem, total;
};

__host__ __device__ inline MmaSmem mma_smem_layout(uint32_t blob_cap, int n_blob, int stages) {
  MmaSmem L;
  uint32_t o = (uint32_t)stages * kMmaStageBytes;
  L.off_out = o;   o += 2u * kMmaOutBytes;
  L.off_blob = o;  o += (uint32_t)n_blob * blob_cap;
  L.off_fac = o;   o += (uint32_t)kMmaFacSlots * kMmaFacBytes;
  L.off_shdr = o;  o += (uint32_t)stages * sizeof(MmaTag);
  L.off_btag = o;  o += (uint32_t)kMmaBlobSlotsMax * sizeof(MmaTag);
  L.off_atag = o;  o += 2u * sizeof(MmaTag);
  L.off_bar = o;   o += 8u * (2u * stages + 2u * kMmaBlobSlotsMax + 2u * kMmaFacSlots + 4u);
  L.off_tmem = o;  o += 16u;
  L.total = o + 1024u;   // the base is rounded up to 1024 bytes inside the kernel
  return L;
}

// instruction descriptor, kind::i8: D s32, A u8 MN-major, B s8 K-major, M = 128, N = 48
// with N = 192 (the four weight planes, 48 bins each, side by side), 144 (planes 0-2) or 48
__host__ __device__ constexpr uint32_t mma_idesc(int n) {
  return (2u << 4) | (1u << 10) | (1u << 15) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kMmaFrames >> 4) << 24);
}

__device__ __forceinline__ void m_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                      uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
template <int kMmaStages, int kMmaProducers>
__global__ void __launch_bounds__(mma_threads(kMmaProducers), 1) k_mma(const __grid_constant__ MmaArgs a) {
  static_assert(kMmaProducers <= kMmaStages, "more producers than stage slots aliases barrier phases");
  extern __shared__ uint8_t smem_raw[];
  // 1024-byte aligned base: the swizzled A operand's atoms start on 1024-byte boundaries
  const uint32_t raw = m_smem(smem_raw);
  uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  const MmaSmem L = mma_smem_layout(a.blob_cap, a.n_blob, kMmaStages);
  const int NB = a.n_blob;
  MmaTag *s_shdr = (MmaTag *)(smem + L.off_shdr);
  MmaTag *s_btag = (MmaTag *)(smem + L.off_btag);
  MmaTag *s_atag = (MmaTag *)(smem + L.off_atag);
  uint64_t *bar = (uint64_t *)(smem + L.off_bar);
  uint64_t *full = bar, *empty = bar + kMmaStages;
  uint64_t *bfull = bar + 2 * kMmaStages, *bempty = bfull + kMmaBlobSlotsMax;
  uint64_t *afull = bempty + kMmaBlobSlotsMax, *aempty = afull + 2;
  uint64_t *ffull = aempty + 2, *fempty = ffull + kMmaFacSlots;
  uint32_t *s_tmem = (uint32_t *)(smem + L.off_tmem);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    for (int q = 0; q < kMmaStages; ++q) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(m_smem(&full[q])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(m_smem(&empty[q])) : "memory");
    }
    for (int q = 0; q < kMmaBlobSlotsMax; ++q) {
      // a blob slot is free again when the producers have built its stages
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(m_smem(&bfull[q])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(m_smem(&bempty[q])), "r"(kMmaProducers)
                   : "memory");
    }
    for (int q = 0; q < kMmaFacSlots; ++q) {
      // a factor entry is free again when every epilogue warp has used it
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(m_smem(&ffull[q])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(m_smem(&fempty[q])), "r"(kMmaEpiWarps)
                   : "memory");
    }
    for (int q = 0; q < 2; ++q) {
      // two arrivals: the MMA lane's (after it wrote the set's tag) and the commit of the
      // tile's last MMAs
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;" ::"r"(m_smem(&afull[q])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(m_smem(&aempty[q])), "r"(kMmaEpiWarps)
                   : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(m_smem(s_tmem)),
                 "r"(kMmaTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  m_fence_before();
  __syncthreads();
  m_fence_after();
  const uint32_t tmem = *s_tmem;

  if (warp == 0) {
    // ================= MMA issue (one lane)
    if (lane == 0) {
      bool ok = true;
      // the stages of a tile arrive in order, so the lane counts them itself and reads a stage
      // tag only at a tile's first stage (or the end marker): shared memory is busy with the
      // producers' and the epilogue's traffic, and a read on this serial path costs every stage
      int st = 0, n_st = 0, nk = 0, ab = 0;
      for (uint32_t g = 0;; ++g) {
        const int q = (int)(g % kMmaStages);
        if (!m_wait(&full[q], (g / kMmaStages) & 1u)) { ok = false; break; }
        if (st == n_st) {
          const int4 hq = *(const int4 *)&s_shdr[q];   // end, tile, step, n_k
          ab = hq.y & 1;
          if (hq.x) {
            // no more tiles: pass the end marker to the epilogue through the next set
            if (!m_wait(&aempty[ab], ((uint32_t)(hq.y >> 1) & 1u) ^ 1u)) { ok = false; break; }
            s_atag[ab] = s_shdr[q];
            m_arrive(&afull[ab]);
            m_arrive(&afull[ab]);
            break;
          }
          nk = hq.w;
          n_st = (nk + kMmaStepsPerStage - 1) / kMmaStepsPerStage;
          st = 0;
          if (!m_wait(&aempty[ab], ((uint32_t)(hq.y >> 1) & 1u) ^ 1u)) { ok = false; break; }
          m_fence_after();
          s_atag[ab] = s_shdr[q];
          m_arrive(&afull[ab]);
        }
        const uint32_t sb = m_smem(smem + (size_t)q * kMmaStageBytes);
        const uint32_t dbase = tmem + (uint32_t)(ab * kMmaAccCols);
        // the four weight planes are one N = 192 operand (plane j = rows 48 j ..): the low
        // frame plane's product lands on accumulators 0-3 (columns 0..191), the high plane's,
        // one byte up, on accumulators 1-4 (columns 48..239).  At a tile's first K step the
        // first product into each accumulator starts it from zero, so the high plane's
        // product is split there into planes 0-2 (accumulate) and plane 3 (fresh).
#pragma unroll
        for (int hs = 0; hs < kMmaStepsPerStage; ++hs) {
          if (kMmaStepsPerStage * st + hs >= nk) break;
          const uint64_t alo = m_desc(sb + 4096u * hs, 0u, 1024u, 2u);
          const uint64_t ahi = m_desc(sb + kMmaAHi + 4096u * hs, 0u, 1024u, 2u);
          const uint32_t bsa = sb + kMmaB + 256u * hs;
          const uint64_t bd = m_desc(bsa, 128u, kMmaBSbo, 0u);
          const bool first = st == 0 && hs == 0;
          m_mma(dbase, alo, bd, mma_idesc(4 * kMmaN), first ? 0u : 1u);
          if (!first) {
            m_mma(dbase + (uint32_t)kMmaN, ahi, bd, mma_idesc(4 * kMmaN), 1u);
          } else {
            m_mma(dbase + (uint32_t)kMmaN, ahi, bd, mma_idesc(3 * kMmaN), 1u);
            m_mma(dbase + (uint32_t)(4 * kMmaN), ahi, m_desc(bsa + 3u * kMmaBPlane, 128u, kMmaBSbo, 0u),
                  mma_idesc(kMmaN), 0u);
          }
        }
        m_commit(&empty[q]);
        if (++st == n_st) m_commit(&afull[ab]);
      }
      if (!ok) atomicExch(a.err, MI_E_TIMEOUT);
    }
    __syncwarp();
  } else if (warp == 1) {
    // ================= loader: items -> tile blobs
    int j = 0;
    bool ok = true;
    for (;;) {
      int claimed = 0;
      if (lane == 0) claimed = atomicAdd(a.counter, 1);
      claimed = __shfl_sync(0xffffffffu, claimed, 0);
      if (claimed >= a.n_items) break;
      const WorkItem it = a.items[claimed];
      const int nt = it.tile_end - it.tile_begin;
      for (int t = 0; t < nt && ok; ++t, ++j) {
        const int sl = j % NB;
        if (lane == 0) {
          const TileRef tr = a.tiles[it.tile_begin + t];
          const int fs = j % kMmaFacSlots;
          if (!m_wait(&bempty[sl], ((uint32_t)(j / NB) & 1u) ^ 1u) ||
              !m_wait(&fempty[fs], ((uint32_t)(j / kMmaFacSlots) & 1u) ^ 1u)) {
            ok = false;
          } else {
            MmaTag tg{};
            tg.end = 0;
            tg.slot = it.slot;
            tg.first = (t == 0);
            tg.last = (t == nt - 1);
            tg.pos = t;
            tg.tile = j;
            s_btag[sl] = tg;
            uint8_t *dst = smem + L.off_blob + (size_t)sl * a.blob_cap;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            m_arrive_tx(&bfull[sl], tr.bytes);
            m_copy(dst, a.blobs + tr.off, tr.bytes, &bfull[sl]);
            // the per-bin factors also go to the epilogue's ring, which outlives the blob slot
            m_arrive_tx(&ffull[fs], kMmaBinsBytes);
            m_copy(smem + L.off_fac + (size_t)fs * kMmaFacBytes, a.blobs + tr.off + kMmaBinsOff, kMmaBinsBytes,
                   &ffull[fs]);
          }
        }
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      }
      if (!ok) break;
    }
    if (lane == 0) {
      const int sl = j % NB;
      if (ok && m_wait(&bempty[sl], ((uint32_t)(j / NB) & 1u) ^ 1u)) {
        MmaTag tg{};
        tg.end = 1;
        tg.tile = j;
        s_btag[sl] = tg;
        m_arrive(&bfull[sl]);
      } else {
        atomicExch(a.err, MI_E_TIMEOUT);
      }
    }
    __syncwarp();
  } else if (warp == 2 || warp == 3 || warp >= 4 + kMmaEpiWarps) {
    // ================= producers: stages (weight planes + frame planes) of K steps
    const int pw = warp < 4 ? warp - 2 : warp - (2 + kMmaEpiWarps);
    uint32_t g = 0;
    bool ok = true;
    for (int j = 0; ok; ++j) {
      const int sl = j % NB;
      if (!m_wait(&bfull[sl], (uint32_t)(j / NB) & 1u)) { ok = false; break; }
      const MmaTag bt = s_btag[sl];
      const uint8_t *blob = smem + L.off_blob + (size_t)sl * a.blob_cap;
      if (bt.end) {
        if ((int)(g % kMmaProducers) == pw) {
          const int q = (int)(g % kMmaStages);
          if (lane == 0) {
            if (m_wait(&empty[q], ((g / kMmaStages) & 1u) ^ 1u)) {
              MmaTag e = bt;
              s_shdr[q] = e;
              m_arrive(&full[q]);
            } else {
              atomicExch(a.err, MI_E_TIMEOUT);
            }
          }
        }
        break;
      }
      const MmaHdr hd = *(const MmaHdr *)blob;
      const MmaBlob BL = mma_blob_layout(hd.n_k, hd.n_runs, hd.n_terms);
      const uint2 *runs = (const uint2 *)(blob + BL.runs);
      const uint32_t *rptr = (const uint32_t *)(blob + BL.run_ptr);
      const uint32_t *sp = (const uint32_t *)(blob + BL.step_ptr);
      const uint4 *wpl = (const uint4 *)(blob + BL.wpl);
      const uint16_t *widx = (const uint16_t *)(blob + BL.widx);
      const int n_st = (hd.n_k + kMmaStepsPerStage - 1) / kMmaStepsPerStage;
      for (int s2 = 0; s2 < n_st; ++s2, ++g) {
        if ((int)(g % kMmaProducers) != pw) continue;
        const int q = (int)(g % kMmaStages);
        bool got = true;
        if (lane == 0) got = m_wait(&empty[q], ((g / kMmaStages) & 1u) ^ 1u);
        if (!__shfl_sync(0xffffffffu, got ? 1 : 0, 0)) { ok = false; break; }
        uint8_t *st = smem + (size_t)q * kMmaStageBytes;
        const int s0 = kMmaStepsPerStage * s2, s1 = min(s0 + kMmaStepsPerStage, hd.n_k);
        // frame planes: one bulk copy per run of consecutive pixels and plane; pixel slot k of
        // the stage is the 128-byte row k of each plane's operand (a K step is 32 rows)
        uint2 rn[kMmaStepsPerStage];
        uint32_t len[kMmaStepsPerStage], bytes = 0;
#pragma unroll
        for (int hs = 0; hs < kMmaStepsPerStage; ++hs) {
          rn[hs] = make_uint2(0u, 0u);
          if (s0 + hs < s1) {
            const int r0s = (int)rptr[s0 + hs], nrun = (int)rptr[s0 + hs + 1] - r0s;   // <= 32
            if (lane < nrun) rn[hs] = runs[r0s + lane];
          }
          len[hs] = rn[hs].y >> 8;
          bytes += __reduce_add_sync(0xffffffffu, len[hs]) * 256u;
        }
        if (lane == 0) m_expect_tx(&full[q], bytes);
        __syncwarp();
#pragma unroll
        for (int hs = 0; hs < kMmaStepsPerStage; ++hs)
          if (len[hs]) {
            const uint32_t ro = (uint32_t)(kMmaKStep * hs + (rn[hs].y & 0xFFu)) * 128u;
            m_copy(st + ro, a.xc_lo + (size_t)rn[hs].x * 128u, len[hs] * 128u, &full[q]);
            m_copy(st + kMmaAHi + ro, a.xc_hi + (size_t)rn[hs].x * 128u, len[hs] * 128u, &full[q]);
          }
        // weight planes: zero, then the stage's terms; byte (n', k) of the K-major operand at
        // (n' % 8) * 16 + (n' / 8) * kMmaBSbo + (k % 16) + (k / 16) * 128, n' = 48 j + n
        uint4 *bz = (uint4 *)(st + kMmaB);
        for (int i = lane; i < (int)(4u * kMmaBPlane / 16u); i += 32) bz[i] = make_uint4(0u, 0u, 0u, 0u);
        __syncwarp();
        static_assert(kMmaStepsPerStage == 1, "weight words are indexed within one K step");
        const int t0 = (int)sp[s0], t1 = (int)sp[s1];
        // four words per lane loaded before any store: the words and the planes share shared
        // memory, so the compiler cannot hoist the next loads above the stores by itself
        for (int t = t0 + lane; t < t1; t += 4 * 32) {
          uint4 wv[4];
          uint32_t wi[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const bool in = t + 32 * u < t1;
            wv[u] = in ? wpl[t + 32 * u] : make_uint4(0u, 0u, 0u, 0u);
            wi[u] = in ? widx[t + 32 * u] : 0u;
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (t + 32 * u >= t1) break;
            // word w of bin n: slots 4w .. 4w+3, bytes (k % 16) + (k / 16) * 128 of row n
            const uint32_t w = wi[u] & 7u, n = wi[u] >> 3;
            const uint32_t off = (n & 7u) * 16u + (n >> 3) * kMmaBSbo + (w & 3u) * 4u + (w >> 2) * 128u;
            uint32_t *b0 = (uint32_t *)(st + kMmaB + off);
            b0[0] = wv[u].x;
            b0[kMmaBPlane / 4] = wv[u].y;
            b0[2 * kMmaBPlane / 4] = wv[u].z;
            b0[3 * kMmaBPlane / 4] = wv[u].w;
          }
        }
        if (lane == 0) {
          MmaTag h = bt;
          h.r0 = hd.r0;
          h.n_rows = hd.n_rows;
          h.e0 = hd.e0;
          h.n_cols = hd.n_cols;
          h.step = s2;
          h.n_k = hd.n_k;
          h.box = hd.box_rows;
          s_shdr[q] = h;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) m_arrive(&full[q]);
      }
      __syncwarp();
      if (lane == 0) m_arrive(&bempty[sl]);
    }
    if (!ok && lane == 0) atomicExch(a.err, MI_E_TIMEOUT);
    __syncwarp();
  } else {
    // ================= epilogue: TMEM -> cake tile (TMA store) + lineout partials
    constexpr int kHalf = kMmaN / 2;               // bins per epilogue warp
    constexpr int kHalfRows = kHalf / kMmaCols;
    const int e = warp - 4, quad = warp & 3, half = e >> 2;
    const int m = quad * 32 + lane;                 // frame of the launch
    const bool live = m < a.F;
    const bool issuer = e == 0 && lane == 0;
    double saw[kHalfRows], ssm[kHalfRows];
#pragma unroll
    for (int i = 0; i < kHalfRows; ++i) saw[i] = ssm[i] = 0.0;
    for (int j = 0;; ++j) {
      const int ab = j & 1;
      bool got = true;
      if (lane == 0) got = m_wait(&afull[ab], (uint32_t)(j >> 1) & 1u);
      if (!__shfl_sync(0xffffffffu, got ? 1 : 0, 0)) {
        if (lane == 0) atomicExch(a.err, MI_E_TIMEOUT);
        break;
      }
      m_fence_after();
      const MmaTag tg = s_atag[ab];
      if (tg.end) break;
      if (tg.first) {
#pragma unroll
        for (int i = 0; i < kHalfRows; ++i) saw[i] = ssm[i] = 0.0;
      }
      // cake tiles go out in pairs through one store box (cake_box_off); an item's odd last
      // tile goes alone
      float *ot = (float *)(smem + L.off_out);
      const bool second = (tg.pos & 1) != 0;
      const int pitch = (second || !tg.last) ? 2 * kMmaCols : kMmaCols;
      const int coff = second ? kMmaCols : 0;
      if (a.use_tma && !second) {
        // the previous store has read the tile's shared memory
        if (issuer) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
        asm volatile("bar.sync 1, %0;" ::"r"(kMmaEpiWarps * 32) : "memory");
      }
      const uint32_t tbase = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(ab * kMmaAccCols + kHalf * half);
      float *crow = a.cake + (size_t)m * (size_t)a.n_bins;
      // the tile's per-bin factors, in its entry of the factor ring
      const int fs = j % kMmaFacSlots;
      if (lane == 0) got = m_wait(&ffull[fs], (uint32_t)(j / kMmaFacSlots) & 1u);
      if (!__shfl_sync(0xffffffffu, got ? 1 : 0, 0)) {
        if (lane == 0) atomicExch(a.err, MI_E_TIMEOUT);
        break;
      }
      const uint8_t *bb = smem + L.off_fac + (size_t)fs * kMmaFacBytes;
      const double *bfac = (const double *)bb + kHalf * half;
      const double *bdk = (const double *)bb + kMmaN + kHalf * half;
      const float *blw = (const float *)(bb + 16 * kMmaN) + kHalf * half;
#pragma unroll
      for (int c = 0; c < kHalf / 8; ++c) {
        uint32_t r[5][8];
#pragma unroll
        for (int k = 0; k < 5; ++k) m_ld8(tbase + (uint32_t)(k * kMmaN + 8 * c), r[k]);
        m_ld_wait();
        if (c == kHalf / 8 - 1) {
          // every accumulator of the set has been read: hand it back to the MMA lane
          m_fence_before();
          __syncwarp();
          if (lane == 0) m_arrive(&aempty[ab]);
        }
        // bins outside the tile have fac = dk = lw = 0: no branches
        float o[8];
        double fv[8], dv[8];
        float lv[8];
#pragma unroll
        for (int i = 0; i < 8; i += 2) {
          const double2 f2 = *(const double2 *)(bfac + 8 * c + i), d2 = *(const double2 *)(bdk + 8 * c + i);
          fv[i] = f2.x; fv[i + 1] = f2.y; dv[i] = d2.x; dv[i + 1] = d2.y;
        }
#pragma unroll
        for (int i = 0; i < 8; i += 4) {
          const float4 l4 = *(const float4 *)(blw + 8 * c + i);
          lv[i] = l4.x; lv[i + 1] = l4.y; lv[i + 2] = l4.z; lv[i + 3] = l4.w;
        }
        double rw[8], rs[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const double v = m_acc5(r[0][i], r[1][i], r[2][i], r[3][i], r[4][i]);
          const double res = fma(fv[i], v, -dv[i]);
          o[i] = (float)res;
          rw[i] = res * (double)lv[i];
          rs[i] = (lv[i] > 0.0f) ? res : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int lrow = (8 * c) / kMmaCols + q;
          saw[lrow] += (rw[4 * q] + rw[4 * q + 1]) + (rw[4 * q + 2] + rw[4 * q + 3]);
          ssm[lrow] += (rs[4 * q] + rs[4 * q + 1]) + (rs[4 * q + 2] + rs[4 * q + 3]);
        }
        if (!a.use_tma && live && a.want_cake) {
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const int n = kHalf * half + 8 * c + i, row = n / kMmaCols, col = n % kMmaCols;
            if (row < tg.n_rows && col < tg.n_cols) crow[(int64_t)(tg.r0 + row) * a.n_eta + tg.e0 + col] = o[i];
          }
        }
        if (a.use_tma) {
          // rows 2c, 2c+1 of this warp's half: one float4 each, if inside the store box
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int row = kHalfRows * half + 2 * c + q;
            if (row < tg.box) *(float4 *)(ot + cake_box_off(row, m, pitch, coff)) =
                make_float4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
          }
        }
      }
      if (a.use_tma && (second || tg.last)) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("bar.sync 1, %0;" ::"r"(kMmaEpiWarps * 32) : "memory");
        if (issuer) {
          const int bi = cake_box_index(tg.box, second);
          asm volatile(
              "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(&a.tmap[bi]),
              "r"(tg.e0 - coff), "r"(0), "r"(tg.r0), "r"(m_smem(ot))
              : "memory");
          asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
      }
      __syncwarp();
      if (lane == 0) m_arrive(&fempty[fs]);   // this warp is done with the tile's factors
      if (tg.last && a.want_lo && live) {
#pragma unroll
        for (int i = 0; i < kHalfRows; ++i) {
          const int row = kHalfRows * half + i;
          if (row < tg.n_rows) {
            double *dst = a.partial + (((int64_t)m * a.n_r + tg.r0 + row) * a.n_slots + tg.slot) * 2;
            dst[0] = saw[i];
            dst[1] = ssm[i];
          }
        }
      }
    }
    if (issuer) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  }
  m_fence_before();
  __syncthreads();
  if (warp == 0) {
    m_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kMmaTmemCols) : "memory");
  }
}

// dark term of each bin: dk = fac * sum over the bin's terms of q * dark[pixel], written into
// the tile's blob; one block per tile, one warp per six bins (deterministic order)
__global__ void k_mma_dark(const TileRef *tiles, uint8_t *blobs, const int32_t *xc_pix, const float *dark,
                           int has_dark) {
  const TileRef tr = tiles[blockIdx.x];
  uint8_t *blob = blobs + tr.off;
  const MmaHdr hd = *(const MmaHdr *)blob;
  const MmaBlob BL = mma_blob_layout(hd.n_k, hd.n_runs, hd.n_terms);
  const uint2 *runs = (const uint2 *)(blob + BL.runs);
  const uint32_t *rptr = (const uint32_t *)(blob + BL.run_ptr);
  const uint32_t *sp = (const uint32_t *)(blob + BL.step_ptr);
  const uint4 *wpl = (const uint4 *)(blob + BL.wpl);
  const uint16_t *widx = (const uint16_t *)(blob + BL.widx);
  // warp w sums the terms of bins w, w + 8, ..., its lanes striding over the tile's terms,
  // then reduces over the lanes in a fixed order: the same dark gives the same dk bits
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  constexpr int kW = kMmaDarkWarps, kPer = kMmaN / kMmaDarkWarps;
  const double *fac = (const double *)(blob + kMmaBinsOff);
  double *dk = (double *)(blob + kMmaBinsOff) + kMmaN;
  double d[kPer];
#pragma unroll
  for (int i = 0; i < kPer; ++i) d[i] = 0.0;
  if (has_dark)
    for (int t = lane; t < hd.n_terms; t += 32) {
      const int n = (int)(widx[t] >> 3);
      if (n % kW != w) continue;
      // the word's K step: the step whose word range holds it
      uint32_t s = 0;
      while (sp[s + 1] <= (uint32_t)t) ++s;
      const uint4 wv = wpl[t];
      for (int b = 0; b < 4; ++b) {
        const uint32_t dg = ((wv.x >> (8 * b)) & 0xFFu) | (((wv.y >> (8 * b)) & 0xFFu) << 8) |
                            (((wv.z >> (8 * b)) & 0xFFu) << 16) | (((wv.w >> (8 * b)) & 0xFFu) << 24);
        if (dg == 0u) continue;
        // the slot's pixel: the run of the step that covers the slot
        const uint32_t kk = (widx[t] & 7u) * 4u + (uint32_t)b;
        uint32_t c = 0;
        for (uint32_t r = rptr[s]; r < rptr[s + 1]; ++r) {
          const uint32_t k0 = runs[r].y & 0xFFu, len = runs[r].y >> 8;
          if (kk >= k0 && kk < k0 + len) { c = runs[r].x + (kk - k0); break; }
        }
        const double v = (double)mma_digits_value(dg) * (double)dark[xc_pix[c]];
#pragma unroll
        for (int i = 0; i < kPer; ++i)
          if (n / kW == i) d[i] += v;
      }
    }
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d[i] += __shfl_xor_sync(0xffffffffu, d[i], o);
    if (lane == 0) dk[w + kW * i] = fac[w + kW * i] * d[i];
  }
}

// the compiled (stages, producers) pairs
static constexpr int kMmaPipelines[][2] = {{8, 6}, {7, 6}, {6, 6}, {5, 5}, {7, 7}, {4, 4}};

template <int S, int P>
static int launch_mma_t(int grid, uint32_t smem, const MmaArgs &a, cudaStream_t s) {
  MI_CUDA(cudaFuncSetAttribute(k_mma<S, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_mma<S, P><<<grid, mma_threads(P), smem, s>>>(a);
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

static int launch_mma_variant(int S, int P, int grid, uint32_t smem, const MmaArgs &a, cudaStream_t s) {
  if (S == 7 && P == 6) return launch_mma_t<7, 6>(grid, smem, a, s);
  if (S == 6 && P == 6) return launch_mma_t<6, 6>(grid, smem, a, s);
  if (S == 5 && P == 5) return launch_mma_t<5, 5>(grid, smem, a, s);
  if (S == 7 && P == 7) return launch_mma_t<7, 7>(grid, smem, a, s);
  if (S == 4 && P == 4) return launch_mma_t<4, 4>(grid, smem, a, s);
  if (S == 8 && P == 6) return launch_mma_t<8, 6>(grid, smem, a, s);
  return set_error(MI_E_UNSUPPORTED, "launch_mma: no kernel for %d stages and %d producers", S, P);
}

int launch_mma(Plan *p, int F, float *cake, double *partial, bool want_lo, cudaStream_t s) {
  if (F <= 0 || F > kMmaFrames) return set_error(MI_E_ARG, "launch_mma: %d frames (1..%d)", F, kMmaFrames);
  MmaArgs a;
  memset(&a, 0, sizeof(a));
  a.items = p->d_items;
  a.tiles = p->d_tiles;
  a.blobs = p->d_blobs;
  a.xc_lo = p->d_xc;
  a.xc_hi = p->d_xc + (size_t)p->n_xc * 128;
  a.cake = cake;
  a.partial = partial;
  a.F = F;
  a.n_r = p->n_r;
  a.n_eta = p->n_eta;
  a.n_slots = p->n_slots;
  a.n_bins = p->n_bins;
  a.want_cake = cake != nullptr;
  a.want_lo = want_lo;
  a.n_items = p->n_items;
  a.counter = p->d_ctr;
  a.err = p->d_err;
  a.blob_cap = (p->max_blob + 15u) & ~15u;
  if (a.blob_cap > kMmaBlobCap) return set_error(MI_E_RANGE, "launch_mma: tile blob of %u B", a.blob_cap);
  // cake tiles leave through TMA tensor stores when the cake rows are 16-byte multiples
  // (n_eta % 4 == 0) and the cake is 16-byte aligned; otherwise through plain stores
  a.use_tma = 0;
  if (cake && p->n_eta % kMmaCols == 0 && (uintptr_t)cake % 16 == 0) {
    const int rc = encode_cake_boxes(a.tmap, cake, p->n_eta, p->n_r, p->n_bins, F, "launch_mma");
    if (rc != MI_OK) return rc;
    a.use_tma = 1;
  }
  // up to four blob slots, as shared memory allows (two suffice for progress: the epilogue
  // holds one, the producers use the next)
  int dev_smem = 0;
  MI_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, p->device));
  const int S = p->mma_stages;
  a.n_blob = kMmaBlobSlotsMax;
  while (a.n_blob > 2 && mma_smem_layout(a.blob_cap, a.n_blob, S).total > (uint32_t)dev_smem) --a.n_blob;
  const MmaSmem L = mma_smem_layout(a.blob_cap, a.n_blob, S);
  if (L.total > (uint32_t)dev_smem)
    return set_error(MI_E_RANGE, "launch_mma: %u B of shared memory needed (device allows %d)", L.total, dev_smem);
  MI_CUDA(cudaMemsetAsync(p->d_ctr, 0, sizeof(int), s));
  const int grid = std::max(1, std::min(p->n_items, p->n_sms));
  return launch_mma_variant(p->mma_stages, p->mma_producers, grid, L.total, a, s);
}

bool mma_pipeline_supported(int stages, int producers) {
  for (const auto &v : kMmaPipelines)
    if (v[0] == stages && v[1] == producers) return true;
  return false;
}

int launch_mma_dark(Plan *p, cudaStream_t s) {
  if (p->n_tiles == 0) return MI_OK;
  k_mma_dark<<<(unsigned)p->n_tiles, 32 * kMmaDarkWarps, 0, s>>>(p->d_tiles, p->d_blobs, p->d_xc_pix, p->d_dark,
                                                                  p->has_dark);
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

}  // namespace mi
