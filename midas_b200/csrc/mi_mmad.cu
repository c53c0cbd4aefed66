// mi_mmad.cu -- kernel (b), direct MMA encoding: batched caking on the tensor cores with the
// frames read in place (no pixel-major staging pass).
//
// Same contract as the other caking kernels (integrate() of packages/midas_integrate/
// midas_integrate/kernels.py:416-473, integrate_noMapMask of FF_HEDM/src/
// IntegratorFitPeaksGPUStream.cu:975-1050): cake = diag(scale) W (frames - dark) and the eta
// partial sums of both lineouts, for batches of up to 128 frames of 16-bit (or 8-bit) pixels.
//
// A tile (kMmaRows x kMmaCols = 48 bins) is a dense int8 product on the tensor cores:
//   D[frame][bin] (int32, TMEM) += A[frame][slot] (a byte plane of the frames, in TMEM)
//                                  x B[slot][bin]  (a byte plane of the weights, in SMEM)
// K = 32 slots per step = four 8-pixel granules (8 consecutive pixels of one detector row).
// Per K step two tcgen05.mma of N = 192 (the four weight planes side by side): the frames'
// low byte plane into accumulators 0-3, the high plane, one byte up, into accumulators 1-4.
// Every product and sum is exact; the epilogue forms sum_k 2^(8k) acc_k in FP64, subtracts
// the bin's dark term and scales: cake = fac * value - dk.  The approximation is the 32-bit
// fixed-point weight (2^-33 of the bin's largest weight) and the final rounding to float.
//
// Operands:
//   A (frames): in tensor memory, a ring of kDASlots K steps of 16 columns each (8 columns
//     low byte plane, 8 columns high byte plane; lane = frame, column c = slots 4c..4c+3).
//     Producer warp q (TMEM lanes 32q..32q+31) loads, per frame, each granule with one
//     16-byte load from the frame's own rows, splits the eight u16 pixels into their two
//     byte planes with byte permutes and stores both planes with one tcgen05.st.
//   B (weights): K-major without swizzle in shared memory, the four byte planes as rows
//     n' = 48 j + n; byte (n', k) at (n' % 8) * 16 + (n' / 8) * 256 + (k % 16) + (k / 16) * 128,
//     zeroed and scattered per stage from the stage's terms.
//
// Roles (one persistent CTA per SM, 16 warps, 128 registers a thread):
//   warp 0             TMEM allocation (512 columns: two accumulator sets of 5 x 48 and the
//                      two-slot A ring) and, on one lane, the MMA issue
//   warp 1             loader: claims work items (heaviest first), bulk-copies each tile's
//                      blob into a blob slot and its bins' factors into the epilogue's ring
//   warps 2,3,12-15    B producers: stage g (over the CTA's tiles) built by producer g % 6
//                      into stage slot g % kDStages (six, so that their proxy fences overlap)
//   warps 4-7          epilogue (TMEM lane quarters 0-3 = frames): TMEM -> FP64 recombination
//                      -> cake tile in shared memory -> one TMA tensor store per pair of
//                      adjacent tiles; lineout partial sums
//   warps 8-11         A producers (TMEM lane quarters 0-3): every K step, its granules loaded
//                      four steps ahead of its store into the ring
// Every wait is an mbarrier poll with an iteration limit; on expiry the kernel sets the
// plan's error word (MI_E_TIMEOUT) and the role leaves its loop.
#include <cuda.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>

#include "mi_internal.h"
#include "mi_tc.cuh"

namespace mi {

constexpr int kDStages = 8;
constexpr int kDProducers = 6;
static_assert(kDProducers <= kDStages, "more producers than stage slots aliases barrier phases");
constexpr int kDEpiWarps = 4;
constexpr int kDAWarps = 4;
constexpr int kDWarps = 2 + kDProducers + kDEpiWarps + kDAWarps;
constexpr int kDThreads = kDWarps * 32;
constexpr int kDPlanes = 4;                              // weight byte planes
constexpr int kDAcc = 5;                                 // accumulators (byte shifts 0..4)
constexpr uint32_t kDBPlane = 1536u;                     // 48 rows x 32 bytes
constexpr uint32_t kDStageBytes = kDPlanes * kDBPlane;   // 6144
constexpr int kDAccCols = kDAcc * kMmaN;                 // 240 columns per accumulator set
constexpr int kDASlots = 2;                              // A ring: K steps in tensor memory
constexpr int kDACol0 = 2 * kDAccCols;                   // 480: first column of the ring
constexpr int kDAhead = 4;                               // K steps loaded ahead of their store
constexpr int kDTmemCols = 512;
static_assert(kDACol0 + 16 * kDASlots <= kDTmemCols, "TMEM budget");
constexpr int kDBlobSlotsMax = 4;
constexpr int kDFacSlots = 6;
constexpr uint32_t kDFacBytes = 1024;
constexpr uint32_t kDOutBytes = kMmaFrames * kMmaN * 4;

struct MmadArgs {
  CUtensorMap tmap[kCakeBoxes];
  const WorkItem *items;
  const TileRef *tiles;
  const uint8_t *blobs;
  const uint8_t *frames;    // frame f at frames + f * stride elements
  int64_t stride;           // elements
  int u8;                   // 1: 8-bit frames
  int ny;
  float *cake;
  double *partial;          // [F][n_r][n_slots][2]
  int F, n_r, n_eta, n_slots;
  int64_t n_bins;
  int want_cake, want_lo, use_tma;
  int n_items;
  int *counter;
  int *err;
  uint32_t blob_cap;
  int n_blob;
};

struct MmadTag {
  int32_t end, tile, step, n_k;
  int32_t slot, first, last, box;
  int32_t r0, n_rows, e0, n_cols;
  int32_t pos, pad0, pad1, pad2;
};

struct MmadSmem {
  uint32_t off_out, off_blob, off_fac, off_shdr, off_btag, off_atag, off_bar, off_tmem, total;
};

__host__ __device__ inline MmadSmem mmad_smem_layout(uint32_t blob_cap, int n_blob) {
  MmadSmem L;
  uint32_t o = (uint32_t)kDStages * kDStageBytes;
  o = (o + 1023u) & ~1023u;
  L.off_out = o;   o += 2u * kDOutBytes;
  L.off_blob = o;  o += (uint32_t)n_blob * blob_cap;
  L.off_fac = o;   o += (uint32_t)kDFacSlots * kDFacBytes;
  L.off_shdr = o;  o += (uint32_t)kDStages * sizeof(MmadTag);
  L.off_btag = o;  o += (uint32_t)kDBlobSlotsMax * sizeof(MmadTag);
  L.off_atag = o;  o += 2u * sizeof(MmadTag);
  L.off_bar = o;
  o += 8u * (2u * kDStages + 2u * kDBlobSlotsMax + 2u * kDFacSlots + 4u + 2u * kDASlots);
  L.off_tmem = o;  o += 16u;
  L.total = o + 1024u;
  return L;
}

// instruction descriptor, kind::i8: D s32, A u8 K-major (tensor memory), B s8 K-major, M = 128
__host__ __device__ constexpr uint32_t mmad_idesc(int n) {
  return (2u << 4) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kMmaFrames >> 4) << 24);
}

__device__ __forceinline__ void m_mma_ta(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void m_st16(uint32_t taddr, const uint32_t *r) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
      "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
}
__device__ __forceinline__ void m_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// one granule (pixels y0 .. y0 + 7 of row z) of one frame, as eight u16 in a uint4 (u8
// frames: eight bytes in .x, .y).  VEC: one 16-byte (8-byte) load, the granule aligned in
// memory; else pixel by pixel, pixels past the row's end read as 0.
template <bool VEC>
__device__ __forceinline__ uint4 gran_load(const uint8_t *frame, int u8, int ny, uint32_t g) {
  if (g == kMmadEmpty || frame == nullptr) return make_uint4(0u, 0u, 0u, 0u);
  const uint32_t z = g & 0xFFFFu, y0 = g >> 16;
  const size_t px = (size_t)z * (size_t)ny + y0;
  if (VEC) {
    if (u8) {
      const uint2 t = __ldg((const uint2 *)(frame + px));
      return make_uint4(t.x, t.y, 0u, 0u);
    }
    return __ldg((const uint4 *)(frame + 2 * px));
  }
  uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
  for (int i = 0; i < kMmadGranPx; ++i) {
    if ((int)y0 + i >= ny) break;
    const uint32_t v = u8 ? (uint32_t)__ldg(frame + px + i) : (uint32_t)__ldg((const uint16_t *)frame + px + i);
    if (u8) w[i >> 2] |= v << (8 * (i & 3));
    else w[i >> 1] |= v << (16 * (i & 1));
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

template <bool VEC>
__global__ void __launch_bounds__(kDThreads, 1) k_mmad(const __grid_constant__ MmadArgs a) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = m_smem(smem_raw);
  uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  const MmadSmem L = mmad_smem_layout(a.blob_cap, a.n_blob);
  const int NB = a.n_blob;
  MmadTag *s_shdr = (MmadTag *)(smem + L.off_shdr);
  MmadTag *s_btag = (MmadTag *)(smem + L.off_btag);
  MmadTag *s_atag = (MmadTag *)(smem + L.off_atag);
  uint64_t *bar = (uint64_t *)(smem + L.off_bar);
  uint64_t *full = bar, *empty = bar + kDStages;
  uint64_t *bfull = bar + 2 * kDStages, *bempty = bfull + kDBlobSlotsMax;
  uint64_t *afull = bempty + kDBlobSlotsMax, *aempty = afull + 2;
  uint64_t *ffull = aempty + 2, *fempty = ffull + kDFacSlots;
  uint64_t *rfull = fempty + kDFacSlots, *rempty = rfull + kDASlots;   // A ring in TMEM
  uint32_t *s_tmem = (uint32_t *)(smem + L.off_tmem);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    for (int q = 0; q < kDStages; ++q) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(m_smem(&full[q])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(m_smem(&empty[q])) : "memory");
    }
    for (int q = 0; q < kDBlobSlotsMax; ++q) {
      // a blob slot is free again when the B producers have built its stages and the A
      // producers have issued its granule loads
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(m_smem(&bfull[q])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(m_smem(&bempty[q])), "r"(kDProducers + kDAWarps)
                   : "memory");
    }
    for (int q = 0; q < kDFacSlots; ++q) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(m_smem(&ffull[q])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(m_smem(&fempty[q])), "r"(kDEpiWarps) : "memory");
    }
    for (int q = 0; q < 2; ++q) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;" ::"r"(m_smem(&afull[q])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(m_smem(&aempty[q])), "r"(kDEpiWarps) : "memory");
    }
    for (int q = 0; q < kDASlots; ++q) {
      // a ring slot is full when all four A producer warps stored their lanes; empty when the
      // MMAs reading it have completed (one commit)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(m_smem(&rfull[q])), "r"(kDAWarps) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(m_smem(&rempty[q])) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(m_smem(s_tmem)),
                 "r"(kDTmemCols)
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
      int st = 0, n_st = 0, ab = 0;
      for (uint32_t g = 0;; ++g) {
        const int q = (int)(g % kDStages);
        if (!m_wait(&full[q], (g / kDStages) & 1u)) { ok = false; break; }
        if (st == n_st) {
          const int4 hq = *(const int4 *)&s_shdr[q];   // end, tile, step, n_k
          ab = hq.y & 1;
          if (hq.x) {
            if (!m_wait(&aempty[ab], ((uint32_t)(hq.y >> 1) & 1u) ^ 1u)) { ok = false; break; }
            s_atag[ab] = s_shdr[q];
            m_arrive(&afull[ab]);
            m_arrive(&afull[ab]);
            break;
          }
          n_st = hq.w;
          st = 0;
          if (!m_wait(&aempty[ab], ((uint32_t)(hq.y >> 1) & 1u) ^ 1u)) { ok = false; break; }
          m_fence_after();
          s_atag[ab] = s_shdr[q];
          m_arrive(&afull[ab]);
        }
        // the K step's frame planes in the A ring
        const int rs = (int)(g % kDASlots);
        if (!m_wait(&rfull[rs], (g / kDASlots) & 1u)) { ok = false; break; }
        m_fence_after();
        const uint32_t a_lo = tmem + (uint32_t)(kDACol0 + 16 * rs), a_hi = a_lo + 8u;
        const uint32_t bsa = m_smem(smem + (size_t)q * kDStageBytes);
        const uint32_t dbase = tmem + (uint32_t)(ab * kDAccCols);
        const uint64_t bd = m_desc(bsa, 128u, 256u, 0u);
        if (st != 0) {
          m_mma_ta(dbase, a_lo, bd, mmad_idesc(kDPlanes * kMmaN), 1u);
          m_mma_ta(dbase + (uint32_t)kMmaN, a_hi, bd, mmad_idesc(kDPlanes * kMmaN), 1u);
        } else {
          // a tile's first step starts each accumulator from zero: the low plane's product
          // starts 0-3, the high plane's adds onto 1-3 and starts 4
          m_mma_ta(dbase, a_lo, bd, mmad_idesc(kDPlanes * kMmaN), 0u);
          m_mma_ta(dbase + (uint32_t)kMmaN, a_hi, bd, mmad_idesc((kDPlanes - 1) * kMmaN), 1u);
          m_mma_ta(dbase + (uint32_t)(kDPlanes * kMmaN), a_hi,
                   m_desc(bsa + (uint32_t)(kDPlanes - 1) * kDBPlane, 128u, 256u, 0u), mmad_idesc(kMmaN), 0u);
        }
        m_commit(&empty[q]);
        m_commit(&rempty[rs]);
        if (++st == n_st) m_commit(&afull[ab]);
      }
      if (!ok) atomicExch(a.err, MI_E_TIMEOUT);
    }
    __syncwarp();
  } else if (warp == 1) {
    // ================= loader: items -> tile blobs and factors
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
          const int fs = j % kDFacSlots;
          if (!m_wait(&bempty[sl], ((uint32_t)(j / NB) & 1u) ^ 1u) ||
              !m_wait(&fempty[fs], ((uint32_t)(j / kDFacSlots) & 1u) ^ 1u)) {
            ok = false;
          } else {
            MmadTag tg{};
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
            m_arrive_tx(&ffull[fs], kMmaBinsBytes);
            m_copy(smem + L.off_fac + (size_t)fs * kDFacBytes, a.blobs + tr.off + kMmaBinsOff, kMmaBinsBytes,
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
        MmadTag tg{};
        tg.end = 1;
        tg.tile = j;
        s_btag[sl] = tg;
        m_arrive(&bfull[sl]);
      } else {
        atomicExch(a.err, MI_E_TIMEOUT);
      }
    }
    __syncwarp();
  } else if (warp == 2 || warp == 3 || warp >= 4 + kDEpiWarps + kDAWarps) {
    static_assert(4 + kDEpiWarps + kDAWarps + kDProducers - 2 == kDWarps, "warp roles");
    // ================= B producers: weight planes of K steps
    const int pw = warp < 4 ? warp - 2 : warp - (2 + kDEpiWarps + kDAWarps);
    uint32_t g = 0;
    bool ok = true;
    for (int j = 0; ok; ++j) {
      const int sl = j % NB;
      if (!m_wait(&bfull[sl], (uint32_t)(j / NB) & 1u)) { ok = false; break; }
      const MmadTag bt = s_btag[sl];
      const uint8_t *blob = smem + L.off_blob + (size_t)sl * a.blob_cap;
      if (bt.end) {
        if ((int)(g % kDProducers) == pw) {
          const int q = (int)(g % kDStages);
          if (lane == 0) {
            if (m_wait(&empty[q], ((g / kDStages) & 1u) ^ 1u)) {
              s_shdr[q] = bt;
              m_arrive(&full[q]);
            } else {
              atomicExch(a.err, MI_E_TIMEOUT);
            }
          }
        }
        break;
      }
      const MmaHdr hd = *(const MmaHdr *)blob;
      const MmadBlob BL = mmad_blob_layout(hd.n_k, hd.n_terms);
      const uint32_t *sp = (const uint32_t *)(blob + BL.step_ptr);
      const uint2 *terms = (const uint2 *)(blob + BL.terms);
      for (int s2 = 0; s2 < hd.n_k; ++s2, ++g) {
        if ((int)(g % kDProducers) != pw) continue;
        const int q = (int)(g % kDStages);
        bool got = true;
        if (lane == 0) got = m_wait(&empty[q], ((g / kDStages) & 1u) ^ 1u);
        if (!__shfl_sync(0xffffffffu, got ? 1 : 0, 0)) { ok = false; break; }
        uint8_t *stg = smem + (size_t)q * kDStageBytes;
        uint4 *bz = (uint4 *)stg;
        for (int i = lane; i < (int)(kDStageBytes / 16u); i += 32) bz[i] = make_uint4(0u, 0u, 0u, 0u);
        __syncwarp();
        const int t0 = (int)sp[s2], t1 = (int)sp[s2 + 1];
        const uint32_t kbase = (uint32_t)(kMmaKStep * s2);
        for (int t = t0 + lane; t < t1; t += 4 * 32) {
          uint2 tmv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) tmv[u] = t + 32 * u < t1 ? terms[t + 32 * u] : make_uint2(0u, 0u);
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (t + 32 * u >= t1) break;
            const uint2 tm = tmv[u];
            const uint32_t kk = (tm.y & 0xFFFFu) - kbase, n = tm.y >> 16;
            const uint32_t off = (n & 7u) * 16u + (n >> 3) * 256u + (kk & 15u) + (kk >> 4) * 128u;
            uint8_t *b0 = stg + off;
            b0[0] = (uint8_t)(tm.x & 0xFFu);
            b0[kDBPlane] = (uint8_t)((tm.x >> 8) & 0xFFu);
            b0[2 * kDBPlane] = (uint8_t)((tm.x >> 16) & 0xFFu);
            b0[3 * kDBPlane] = (uint8_t)(tm.x >> 24);
          }
        }
        if (lane == 0) {
          MmadTag h = bt;
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
  } else if (warp >= 4 + kDEpiWarps) {
    // ================= A producers: frame granules -> byte planes -> tensor memory
    const int qw = warp & 3;                       // TMEM lane quarter
    const int m = qw * 32 + lane;                  // frame of the launch
    const uint8_t *fb = m < a.F ? a.frames + (size_t)m * (size_t)a.stride * (a.u8 ? 1u : 2u) : nullptr;
    const uint32_t trow = tmem + ((uint32_t)(qw * 32) << 16);
    // issue cursor: the tile (blob slot, -1 before the first) and step whose granules are
    // loaded next
    int ji = -1, si = 0, nki = 0;
    const uint32_t *gi = nullptr;
    bool more = true, ok = true;
    uint4 buf[kDAhead][kMmadGran];
    uint32_t n_iss = 0;
    // load the granules of the next K step into buf[b]; false when no step is left
    auto issue = [&](uint4 *dst) -> bool {
      while (more && si == nki) {
        // the current tile's steps are all issued: its blob slot is free for the loader
        if (ji >= 0) {
          __syncwarp();
          if (lane == 0) m_arrive(&bempty[ji % NB]);
        }
        ++ji;
        const int sl = ji % NB;
        bool got = true;
        if (lane == 0) got = m_wait(&bfull[sl], (uint32_t)(ji / NB) & 1u);
        if (!__shfl_sync(0xffffffffu, got ? 1 : 0, 0)) { ok = false; more = false; break; }
        const uint8_t *blob = smem + L.off_blob + (size_t)sl * a.blob_cap;
        if (s_btag[sl].end) {
          more = false;
          break;
        }
        const MmaHdr hd = *(const MmaHdr *)blob;
        gi = (const uint32_t *)(blob + mmad_blob_layout(hd.n_k, hd.n_terms).gran);
        nki = hd.n_k;
        si = 0;
      }
      if (!more) return false;
      const uint4 gq = *(const uint4 *)(gi + kMmadGran * si);
      dst[0] = gran_load<VEC>(fb, a.u8, a.ny, gq.x);
      dst[1] = gran_load<VEC>(fb, a.u8, a.ny, gq.y);
      dst[2] = gran_load<VEC>(fb, a.u8, a.ny, gq.z);
      dst[3] = gran_load<VEC>(fb, a.u8, a.ny, gq.w);
      ++si;
      ++n_iss;
      return true;
    };
    // split one K step into its two byte planes and store them into ring slot g % kDASlots
    auto store = [&](const uint4 *src, uint32_t g) -> bool {
      const int rs = (int)(g % kDASlots);
      bool got = true;
      if (lane == 0) got = m_wait(&rempty[rs], ((g / kDASlots) & 1u) ^ 1u);
      if (!__shfl_sync(0xffffffffu, got ? 1 : 0, 0)) return false;
      m_fence_after();
      uint32_t r[16];
#pragma unroll
      for (int k = 0; k < kMmadGran; ++k) {
        if (a.u8) {
          r[2 * k] = src[k].x;
          r[2 * k + 1] = src[k].y;
          r[8 + 2 * k] = 0u;
          r[8 + 2 * k + 1] = 0u;
        } else {
          r[2 * k] = __byte_perm(src[k].x, src[k].y, 0x6420);
          r[2 * k + 1] = __byte_perm(src[k].z, src[k].w, 0x6420);
          r[8 + 2 * k] = __byte_perm(src[k].x, src[k].y, 0x7531);
          r[8 + 2 * k + 1] = __byte_perm(src[k].z, src[k].w, 0x7531);
        }
      }
      m_st16(trow + (uint32_t)(kDACol0 + 16 * rs), r);
      m_st_wait();
      m_fence_before();
      __syncwarp();
      if (lane == 0) m_arrive(&rfull[rs]);
      return true;
    };
#pragma unroll
    for (int b = 0; b < kDAhead; ++b)
      if (!issue(buf[b])) break;
    for (uint32_t g = 0; ok && g < n_iss; g += kDAhead) {
#pragma unroll
      for (int b = 0; b < kDAhead; ++b) {
        if (g + b >= n_iss) break;
        if (!store(buf[b], g + b)) { ok = false; break; }
        issue(buf[b]);
      }
    }
    if (!ok && lane == 0) atomicExch(a.err, MI_E_TIMEOUT);
    __syncwarp();
  } else {
    // ================= epilogue: TMEM -> cake tile (TMA store) + lineout partials
    constexpr int kHalf = kMmaN;                 // bins per epilogue warp (all of the tile)
    constexpr int kHalfRows = kHalf / kMmaCols;
    const int e = warp - 4, quad = warp & 3, half = 0;
    const int m = quad * 32 + lane;
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
      const MmadTag tg = s_atag[ab];
      if (tg.end) break;
      if (tg.first) {
#pragma unroll
        for (int i = 0; i < kHalfRows; ++i) saw[i] = ssm[i] = 0.0;
      }
      float *ot = (float *)(smem + L.off_out);
      const bool second = (tg.pos & 1) != 0;
      const int pitch = (second || !tg.last) ? 2 * kMmaCols : kMmaCols;
      const int coff = second ? kMmaCols : 0;
      if (a.use_tma && !second) {
        if (issuer) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
        asm volatile("bar.sync 1, %0;" ::"r"(kDEpiWarps * 32) : "memory");
      }
      const uint32_t tbase = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(ab * kDAccCols + kHalf * half);
      float *crow = a.cake + (size_t)m * (size_t)a.n_bins;
      const int fs = j % kDFacSlots;
      if (lane == 0) got = m_wait(&ffull[fs], (uint32_t)(j / kDFacSlots) & 1u);
      if (!__shfl_sync(0xffffffffu, got ? 1 : 0, 0)) {
        if (lane == 0) atomicExch(a.err, MI_E_TIMEOUT);
        break;
      }
      const uint8_t *bb = smem + L.off_fac + (size_t)fs * kDFacBytes;
      const double *bfac = (const double *)bb + kHalf * half;
      const double *bdk = (const double *)bb + kMmaN + kHalf * half;
      const float *blw = (const float *)(bb + 16 * kMmaN) + kHalf * half;
#pragma unroll
      for (int c = 0; c < kHalf / 8; ++c) {
        uint32_t r[kDAcc][8];
#pragma unroll
        for (int k = 0; k < kDAcc; ++k) m_ld8(tbase + (uint32_t)(k * kMmaN + 8 * c), r[k]);
        m_ld_wait();
        if (c == kHalf / 8 - 1) {
          m_fence_before();
          __syncwarp();
          if (lane == 0) m_arrive(&aempty[ab]);
        }
        float o[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int lrow = (8 * c + i) / kMmaCols;
          // sum_k 2^(8k) acc_k exactly in int64 (|sum| < 2^63), one rounding to FP64
          const double v = m_acc5(r[0][i], r[1][i], r[2][i], r[3][i], r[4][i]);
          const double res = fma(bfac[8 * c + i], v, -bdk[8 * c + i]);
          const float l = blw[8 * c + i];
          o[i] = (float)res;
          saw[lrow] = fma(res, (double)l, saw[lrow]);
          ssm[lrow] += (l > 0.0f) ? res : 0.0;
        }
        if (!a.use_tma && live && a.want_cake) {
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const int n = kHalf * half + 8 * c + i, row = n / kMmaCols, col = n % kMmaCols;
            if (row < tg.n_rows && col < tg.n_cols) crow[(int64_t)(tg.r0 + row) * a.n_eta + tg.e0 + col] = o[i];
          }
        }
        if (a.use_tma) {
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
        asm volatile("bar.sync 1, %0;" ::"r"(kDEpiWarps * 32) : "memory");
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
      if (lane == 0) m_arrive(&fempty[fs]);
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
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kDTmemCols) : "memory");
  }
}

// dark term of each bin: dk = fac * sum over the bin's terms of q * dark[pixel], written into
// the tile's blob; one block per tile, one warp per six bins (deterministic order)
__global__ void k_mmad_dark(const TileRef *tiles, uint8_t *blobs, int ny, const float *dark, int has_dark) {
  const TileRef tr = tiles[blockIdx.x];
  uint8_t *blob = blobs + tr.off;
  const MmaHdr hd = *(const MmaHdr *)blob;
  const MmadBlob BL = mmad_blob_layout(hd.n_k, hd.n_terms);
  const uint32_t *gran = (const uint32_t *)(blob + BL.gran);
  const uint2 *terms = (const uint2 *)(blob + BL.terms);
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
      const uint2 tm = terms[t];
      const int n = (int)(tm.y >> 16);
      if (n % kW != w) continue;
      const uint32_t k = tm.y & 0xFFFFu, g = gran[k / kMmadGranPx];
      const size_t px = (size_t)(g & 0xFFFFu) * (size_t)ny + (g >> 16) + (k % kMmadGranPx);
      const double v = (double)mma_digits_value(tm.x) * (double)dark[px];
#pragma unroll
      for (int i = 0; i < kPer; ++i)
        if (n / kW == i) d[i] += v;
    }
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d[i] += __shfl_xor_sync(0xffffffffu, d[i], o);
    if (lane == 0) dk[w + kW * i] = fac[w + kW * i] * d[i];
  }
}

int launch_mmad(Plan *p, const void *frames, int dtype, int F, int64_t stride, float *cake, double *partial,
                bool want_lo, cudaStream_t s) {
  if (F <= 0 || F > kMmaFrames) return set_error(MI_E_ARG, "launch_mmad: %d frames (1..%d)", F, kMmaFrames);
  if (dtype != MI_DT_U16 && dtype != MI_DT_U8)
    return set_error(MI_E_UNSUPPORTED, "launch_mmad: 8/16-bit frames only (dtype %d)", dtype);
  const int u8 = dtype == MI_DT_U8;
  const size_t gb = u8 ? 8u : 16u;   // bytes of one granule
  // granules aligned in memory load with one vector load each, else pixel by pixel
  const bool vec = (uintptr_t)frames % gb == 0 && ((size_t)stride * (u8 ? 1u : 2u)) % gb == 0 &&
                   p->ny % kMmadGranPx == 0;
  if (!u8 && (uintptr_t)frames % 2 != 0) return set_error(MI_E_ARG, "launch_mmad: u16 frames at an odd address");
  MmadArgs a;
  memset(&a, 0, sizeof(a));
  a.items = p->d_items;
  a.tiles = p->d_tiles;
  a.blobs = p->d_blobs;
  a.frames = (const uint8_t *)frames;
  a.stride = stride;
  a.u8 = u8;
  a.ny = p->ny;
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
  if (a.blob_cap > kMmaBlobCap) return set_error(MI_E_RANGE, "launch_mmad: tile blob of %u B", a.blob_cap);
  a.use_tma = 0;
  if (cake && p->n_eta % kMmaCols == 0 && (uintptr_t)cake % 16 == 0) {
    const int rc = encode_cake_boxes(a.tmap, cake, p->n_eta, p->n_r, p->n_bins, F, "launch_mmad");
    if (rc != MI_OK) return rc;
    a.use_tma = 1;
  }
  int dev_smem = 0;
  MI_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, p->device));
  a.n_blob = kDBlobSlotsMax;
  while (a.n_blob > 2 && mmad_smem_layout(a.blob_cap, a.n_blob).total > (uint32_t)dev_smem) --a.n_blob;
  const MmadSmem L = mmad_smem_layout(a.blob_cap, a.n_blob);
  if (L.total > (uint32_t)dev_smem)
    return set_error(MI_E_RANGE, "launch_mmad: %u B of shared memory needed (device allows %d)", L.total, dev_smem);
  MI_CUDA(cudaFuncSetAttribute(vec ? k_mmad<true> : k_mmad<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)L.total));
  MI_CUDA(cudaMemsetAsync(p->d_ctr, 0, sizeof(int), s));
  const int grid = std::max(1, std::min(p->n_items, p->n_sms));
  if (vec) k_mmad<true><<<grid, kDThreads, L.total, s>>>(a);
  else k_mmad<false><<<grid, kDThreads, L.total, s>>>(a);
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

int launch_mmad_dark(Plan *p, cudaStream_t s) {
  if (p->n_tiles == 0) return MI_OK;
  k_mmad_dark<<<(unsigned)p->n_tiles, 32 * kMmaDarkWarps, 0, s>>>(p->d_tiles, p->d_blobs, p->ny, p->d_dark,
                                                                   p->has_dark);
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

}  // namespace mi
