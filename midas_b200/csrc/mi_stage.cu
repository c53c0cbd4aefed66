// mi_stage.cu -- kernel (a) of the batched path: pixel-major staging of a launch's frames.
//
// The reference casts each frame to float and subtracts the dark per pixel before the
// per-bin sums (process_direct_kernel<T>, FF_HEDM/src/IntegratorFitPeaksGPUStream.cu:
// 1148-1160).  Here the frames of a launch are transposed from frame-major [f][z][y] to
// pixel-major rows over the compact pixel index c of the plan's row spans, so a tile
// stages each of its pixels (one frame group) with one 128-byte bulk copy instead of
// scattered 2- or 4-byte loads across frames that lie megabytes apart:
//  * 8/16-bit frames: u16 rows of 128 frames; the cast and the dark stay in kernel (b),
//    (float)raw - dark per staged value, the reference's arithmetic;
//  * other frame types: fp32 rows of 64 frames holding (float)raw - dark, the same
//    arithmetic done here once per pixel and frame.
// Each panel of a panel plan is transposed by its own launch into its part of the
// buffer (its rows of the virtual detector).
//
// One CTA per chunk (<= 256 pixels of one span): 16-byte loads of the chunk's frame rows
// where alignment allows (u16), into shared memory with 16-byte groups XOR-swizzled by
// frame octet so the transposed reads are conflict-free; then 16-byte stores, eight
// consecutive threads writing one pixel's 128-byte row of a frame group.
#include <stdint.h>

#include "mi_internal.h"

namespace mi {

// PLANES (MMA encoding): two byte planes [lo: n_xc x 128][hi: n_xc x 128] (the buffer's
// n_xc x 256 bytes); row c of a plane holds that byte of compact pixel c's 128 frames, the
// 16-byte granule of frames 16g .. 16g+15 at position g ^ (c % 8): the 128-byte swizzle
// phase the tensor-core operand of a K slot with k % 8 == c % 8 expects, so a run of
// consecutive pixels is staged with one plain bulk copy per plane.
constexpr int kXcLoads = 8;

template <typename T, bool VEC, bool PLANES>
__global__ void __launch_bounds__(256) k_xc(const T *__restrict__ frames, int64_t stride, int F, int ny, int z_off,
                                            const XcChunk *__restrict__ chunks, uint8_t *__restrict__ xc,
                                            int64_t n_xc) {
  constexpr int kPitch = kXcRowBytes / 2;  // u16 per compact pixel
  __shared__ __align__(16) uint16_t S[kXcFrames][kXcChunk + 8];
  const XcChunk ch = chunks[blockIdx.x];
  const int nv = (ch.n + 7) >> 3;  // groups of 8 pixels
  const int64_t base = (int64_t)(ch.z - z_off) * ny + ch.y0;
  uint16_t *out = (uint16_t *)xc;
  for (int h = 0; h * kXcFrames < F; ++h) {
    const int fh = min(kXcFrames, F - h * kXcFrames);
    if (h) __syncthreads();
    // kXcLoads groups per thread per pass, all loads issued before the first shared-memory
    // store, so each thread keeps that many 16-byte reads in flight
    const int n_items = kXcFrames * nv;
    for (int i0 = threadIdx.x; i0 < n_items; i0 += kXcLoads * blockDim.x) {
      uint4 val[kXcLoads];
#pragma unroll
      for (int u = 0; u < kXcLoads; ++u) {
        const int i = i0 + u * blockDim.x;
        const int f = i / nv, v = i - f * nv;
        val[u] = make_uint4(0u, 0u, 0u, 0u);
        if (i < n_items && f < fh) {
          const T *src = frames + (int64_t)(h * kXcFrames + f) * stride + base + 8 * v;
          if constexpr (VEC) {
            val[u] = __ldg((const uint4 *)src);
          } else {
            uint32_t t[4];
#pragma unroll
            for (int j = 0; j < 8; j += 2) {
              const uint32_t lo = (8 * v + j < ch.n) ? (uint32_t)(uint16_t)__ldg(src + j) : 0u;
              const uint32_t hi = (8 * v + j + 1 < ch.n) ? (uint32_t)(uint16_t)__ldg(src + j + 1) : 0u;
              t[j / 2] = lo | (hi << 16);
            }
            val[u] = make_uint4(t[0], t[1], t[2], t[3]);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < kXcLoads; ++u) {
        const int i = i0 + u * blockDim.x;
        if (i < n_items) {
          const int f = i / nv, v = i - f * nv;
          *(uint4 *)&S[f][8 * (v ^ ((f >> 3) & 7))] = val[u];
        }
      }
    }
    __syncthreads();
    if constexpr (PLANES) {
      // pixel p, 16-frame granule g of this half (frame octets 2g, 2g+1): one 16-byte store
      // per byte plane, four consecutive threads writing one pixel's half row
      for (int i = threadIdx.x; i < ch.n * 4; i += blockDim.x) {
        const int p = i >> 2, g = i & 3;
        uint32_t w[8];
#pragma unroll
        for (int o = 0; o < 2; ++o) {
          const int q = 2 * g + o;
          const int col = 8 * ((p >> 3) ^ q) + (p & 7);
#pragma unroll
          for (int j = 0; j < 8; j += 2)
            w[4 * o + j / 2] = (uint32_t)S[8 * q + j][col] | ((uint32_t)S[8 * q + j + 1][col] << 16);
        }
        const int cc = ch.c0 + p;
        uint8_t *row = xc + (int64_t)cc * 128 + 16 * ((4 * h + g) ^ (cc & 7));
        *(uint4 *)row = make_uint4(__byte_perm(w[0], w[1], 0x6420), __byte_perm(w[2], w[3], 0x6420),
                                   __byte_perm(w[4], w[5], 0x6420), __byte_perm(w[6], w[7], 0x6420));
        *(uint4 *)(row + n_xc * 128) = make_uint4(__byte_perm(w[0], w[1], 0x7531), __byte_perm(w[2], w[3], 0x7531),
                                                  __byte_perm(w[4], w[5], 0x7531), __byte_perm(w[6], w[7], 0x7531));
      }
    } else {
      for (int i = threadIdx.x; i < ch.n * 8; i += blockDim.x) {
        const int p = i >> 3, q = i & 7;
        const int col = 8 * ((p >> 3) ^ q) + (p & 7);
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 8; j += 2)
          w[j / 2] = (uint32_t)S[8 * q + j][col] | ((uint32_t)S[8 * q + j + 1][col] << 16);
        *(uint4 *)(out + (int64_t)(ch.c0 + p) * kPitch + h * kXcFrames + 8 * q) = make_uint4(w[0], w[1], w[2], w[3]);
      }
    }
  }
}

// fp32 rows, (float)raw - dark: 64 frames per compact pixel, transposed 32 frames at a
// time; a frame's dark is the plan's (virtual-detector) dark at the pixel
template <typename T>
__global__ void __launch_bounds__(256) k_xcf(const T *__restrict__ frames, int64_t stride, int F, int ny, int z_off,
                                             int ny_v, const float *__restrict__ dark,
                                             const XcChunk *__restrict__ chunks, uint8_t *__restrict__ xc) {
  constexpr int kPitch = kXcRowBytes / 4;             // floats per compact pixel
  __shared__ float S[kXcFramesF][kXcChunk + 1];
  const XcChunk ch = chunks[blockIdx.x];
  const int64_t base = (int64_t)(ch.z - z_off) * ny + ch.y0;
  const int64_t vbase = (int64_t)ch.z * ny_v + ch.y0;
  float *out = (float *)xc;
  for (int h = 0; h * kXcFramesF < F; ++h) {
    const int fh = min(kXcFramesF, F - h * kXcFramesF);
    if (h) __syncthreads();
    for (int i = threadIdx.x; i < kXcFramesF * ch.n; i += blockDim.x) {
      const int f = i / ch.n, y = i - f * ch.n;
      float v = 0.0f;
      if (f < fh)
        v = (float)__ldg(frames + (int64_t)(h * kXcFramesF + f) * stride + base + y) - __ldg(dark + vbase + y);
      S[f][y] = v;
    }
    __syncthreads();
    // pixel p, frames 4q .. 4q+3 of the group: eight consecutive threads write one pixel's
    // 128-byte row
    for (int i = threadIdx.x; i < ch.n * 8; i += blockDim.x) {
      const int p = i >> 3, q = i & 7;
      *(float4 *)(out + (int64_t)(ch.c0 + p) * kPitch + h * kXcFramesF + 4 * q) =
          make_float4(S[4 * q][p], S[4 * q + 1][p], S[4 * q + 2][p], S[4 * q + 3][p]);
    }
  }
}

bool runs_uses_xc(const Plan *p, int dtype) { return p->n_xc > 0 && dtype_size(dtype) > 0; }

template <typename T>
static void xcf_launch(Plan *p, const Plan::Panel &pn, const void *frames, int F, int64_t stride, cudaStream_t s) {
  k_xcf<T><<<(unsigned)(pn.chunk_end - pn.chunk_begin), 256, 0, s>>>(
      (const T *)frames, stride, F, pn.ny, pn.z_off, p->ny, p->d_dark, p->d_xchunks + pn.chunk_begin, p->d_xc);
}

int launch_xc(Plan *p, int panel, const void *frames, int dtype, int F, int64_t stride, bool as_f32,
              cudaStream_t s) {
  const int cap = as_f32 ? kXcFramesF * kXcGroupsF : kXcFrames * kXcGroups;
  if (F <= 0 || F > cap) return set_error(MI_E_ARG, "launch_xc: %d frames (1..%d)", F, cap);
  const Plan::Panel &pn = p->panels[panel];
  const unsigned grid = (unsigned)(pn.chunk_end - pn.chunk_begin);
  if (grid == 0) return MI_OK;
  const XcChunk *chunks = p->d_xchunks + pn.chunk_begin;
  if (!as_f32) {
    const bool planes = p->encoding == MI_ENC_MMA;
    if (dtype == MI_DT_U16) {
      const bool vec = ((uintptr_t)frames % 16 == 0) && ((stride * 2) % 16 == 0) && ((pn.ny * 2) % 16 == 0);
      const uint16_t *f16 = (const uint16_t *)frames;
      if (vec && planes)
        k_xc<uint16_t, true, true><<<grid, 256, 0, s>>>(f16, stride, F, pn.ny, pn.z_off, chunks, p->d_xc, p->n_xc);
      else if (vec)
        k_xc<uint16_t, true, false><<<grid, 256, 0, s>>>(f16, stride, F, pn.ny, pn.z_off, chunks, p->d_xc, p->n_xc);
      else if (planes)
        k_xc<uint16_t, false, true><<<grid, 256, 0, s>>>(f16, stride, F, pn.ny, pn.z_off, chunks, p->d_xc, p->n_xc);
      else
        k_xc<uint16_t, false, false><<<grid, 256, 0, s>>>(f16, stride, F, pn.ny, pn.z_off, chunks, p->d_xc, p->n_xc);
    } else if (dtype == MI_DT_U8) {
      const uint8_t *f8 = (const uint8_t *)frames;
      if (planes)
        k_xc<uint8_t, false, true><<<grid, 256, 0, s>>>(f8, stride, F, pn.ny, pn.z_off, chunks, p->d_xc, p->n_xc);
      else
        k_xc<uint8_t, false, false><<<grid, 256, 0, s>>>(f8, stride, F, pn.ny, pn.z_off, chunks, p->d_xc, p->n_xc);
    } else {
      return set_error(MI_E_ARG, "launch_xc: dtype %d does not fit u16 staging", dtype);
    }
  } else {
    if (p->encoding == MI_ENC_MMA) return set_error(MI_E_UNSUPPORTED, "launch_xc: MMA plans stage 8/16-bit frames only");
    switch (dtype) {
      case MI_DT_U8: xcf_launch<uint8_t>(p, pn, frames, F, stride, s); break;
      case MI_DT_U16: xcf_launch<uint16_t>(p, pn, frames, F, stride, s); break;
      case MI_DT_U32: xcf_launch<uint32_t>(p, pn, frames, F, stride, s); break;
      case MI_DT_I64: xcf_launch<int64_t>(p, pn, frames, F, stride, s); break;
      case MI_DT_F32: xcf_launch<float>(p, pn, frames, F, stride, s); break;
      case MI_DT_F64: xcf_launch<double>(p, pn, frames, F, stride, s); break;
      case MI_DT_I32: xcf_launch<int32_t>(p, pn, frames, F, stride, s); break;
      default: return set_error(MI_E_ARG, "launch_xc: unknown dtype %d", dtype);
    }
  }
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

}  // namespace mi
