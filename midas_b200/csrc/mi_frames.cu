// mi_frames.cu -- frame preparation on the device: dark averaging and the hybrid
// (dtype code 6) socket payload.
//
//  * Dark: the mean of k dark frames per pixel in FP64, stored as float, as the GPU stream
//    server's main() does on the host (FF_HEDM/src/IntegratorFitPeaksGPUStream.cu:2191-2238;
//    average_dark_frames, packages/midas_integrate/midas_integrate/image.py:161-184).
//  * Hybrid payload: [u32 overflow count C][u16 base, ny*nz][i32 index, C][i64 value, C]
//    (ProcessImageGPU_Hybrid_Impl, IntegratorFitPeaksGPUStream.cu:1491-1560;
//    decode_hybrid_payload, image.py:83-123).  The payload crosses PCIe once, as it
//    arrived; one kernel expands the base to float and another overlays the overflow
//    values, (float)int64 like the reference.  The frame keeps raw counts: the caking
//    kernels subtract the dark, (float)raw - dark, when they stage it.
#include <stdint.h>
#include <string.h>

#include "mi_internal.h"

namespace mi {

template <typename T>
__global__ void k_mean_frames(const T *__restrict__ frames, int64_t stride, int n_frames, int64_t n_pix,
                              float *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_pix; i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int f = 0; f < n_frames; ++f) s += (double)frames[(int64_t)f * stride + i];
    out[i] = (float)(s / n_frames);
  }
}

__global__ void k_hybrid_base(const uint16_t *__restrict__ base, int64_t n_pix, float *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_pix; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)base[i];
}

// The index and value arrays follow the u16 base, so they are only 2-byte aligned (ny*nz
// may be odd): both are read as little-endian u16 halves.
__global__ void k_hybrid_overflow(const uint16_t *__restrict__ idx_h, const uint16_t *__restrict__ val_h,
                                  uint32_t count, int64_t n_pix, float *__restrict__ out, int *err) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int32_t idx = (int32_t)((uint32_t)idx_h[2 * i] | ((uint32_t)idx_h[2 * i + 1] << 16));
  const uint16_t *v = val_h + 4 * (size_t)i;
  const uint64_t u = (uint64_t)v[0] | ((uint64_t)v[1] << 16) | ((uint64_t)v[2] << 32) | ((uint64_t)v[3] << 48);
  if (idx < 0 || idx >= n_pix) {
    atomicExch(err, MI_E_RANGE);
    return;
  }
  out[idx] = (float)(int64_t)u;
}

template <typename T>
static void mean_launch(const void *frames, int64_t stride, int n_frames, int64_t n_pix, float *out, cudaStream_t s) {
  const unsigned grid = (unsigned)std::min<int64_t>((n_pix + 255) / 256, 148 * 16);
  k_mean_frames<T><<<grid, 256, 0, s>>>((const T *)frames, stride, n_frames, n_pix, out);
}

}  // namespace mi

using namespace mi;

extern "C" {

int mi_average_frames(const void *frames, int dtype, int64_t n_pixels, int n_frames, int64_t frame_stride,
                      float *out, void *stream) {
  if (!frames || !out) return set_error(MI_E_ARG, "mi_average_frames: null argument");
  if (n_frames <= 0 || n_pixels <= 0 || frame_stride < n_pixels)
    return set_error(MI_E_ARG, "mi_average_frames: need >= 1 frame, pixels > 0, frame_stride >= n_pixels");
  const cudaStream_t s = (cudaStream_t)stream;
  switch (dtype) {
    case MI_DT_U8: mean_launch<uint8_t>(frames, frame_stride, n_frames, n_pixels, out, s); break;
    case MI_DT_U16: mean_launch<uint16_t>(frames, frame_stride, n_frames, n_pixels, out, s); break;
    case MI_DT_U32: mean_launch<uint32_t>(frames, frame_stride, n_frames, n_pixels, out, s); break;
    case MI_DT_I64: mean_launch<int64_t>(frames, frame_stride, n_frames, n_pixels, out, s); break;
    case MI_DT_F32: mean_launch<float>(frames, frame_stride, n_frames, n_pixels, out, s); break;
    case MI_DT_F64: mean_launch<double>(frames, frame_stride, n_frames, n_pixels, out, s); break;
    case MI_DT_I32: mean_launch<int32_t>(frames, frame_stride, n_frames, n_pixels, out, s); break;
    default: return set_error(MI_E_ARG, "mi_average_frames: unknown dtype code %d", dtype);
  }
  MI_CUDA(cudaGetLastError());
  return MI_OK;
}

int mi_decode_hybrid(const void *payload, size_t payload_bytes, int ny, int nz, void *device_staging,
                     float *out, int *device_status, void *stream) {
  if (!payload || !device_staging || !out || !device_status)
    return set_error(MI_E_ARG, "mi_decode_hybrid: null argument");
  if (ny <= 0 || nz <= 0) return set_error(MI_E_ARG, "mi_decode_hybrid: bad shape %d x %d", ny, nz);
  const int64_t n_pix = (int64_t)ny * nz;
  if (payload_bytes < 4 + (size_t)n_pix * 2)
    return set_error(MI_E_ARG, "mi_decode_hybrid: payload of %zu bytes is smaller than count + base", payload_bytes);
  uint32_t count = 0;
  memcpy(&count, payload, 4);
  const size_t expect = 4 + (size_t)n_pix * 2 + (size_t)count * 12;
  if (payload_bytes != expect)
    return set_error(MI_E_ARG, "mi_decode_hybrid: payload is %zu bytes, count %u and %lld pixels need %zu",
                     payload_bytes, count, (long long)n_pix, expect);
  const cudaStream_t s = (cudaStream_t)stream;
  // the payload lands 4 bytes into the staging buffer, so the u16 base starts 8-byte aligned
  // (the index/value arrays after it are 2-byte aligned)
  uint8_t *st = (uint8_t *)device_staging;
  if ((uintptr_t)st % 16 != 0) return set_error(MI_E_ARG, "mi_decode_hybrid: staging must be 16-byte aligned");
  MI_CUDA(cudaMemcpyAsync(st + 4, payload, payload_bytes, cudaMemcpyHostToDevice, s));
  const uint16_t *base = (const uint16_t *)(st + 8);
  const unsigned grid = (unsigned)std::min<int64_t>((n_pix + 255) / 256, 148 * 16);
  k_hybrid_base<<<grid, 256, 0, s>>>(base, n_pix, out);
  MI_CUDA(cudaGetLastError());
  if (count > 0) {
    const uint16_t *idx = (const uint16_t *)(st + 8 + n_pix * 2);
    const uint16_t *val = idx + 2 * (size_t)count;
    k_hybrid_overflow<<<(count + 255) / 256, 256, 0, s>>>(idx, val, count, n_pix, out, device_status);
    MI_CUDA(cudaGetLastError());
  }
  return MI_OK;
}

}  // extern "C"
