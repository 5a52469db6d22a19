// color_census.cu - CensusSgm.colorCensus on the GPU (CensusSgm.java:302-332): the colour-distance
// census descriptors and texture mask of an interleaved BGR image, for --census-mode
// color-distance.  The reference computes them on the CPU and hands them to GpuSgm.match; here
// csgm_color_census produces them for csgm_match.
//
// A thread per pixel.  Bit k (window order, row-major, centre skipped) is set iff the Euclidean
// BGR distance to neighbour k is at least the mean distance over the window including the
// centre's zero; the pixel is textured iff the largest distance is at least 4.  Border pixels
// (closer than the window radius to an edge) keep zero descriptors and no texture.  The FP64
// sums, square roots and the division are explicitly rounded in the reference's order, so the
// descriptors are bit-identical.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "collinea_sgm.h"
#include "pipeline.h"
#include "stereo_kernels.h"

namespace csgm {
namespace {

__device__ __forceinline__ double bgr_distance(const uint8_t* bgr, int64_t q, int64_t c) {
  double squared = 0;
#pragma unroll
  for (int ch = 0; ch < 3; ch++) {
    const int d = (int)bgr[q + ch] - (int)bgr[c + ch];
    squared = __dadd_rn(squared, (double)(d * d));
  }
  return __dsqrt_rn(squared);
}

// valid (optional): the pair's validity mask, ANDed into the texture mask (CensusSgm.java:127-134).
__global__ void color_census_kernel(const uint8_t* bgr, const uint8_t* valid, int w, int h, int wx,
                                    int wy, int words, uint64_t* desc, uint8_t* tex) {
  const int rx = wx / 2, ry = wy / 2;
  const int64_t n = (int64_t)w * h;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int y = (int)(p / w), x = (int)(p - (int64_t)y * w);
    uint64_t bits[2] = {0, 0};
    uint8_t textured = 0;
    if (x >= rx && x < w - rx && y >= ry && y < h - ry) {
      const int64_t c = 3 * p;
      double total = 0, maximum = 0;
      for (int dy = -ry; dy <= ry; dy++)
        for (int dx = -rx; dx <= rx; dx++) {
          if (dx == 0 && dy == 0) continue;
          const double d = bgr_distance(bgr, 3 * ((int64_t)(y + dy) * w + x + dx), c);
          total = __dadd_rn(total, d);
          maximum = maximum > d ? maximum : d;
        }
      const double mean = __ddiv_rn(total, (double)(wx * wy));
      textured = maximum >= 4;
      int k = 0;
      for (int dy = -ry; dy <= ry; dy++)
        for (int dx = -rx; dx <= rx; dx++) {
          if (dx == 0 && dy == 0) continue;
          const double d = bgr_distance(bgr, 3 * ((int64_t)(y + dy) * w + x + dx), c);
          if (d >= mean) bits[k >> 6] |= 1ull << (k & 63);
          k++;
        }
    }
    for (int j = 0; j < words; j++) desc[(int64_t)j * n + p] = bits[j];
    tex[p] = textured && (valid == nullptr || valid[p] != 0);
  }
}

}  // namespace

cudaError_t launch_color_census(const uint8_t* bgr, const uint8_t* valid, int w, int h, int wx,
                                int wy, uint64_t* desc, uint8_t* tex, int sm_count,
                                cudaStream_t stream) {
  const int64_t n = (int64_t)w * h, blocks = (n + 255) / 256;
  const int grid = (int)(blocks < (int64_t)sm_count * 16 ? blocks : (int64_t)sm_count * 16);
  color_census_kernel<<<grid, 256, 0, stream>>>(bgr, valid, w, h, wx, wy, (wx * wy - 1 + 63) / 64,
                                               desc, tex);
  return cudaGetLastError();
}

}  // namespace csgm

using namespace csgm;

extern "C" int csgm_color_census(csgm_session* s, const uint8_t* bgr, int32_t w, int32_t h,
                                 int32_t window_x, int32_t window_y, uint64_t* descriptors,
                                 uint8_t* textured) {
  if (!s) return fail(CSGM_E_INVALID, "NULL session");
  if (!bgr || !descriptors || !textured) return fail(CSGM_E_INVALID, "NULL image or output");
  if (w <= 0 || h <= 0 || (int64_t)w * h * 3 > INT32_MAX)
    return fail(CSGM_E_INVALID, "invalid image size %dx%d", w, h);
  if (window_x < 3 || window_y < 3 || window_x % 2 == 0 || window_y % 2 == 0 ||
      window_x * window_y - 1 > 128)
    return fail(CSGM_E_INVALID, "census window must be odd, at least 3, at most 128 bits");
  const int words = (window_x * window_y - 1 + 63) / 64;
  std::lock_guard<std::mutex> guard(s->lock);
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return cuda_fail(e, "Device selection");
  const int64_t n = (int64_t)w * h;
  int status = CSGM_OK;
  uint8_t* d_bgr = (uint8_t*)s->workspace.get(kImgL, 3 * n, &status);
  uint64_t* d_desc = d_bgr ? (uint64_t*)s->workspace.get(kDescL, 8 * n * words, &status) : nullptr;
  uint8_t* d_tex = d_desc ? (uint8_t*)s->workspace.get(kTexL, n, &status) : nullptr;
  if (!d_tex) return status ? status : fail(CSGM_E_NOMEM, "colour census workspace");
  cudaStream_t st = s->stream;
  e = cudaMemcpyAsync(d_bgr, bgr, 3 * n, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "colour census upload");
  e = launch_color_census(d_bgr, nullptr, w, h, window_x, window_y, d_desc, d_tex, s->sm_count, st);
  if (e != cudaSuccess) return cuda_fail(e, "colour census launch");
  s->profiler.launches++;
  e = cudaMemcpyAsync(descriptors, d_desc, 8 * n * words, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(textured, d_tex, n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "GPU colour census");
  return CSGM_OK;
}
