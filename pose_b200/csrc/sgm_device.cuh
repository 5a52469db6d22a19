// sgm_device.cuh - device-side helpers shared by the stereo kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "collinea_sgm.h"

namespace csgm {

constexpr int kInvalidCost = 512;  // CensusSgm.java:11
constexpr int kMaxDirections = 16;

// Direction table of CensusSgm.java:421; entries 8..15 are the 16-path extension.
__host__ __device__ inline void direction(int index, int& dx, int& dy) {
  const int table[16][2] = {{1, 0},  {-1, 0}, {0, 1},   {0, -1},  {1, 1},  {-1, 1},
                            {1, -1}, {-1, -1}, {1, 2},  {2, 1},   {-1, 2}, {-2, 1},
                            {1, -2}, {2, -1},  {-1, -2}, {-2, -1}};
  dx = table[index][0];
  dy = table[index][1];
}

// Number of independent lines of direction (dx, dy): the pixels whose predecessor (x-dx, y-dy)
// lies outside the image start a line.
__host__ __device__ inline int64_t line_count(int w, int h, int dx, int dy) {
  int ax = dx < 0 ? -dx : dx, ay = dy < 0 ? -dy : dy;
  return (int64_t)ay * w + (int64_t)ax * (h - ay);
}

// Start pixel of line `line` of direction (dx, dy).
__host__ __device__ inline void line_start(int64_t line, int w, int h, int dx, int dy, int& x,
                                           int& y) {
  int ay = dy < 0 ? -dy : dy;
  if (line < (int64_t)ay * w) {
    int row = (int)(line / w);
    x = (int)(line % w);
    y = dy > 0 ? row : h - 1 - row;
    return;
  }
  int64_t rest = line - (int64_t)ay * w;
  int span = h - ay;
  int c = (int)(rest / span), r = (int)(rest % span);
  x = dx > 0 ? c : w - 1 - c;
  y = dy > 0 ? ay + r : (dy < 0 ? h - 1 - ay - r : r);
}

// StereoCost.pathP2 (StereoCost.java:44-48).
__device__ __forceinline__ int path_p2(int p1, int p2, int scale, int gray_cur, int gray_prev) {
  if (scale == 0) return p2;
  int difference = abs(gray_cur - gray_prev);
  int v = (int)(((long long)p2 * scale) / (scale + difference));
  return max(p1 + 1, v);
}

// java.lang.Math.round(double) for the values the matcher rounds: floor(v + 1/2) exactly.
__device__ __forceinline__ long long java_round(double v) {
  double f = floor(v);
  return (long long)(__dsub_rn(v, f) >= 0.5 ? __dadd_rn(f, 1.0) : f);
}

// java.lang.Math.round(float): the double sum of a float and 0.5 is exact.
__device__ __forceinline__ int java_round_float(float v) {
  return (int)floor(__dadd_rn((double)v, 0.5));
}

__device__ __forceinline__ unsigned long long shfl_min_u64(unsigned long long v) {
#pragma unroll
  for (int offset = 16; offset > 0; offset >>= 1) {
    unsigned long long o = __shfl_xor_sync(0xffffffffu, v, offset);
    v = o < v ? o : v;
  }
  return v;
}

// Warp-aggregated counters: one atomic per warp.
__device__ __forceinline__ void warp_add(unsigned long long* counter, int value) {
  if (!counter) return;
  int total = __reduce_add_sync(0xffffffffu, (unsigned)value);
  if ((threadIdx.x & 31) == 0 && total) atomicAdd(counter, (unsigned long long)total);
}

// Selection counters in device memory (order of csgm_stats' first six fields).
struct DeviceStats {
  unsigned long long lower_boundary_rejected;
  unsigned long long full_interval_pixels;
  unsigned long long boundary_rejected;
  unsigned long long upper_boundary_rejected;
  unsigned long long ambiguity_rejected;
  unsigned long long selected;
  unsigned long long lr_rejected;
  unsigned long long pad;
};

}  // namespace csgm
