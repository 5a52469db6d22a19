// stereo_kernels.h - kernel argument blocks and launchers of the stereo matcher.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sgm_device.cuh"

namespace csgm {

struct CensusImage {
  const uint8_t* img;
  const uint8_t* valid;  // optional validity mask ANDed into the texture mask
  uint64_t* desc;        // [words][n]
  uint8_t* tex;          // [n]
};

struct CensusArgs {
  CensusImage image[2];
  int w, h, wx, wy, words;
};

struct CostArgs {
  const uint64_t* desc_a;
  const uint64_t* desc_b;
  const uint8_t* tex_a;
  const uint8_t* tex_b;
  const uint8_t* gray_a;
  const uint8_t* gray_b;
  uint16_t* out;  // [n][D], 512 = invalid
  int w, h, D, min_disparity, reverse, wx, wy, words, mode, weight, ad_cap, grad_cap, bits;
  // Strip of rows y0 .. y0+rows-1 (rows 0 = the whole image); out is indexed strip-locally.
  int y0 = 0, rows = 0;
  // The listed pixels pixels[i] (i < npixels) only, cost row i (compact SGM's exact pass).
  const int32_t* pixels = nullptr;
  int npixels = 0;
};

struct PathArgs {
  const uint16_t* cost;  // [n][D]
  const uint8_t* tex;    // predecessor must be textured
  const uint8_t* gray;   // edge-aware P2 of the matching view
  int w, h, D, dx, dy, p1, p2, edge_scale;
  // Strip of rows y0 .. y0+rows-1 (rows 0 = the whole image); cost and sum are strip-local.
  // Streamed strips carry path states across strip edges: carry_in holds the states of the |dy|
  // rows of the previous strip in path order that this strip's first pixels follow, carry_out
  // receives this strip's |dy| rows that the next strip follows, both [|dy|][w][D] int32.
  int y0 = 0, rows = 0;
  const int32_t* carry_in = nullptr;
  int32_t* carry_out = nullptr;
};

struct SelectArgs {
  const uint16_t* cost;
  float* out;
  int32_t* summary;  // optional [n][6]
  uint8_t* reasons;  // optional
  uint8_t* boundary; // optional
  DeviceStats* stats;  // optional
  int w, h, D, wx, wy, min_disparity;
  double uniqueness;
  // Strip of rows y0 .. y0+rows-1 (rows 0 = the whole image): cost and sum are strip-local, the
  // outputs are indexed by image pixel.
  int y0 = 0, rows = 0;
  // Compact SGM's exact pass: the listed pixels pixels[i] (i < npixels) only, their cost and sum
  // in row i.
  const int32_t* pixels = nullptr;
  int npixels = 0;
};

// Compact SGM (GpuCandidateStereo.java:53-167, kernel hooks :401-479): per path, a few separated
// proposals per pixel; then the exact aggregate at every proposal and its neighbours and a lower
// bound of the aggregate elsewhere; pixels whose outcome these certify are selected from them, the
// others are aggregated and selected exactly.
// No cost volume is kept: the path walks compute each pixel's costs from the descriptors.
struct EsgmArgs {
  CostArgs cost;  // the view's cost inputs (out unused)
  int directions, p1, p2, edge_scale;
  uint16_t* cand;     // [n][C] proposals (65535: none), C = directions x pool
  uint16_t* compact;  // [n][C][3] aggregates at proposal - 1, proposal, proposal + 1
  // [n] lower bound of the aggregate away from every proposal; bit 31: no such disparity
  uint32_t* outside;
  int C, pool;
  // Exact pass: the full path cost of a pixel whose slot lies in [slot_lo, slot_hi) is added to
  // row slot - slot_lo of sum ([slot_hi - slot_lo][D]).
  const int32_t* slots;
  uint16_t* sum;
  int32_t slot_lo = 0, slot_hi = 0;
  // 2: blocks with blockIdx.y >= directions walk the mirrored view (images, masks and grays
  // swapped, reverse flipped) into the arrays that follow the first view's (cand + n C,
  // compact + 3 n C, outside + n, slots + n); in the exact pass that view's listed pixels in
  // [slot_lo2, slot_hi2) go to sum2.
  int views = 1;
  uint16_t* sum2 = nullptr;
  int32_t slot_lo2 = 0, slot_hi2 = 0;
};

struct EsgmSelectArgs {
  CostArgs cost;  // validity of the disparities
  const uint16_t* cand;
  const uint16_t* compact;
  const uint32_t* outside;
  SelectArgs sel;     // outputs, counters and the selection parameters
  int C;
  int32_t* slots;     // [n] index among the unresolved pixels, -1 when certified
  int32_t* pixels;    // [n] the unresolved pixels, in slot order
  int32_t* count;     // unresolved pixels so far
};

struct LrArgs {
  const float* dl;
  const float* dr;
  float* out;
  uint8_t* reasons;
  DeviceStats* stats;
  int w, h, wx, wy;
  double threshold;
};

// StereoCost.value (StereoCost.java:50-90) for matching pixel p and target q.
__device__ __forceinline__ int cell_cost(const CostArgs& a, int64_t p, int64_t q, int64_t n) {
  int hamming = __popcll(a.desc_a[p] ^ a.desc_b[q]);
  if (a.words > 1) hamming += __popcll(a.desc_a[n + p] ^ a.desc_b[n + q]);
  if (a.mode == CSGM_COST_CENSUS) return hamming;
  if (a.mode == CSGM_COST_AD_CENSUS || a.mode == CSGM_COST_CENSUS_GRADIENT) {
    int difference, cap;
    if (a.mode == CSGM_COST_AD_CENSUS) {
      difference = abs((int)a.gray_a[p] - (int)a.gray_b[q]);
      cap = a.ad_cap;
    } else {
      int w = a.w;
      int ax = (int)a.gray_a[p + 1] - (int)a.gray_a[p - 1];
      int ay = (int)a.gray_a[p + w] - (int)a.gray_a[p - w];
      int bx = (int)a.gray_b[q + 1] - (int)a.gray_b[q - 1];
      int by = (int)a.gray_b[q + w] - (int)a.gray_b[q - w];
      difference = abs(ax - bx) + abs(ay - by);
      cap = a.grad_cap;
    }
    int denominator = 1000 * cap;
    return (a.weight * hamming * cap + (1000 - a.weight) * min(difference, cap) * a.bits +
            denominator / 2) /
           denominator;
  }
  // ZNCC: int64 window sums, FP64 correlation with Java's operation order and rounding.
  int rx = a.wx / 2, ry = a.wy / 2, count = a.wx * a.wy, w = a.w;
  long long sa = 0, sb = 0, saa = 0, sbb = 0, sab = 0;
  for (int dy = -ry; dy <= ry; dy++)
    for (int dx = -rx; dx <= rx; dx++) {
      int x = a.gray_a[p + dy * w + dx], y = a.gray_b[q + dy * w + dx];
      sa += x;
      sb += y;
      saa += x * x;
      sbb += y * y;
      sab += x * y;
    }
  long long va = count * saa - sa * sa, vb = count * sbb - sb * sb;
  if (va <= 0 || vb <= 0) return kInvalidCost;
  double correlation =
      __ddiv_rn((double)(count * sab - sa * sb), sqrt(__dmul_rn((double)va, (double)vb)));
  double clamped = fmax(-1.0, fmin(1.0, correlation));
  return (int)java_round(__dmul_rn(__dmul_rn(__dsub_rn(1.0, clamped), 0.5), (double)a.bits));
}


cudaError_t launch_census_texture(const CensusArgs& a, int images, cudaStream_t stream);
// CensusSgm.colorCensus of an interleaved BGR image (color_census.cu), texture ANDed with valid.
cudaError_t launch_color_census(const uint8_t* bgr, const uint8_t* valid, int w, int h, int wx,
                                int wy, uint64_t* desc, uint8_t* tex, int sm_count,
                                cudaStream_t stream);
cudaError_t launch_cost_volume(const CostArgs& a, int sm_count, cudaStream_t stream);
cudaError_t launch_paths_line(const PathArgs& a, void* sum, int sum_bytes, int sm_count,
                              cudaStream_t stream);
cudaError_t launch_esgm_paths(const EsgmArgs& a, int phase, int sm_count, cudaStream_t stream);
cudaError_t launch_esgm_select(const EsgmSelectArgs& a, int sm_count, cudaStream_t stream);
cudaError_t launch_winners(const SelectArgs& a, const void* sum, int sum_bytes, int sm_count,
                           cudaStream_t stream);
cudaError_t launch_lr_check(const LrArgs& a, int sm_count, cudaStream_t stream);
// Sets *differ to 1 when the device buffers a and b (bytes long) are not identical; *differ is
// cleared by the caller and is never cleared here.
cudaError_t launch_bytes_differ(const void* a, const void* b, size_t bytes, int* differ,
                                int sm_count, cudaStream_t stream);

}  // namespace csgm
