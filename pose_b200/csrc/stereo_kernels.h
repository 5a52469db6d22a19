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
};

struct PathArgs {
  const uint16_t* cost;  // [n][D]
  const uint8_t* tex;    // predecessor must be textured
  const uint8_t* gray;   // edge-aware P2 of the matching view
  int w, h, D, dx, dy, p1, p2, edge_scale;
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

cudaError_t launch_census_texture(const CensusArgs& a, int images, cudaStream_t stream);
cudaError_t launch_cost_volume(const CostArgs& a, int sm_count, cudaStream_t stream);
cudaError_t launch_paths_line(const PathArgs& a, void* sum, int sum_bytes, int sm_count,
                              cudaStream_t stream);
cudaError_t launch_winners(const SelectArgs& a, const void* sum, int sum_bytes, int sm_count,
                           cudaStream_t stream);
cudaError_t launch_lr_check(const LrArgs& a, int sm_count, cudaStream_t stream);

}  // namespace csgm
