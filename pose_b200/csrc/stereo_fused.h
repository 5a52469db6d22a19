// stereo_fused.h - fast path for D <= 256: both views aggregated by fused sweeps.
#pragma once

#include <cstdint>

#include "pipeline.h"
#include "sgm_device.cuh"

namespace csgm {

struct FusedViews {
  const uint64_t* desc_l;
  const uint64_t* desc_r;
  const uint8_t* tex_l;
  const uint8_t* tex_r;
  const uint8_t* gray_l;
  const uint8_t* gray_r;
  float* disp_l;
  float* disp_r;
  // Per view (0 left, 1 right), each optional.
  uint8_t* reasons[2];   // reason codes of the pixels decided by the selection
  uint8_t* boundary[2];  // searchBoundary flags of full-interval pixels
  DeviceStats* stats[2]; // selection counters, added to
  int32_t* summary[2];   // winners records [n][6]
};

bool fused_supported(const csgm_params& p);
// The tuning a fused run uses: the requested values where valid for these parameters (rows per
// block 4, 8, or 12 at 65..128 disparities; line warps 0, 4 or 8 within the shared memory of a
// CTA, 8/16 paths only; line slack 10..1000), otherwise the environment's or the defaults.
SweepTuning resolve_tuning(const csgm_params& p, const SweepTuning& requested);
size_t fused_workspace_bytes(const csgm_params& p, int w, int h, const SweepTuning& tuning);
// Queues both views on ctx.stream; *error_flag receives the device address of the sweep's error
// word (non-zero after a bounded wait ran out).
int run_views_fused(Context& ctx, const csgm_params& p, const FusedViews& v, int w, int h,
                    int** error_flag);

}  // namespace csgm
