// stereo_fused.cu - fused sweep kernels (fast path).
#include "stereo_fused.h"

namespace csgm {

bool fused_supported(const csgm_params&) { return false; }
size_t fused_workspace_bytes(const csgm_params&, int, int) { return 0; }
int run_views_fused(Context&, const csgm_params&, const FusedViews&, int, int) {
  return fail(CSGM_E_UNSUPPORTED, "fused path not built");
}

}  // namespace csgm
