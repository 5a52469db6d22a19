// postfilter.cu - the post-filters of CensusSgm.computeRecorded on the GPU
// (CensusSgm.java:203-272): median of the LR-checked map, post-median reciprocity, ZNCC
// photometric gate and speckle removal, with their counters and reason codes.
//
//  * median_kernel<N>: a thread per pixel gathers the finite values of its N x N window (clipped
//    to the image), sorts them and takes element n/2 (CensusSgm.java:557-573); in edge-preserving
//    mode a pixel whose classic median moved it by max_change or more takes instead the median of
//    the window values within max_change of it whose gray values are within the edge threshold of
//    its own (:576-601).
//  * gate_kernel: reciprocity against the right view (:604-612), then ZNCC of the gray windows
//    at the sub-pixel match with linear interpolation (:615-644).  FP64 in the reference's order
//    with explicitly rounded operations (no contraction), so the scores are bit-identical.
//  * Speckles (:647-681) are the connected components of the graph whose edges join finite
//    neighbours (4 or 8) whose values differ by at most range.  A lock-free union-find labels
//    them: every union links the larger root under the smaller one with atomicCAS, so a parent
//    index never exceeds its child's and every find terminates; a flatten pass, a size count and
//    a removal pass follow.  Components smaller than the minimum become NaN.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>

#include "collinea_sgm.h"
#include "pipeline.h"
#include "sgm_device.cuh"

namespace csgm {
namespace {

// Counters of one call: post-median LR, photometric, speckle, valid.
struct PostCounts {
  unsigned long long lr, photometric, speckle, valid;
};

__device__ __forceinline__ void count_add(unsigned long long* dst, unsigned v) {
  const unsigned total = __reduce_add_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0 && total) atomicAdd(dst, (unsigned long long)total);
}

// Sorts v[0..n) ascending (finite values only; equal values are the same bits).
__device__ __forceinline__ void sort_values(float* v, int n) {
  for (int i = 1; i < n; i++) {
    const float key = v[i];
    int j = i - 1;
    while (j >= 0 && v[j] > key) {
      v[j + 1] = v[j];
      j--;
    }
    v[j + 1] = key;
  }
}

template <int N>
__global__ void median_kernel(const float* a, const uint8_t* gray, int w, int h, int classic,
                              double max_change, int edge_threshold, float* out) {
  constexpr int r = N / 2;
  float v[N * N];
  const int64_t n = (int64_t)w * h;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int y = (int)(p / w), x = (int)(p - (int64_t)y * w);
    const float center = a[p];
    if (!isfinite(center)) {
      out[p] = center;
      continue;
    }
    const int y0 = max(0, y - r), y1 = min(h - 1, y + r);
    const int x0 = max(0, x - r), x1 = min(w - 1, x + r);
    int k = 0;
    for (int yy = y0; yy <= y1; yy++)
      for (int xx = x0; xx <= x1; xx++) {
        const float value = a[(int64_t)yy * w + xx];
        if (isfinite(value)) v[k++] = value;
      }
    sort_values(v, k);
    float m = v[k / 2];
    if (!classic && !((double)fabsf(__fsub_rn(m, center)) < max_change)) {
      const int g = gray[p];
      k = 0;
      for (int yy = y0; yy <= y1; yy++)
        for (int xx = x0; xx <= x1; xx++) {
          const int64_t q = (int64_t)yy * w + xx;
          const float value = a[q];
          if (isfinite(value) && (double)fabsf(__fsub_rn(value, center)) <= max_change &&
              (edge_threshold == 0 || abs((int)gray[q] - g) <= edge_threshold))
            v[k++] = value;
        }
      if (k > 0) {
        sort_values(v, k);
        m = v[k / 2];
      }
    }
    out[p] = m;
  }
}

// ZNCC of the left window at (x, y) and the right window at x - disparity over `channels`
// interleaved channels (CensusSgm.java:615-644: one gray channel, or B, G, R in colour-distance
// mode); -1 where a window leaves the image or is too flat.
__device__ double zncc_score(const uint8_t* a, const uint8_t* b, int w, int h, int x, int y,
                             double disparity, int r, int channels) {
  const double target = __dsub_rn((double)x, disparity);
  const int bx = (int)floor(target);
  const double fraction = __dsub_rn(target, (double)bx);
  if (x - r < 0 || x + r >= w || y - r < 0 || y + r >= h || bx - r < 0 || bx + r + 1 >= w)
    return -1;
  const int n = (2 * r + 1) * (2 * r + 1);
  const double keep = __dsub_rn(1.0, fraction);
  const double dn = (double)n;
  double covariance = 0, var_a = 0, var_b = 0;
  for (int channel = 0; channel < channels; channel++) {
    double sa = 0, sb = 0, saa = 0, sbb = 0, sab = 0;
    for (int dy = -r; dy <= r; dy++)
      for (int dx = -r; dx <= r; dx++) {
        const int64_t ai = ((int64_t)(y + dy) * w + x + dx) * channels + channel;
        const int64_t bi = ((int64_t)(y + dy) * w + bx + dx) * channels + channel;
        const double av = (double)a[ai];
        const double bv = __dadd_rn(__dmul_rn(keep, (double)b[bi]),
                                    __dmul_rn(fraction, (double)b[bi + channels]));
        sa = __dadd_rn(sa, av);
        sb = __dadd_rn(sb, bv);
        saa = __dadd_rn(saa, __dmul_rn(av, av));
        sbb = __dadd_rn(sbb, __dmul_rn(bv, bv));
        sab = __dadd_rn(sab, __dmul_rn(av, bv));
      }
    covariance = __dadd_rn(covariance, __dsub_rn(sab, __ddiv_rn(__dmul_rn(sa, sb), dn)));
    var_a = __dadd_rn(var_a, __dsub_rn(saa, __ddiv_rn(__dmul_rn(sa, sa), dn)));
    var_b = __dadd_rn(var_b, __dsub_rn(sbb, __ddiv_rn(__dmul_rn(sb, sb), dn)));
  }
  if (var_a < channels * n * 4 || var_b < channels * n * 4) return -1;
  const double product = __dmul_rn(var_a, var_b);
  return __ddiv_rn(covariance, __dsqrt_rn(product > 1e-12 ? product : 1e-12));
}

struct GateArgs {
  const uint8_t* left;   // images the gate correlates: gray, or interleaved BGR
  const uint8_t* right;
  const float* dr;
  float* checked;
  uint8_t* reasons;
  PostCounts* counts;
  int w, h, border, radius;
  double tolerance, correlation;
  int channels;  // 1 gray, 3 BGR
};

// Reciprocity (CensusSgm.java:604-612), then the photometric gate (:240-257).
__global__ void gate_kernel(const GateArgs g) {
  const int64_t n = (int64_t)g.w * g.h;
  unsigned lr = 0, photometric = 0;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const float d = g.checked[p];
    if (!isfinite(d)) continue;
    const int y = (int)(p / g.w), x = (int)(p - (int64_t)y * g.w);
    bool ok = y >= g.border && y < g.h - g.border;
    if (ok) {
      const int xr = java_round_float(__fsub_rn((float)x, d));
      ok = xr >= g.border && xr < g.w - g.border;
      if (ok) {
        const float other = g.dr[(int64_t)y * g.w + xr];
        ok = isfinite(other) && (double)fabsf(__fsub_rn(d, other)) <= g.tolerance;
      }
    }
    if (!ok) {
      g.checked[p] = __int_as_float(0x7fc00000);
      lr++;
      if (g.reasons) g.reasons[p] = 5;
      continue;
    }
    const double score =
        zncc_score(g.left, g.right, g.w, g.h, x, y, (double)d, g.radius, g.channels);
    if (score < g.correlation) {
      g.checked[p] = __int_as_float(0x7fc00000);
      photometric++;
      if (g.reasons) g.reasons[p] = 6;
    }
  }
  count_add(&g.counts->lr, lr);
  count_add(&g.counts->photometric, photometric);
}

// ---- speckles: connected components by union-find ----

__device__ __forceinline__ int find_root(const int* parent, int x) {
  // parent[x] <= x everywhere, so the walk ends; values read late are still ancestors.
  for (;;) {
    const int q = __ldcg(parent + x);
    if (q == x) return x;
    x = q;
  }
}

__device__ __forceinline__ void unite(int* parent, int a, int b) {
  for (;;) {
    a = find_root(parent, a);
    b = find_root(parent, b);
    if (a == b) return;
    if (a < b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicCAS(parent + a, a, b);  // larger root under the smaller one
    if (old == a) return;
    a = old;
  }
}

__global__ void speckle_init_kernel(const float* a, int64_t n, int* parent, int* size) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    parent[p] = isfinite(a[p]) ? (int)p : -1;
    size[p] = 0;
  }
}

// Links each finite pixel with its finite forward neighbours (right, below, and the two lower
// diagonals with 8-connectivity) whose values differ by at most range.
__global__ void speckle_union_kernel(const float* a, int w, int h, int connectivity, double range,
                                     int* parent) {
  const int64_t n = (int64_t)w * h;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const float v = a[p];
    if (!isfinite(v)) continue;
    const int y = (int)(p / w), x = (int)(p - (int64_t)y * w);
    auto link = [&](int xx, int yy) {
      if (xx < 0 || xx >= w || yy >= h) return;
      const int64_t q = (int64_t)yy * w + xx;
      const float u = a[q];
      if (isfinite(u) && (double)fabsf(__fsub_rn(u, v)) <= range) unite(parent, (int)p, (int)q);
    };
    link(x + 1, y);
    link(x, y + 1);
    if (connectivity == 8) {
      link(x - 1, y + 1);
      link(x + 1, y + 1);
    }
  }
}

__global__ void speckle_size_kernel(int64_t n, int* parent, int* size) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    if (parent[p] < 0) continue;
    const int root = find_root(parent, (int)p);
    parent[p] = root;
    atomicAdd(size + root, 1);
  }
}

// Removes the pixels of components smaller than minimum (minimum <= 1: none, parent unused) and
// counts the finite pixels left.
__global__ void speckle_remove_kernel(float* a, int64_t n, const int* parent, const int* size,
                                      int minimum, uint8_t* reasons, PostCounts* counts) {
  unsigned removed = 0, valid = 0;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    if (!isfinite(a[p])) continue;
    if (minimum > 1 && size[parent[p]] < minimum) {
      a[p] = __int_as_float(0x7fc00000);
      removed++;
      if (reasons) reasons[p] = 7;
    } else {
      valid++;
    }
  }
  count_add(&counts->speckle, removed);
  count_add(&counts->valid, valid);
}

int grid_for(int64_t n, int sm_count) {
  const int64_t blocks = (n + 255) / 256;
  return (int)std::min<int64_t>(std::max<int64_t>(blocks, 1), (int64_t)sm_count * 16);
}

int validate_post(const csgm_post* post, int w, int h) {
  if (!post) return fail(CSGM_E_INVALID, "NULL post-filter settings");
  if (w <= 0 || h <= 0 || (int64_t)w * h > INT32_MAX)
    return fail(CSGM_E_INVALID, "invalid image size %dx%d", w, h);
  if (post->median < 1 || post->median > 11 || post->median % 2 == 0)
    return fail(CSGM_E_INVALID, "--median must be odd in 1..11");
  if (post->median_edge_threshold < 0 || post->median_edge_threshold > 255 ||
      (post->speckle_connectivity != 4 && post->speckle_connectivity != 8))
    return fail(CSGM_E_INVALID,
                "Median edge threshold must be 0..255; speckle connectivity must be 4 or 8");
  if (!(post->median_max_change >= 0))
    return fail(CSGM_E_INVALID, "--median-max-change must be nonnegative");
  if (!(post->correlation >= -1 && post->correlation <= 1) || !(post->lr_threshold > 0) ||
      !(post->speckle_range >= 0) || post->speckle_size < 0 || post->correlation_window < 3 ||
      post->correlation_window > 15 || post->correlation_window % 2 == 0 || post->border < 0)
    return fail(CSGM_E_INVALID, "invalid correlation, LR threshold, speckle or border setting");
  return CSGM_OK;
}

template <int N>
void launch_median(const float* a, const uint8_t* gray, int w, int h, const csgm_post& post,
                   float* out, int sm_count, cudaStream_t stream) {
  median_kernel<N><<<grid_for((int64_t)w * h, sm_count), 256, 0, stream>>>(
      a, gray, w, h, post.median_classic, post.median_max_change, post.median_edge_threshold, out);
}

}  // namespace
}  // namespace csgm

using namespace csgm;

// The post-filters; with left_bgr / right_bgr the photometric gate correlates the three BGR
// channels (CensusSgm.java:222-224), while the edge-preserving median reads the gray left image.
static int postfilter_impl(csgm_session* s, const csgm_post* post, const uint8_t* left,
                           const uint8_t* right, const uint8_t* left_bgr,
                           const uint8_t* right_bgr, const float* disp_r, int32_t w, int32_t h,
                           float* checked, uint8_t* reasons, csgm_stats* stats) {
  if (!s) return fail(CSGM_E_INVALID, "NULL session");
  if (!left || !right || !disp_r || !checked)
    return fail(CSGM_E_INVALID, "NULL image, right-view or checked buffer");
  int rc = validate_post(post, w, h);
  if (rc) return rc;
  std::lock_guard<std::mutex> guard(s->lock);
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return cuda_fail(e, "Device selection");
  const int64_t n = (int64_t)w * h;
  Workspace& ws = s->workspace;
  cudaStream_t st = s->stream;
  int status = CSGM_OK;
  uint8_t* d_left = (uint8_t*)ws.get(kImgL, n, &status);
  uint8_t* d_right = d_left ? (uint8_t*)ws.get(kImgR, n, &status) : nullptr;
  float* d_dr = d_right ? (float*)ws.get(kDispR, n * 4, &status) : nullptr;
  float* d_checked = d_dr ? (float*)ws.get(kChecked, n * 4, &status) : nullptr;
  float* d_median = d_checked ? (float*)ws.get(kDispL, n * 4, &status) : nullptr;
  uint8_t* d_reasons = nullptr;
  if (d_median && reasons) d_reasons = (uint8_t*)ws.get(kReasons, n, &status);
  int* d_parent = (d_median && (!reasons || d_reasons)) ? (int*)ws.get(kCostL, n * 4, &status)
                                                        : nullptr;
  int* d_size = d_parent ? (int*)ws.get(kCostR, n * 4, &status) : nullptr;
  PostCounts* d_counts = d_size ? (PostCounts*)ws.get(kStats, sizeof(PostCounts), &status)
                                : nullptr;
  if (!d_counts) return status ? status : fail(CSGM_E_NOMEM, "post-filter workspace");
  const int channels = left_bgr ? 3 : 1;
  const uint8_t* photo_l = d_left;
  const uint8_t* photo_r = d_right;
  if (left_bgr) {
    uint8_t* bl = (uint8_t*)ws.get(kBgrL, 3 * n, &status);
    uint8_t* br = bl ? (uint8_t*)ws.get(kBgrR, 3 * n, &status) : nullptr;
    if (!br) return status;
    e = cudaMemcpyAsync(bl, left_bgr, 3 * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(br, right_bgr, 3 * n, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "post-filter BGR upload");
    photo_l = bl;
    photo_r = br;
  }

  e = cudaMemcpyAsync(d_left, left, n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_right, right, n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_dr, disp_r, n * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_checked, checked, n * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && reasons)
    e = cudaMemcpyAsync(d_reasons, reasons, n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_counts, 0, sizeof(PostCounts), st);
  if (e != cudaSuccess) return cuda_fail(e, "post-filter upload");

  const int grid = grid_for(n, s->sm_count);
  float* map = d_checked;
  if (post->median > 1) {  // CensusSgm.java:203-214
    switch (post->median) {
      case 3: launch_median<3>(d_checked, d_left, w, h, *post, d_median, s->sm_count, st); break;
      case 5: launch_median<5>(d_checked, d_left, w, h, *post, d_median, s->sm_count, st); break;
      case 7: launch_median<7>(d_checked, d_left, w, h, *post, d_median, s->sm_count, st); break;
      case 9: launch_median<9>(d_checked, d_left, w, h, *post, d_median, s->sm_count, st); break;
      default: launch_median<11>(d_checked, d_left, w, h, *post, d_median, s->sm_count, st); break;
    }
    map = d_median;
  }
  GateArgs g{photo_l, photo_r, d_dr, map, d_reasons, d_counts, w, h, post->border,
             post->correlation_window / 2, post->lr_threshold, post->correlation, channels};
  gate_kernel<<<grid, 256, 0, st>>>(g);
  const int minimum = post->speckle_size;
  speckle_init_kernel<<<grid, 256, 0, st>>>(map, n, d_parent, d_size);
  if (minimum > 1) {
    speckle_union_kernel<<<grid, 256, 0, st>>>(map, w, h, post->speckle_connectivity,
                                               post->speckle_range, d_parent);
    speckle_size_kernel<<<grid, 256, 0, st>>>(n, d_parent, d_size);
  }
  speckle_remove_kernel<<<grid, 256, 0, st>>>(map, n, d_parent, d_size, minimum, d_reasons,
                                              d_counts);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "post-filter kernel launch");
  s->profiler.launches += 4 + (post->median > 1) + 2 * (minimum > 1);

  PostCounts host{};
  e = cudaMemcpyAsync(checked, map, n * 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && reasons)
    e = cudaMemcpyAsync(reasons, d_reasons, n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&host, d_counts, sizeof host, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "GPU post-filter execution");
  if (stats) {
    stats->post_median_lr_rejected += (int64_t)host.lr;
    stats->photometric_rejected += (int64_t)host.photometric;
    stats->speckle_rejected = (int64_t)host.speckle;
    stats->valid += (int64_t)host.valid;
  }
  return CSGM_OK;
}

extern "C" int csgm_postfilter(csgm_session* s, const csgm_post* post, const uint8_t* left,
                               const uint8_t* right, const float* disp_r, int32_t w, int32_t h,
                               float* checked, uint8_t* reasons, csgm_stats* stats) {
  return postfilter_impl(s, post, left, right, nullptr, nullptr, disp_r, w, h, checked, reasons,
                         stats);
}

extern "C" int csgm_postfilter_color(csgm_session* s, const csgm_post* post, const uint8_t* left,
                                     const uint8_t* right, const uint8_t* left_bgr,
                                     const uint8_t* right_bgr, const float* disp_r, int32_t w,
                                     int32_t h, float* checked, uint8_t* reasons,
                                     csgm_stats* stats) {
  if (!left_bgr || !right_bgr)
    return fail(CSGM_E_INVALID, "Color-distance census requires interleaved BGR inputs");
  return postfilter_impl(s, post, left, right, left_bgr, right_bgr, disp_r, w, h, checked,
                         reasons, stats);
}
