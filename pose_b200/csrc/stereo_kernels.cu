// stereo_kernels.cu - general stereo kernels for sm_100a: census + texture masks, the cost
// volume (four cost modes), path aggregation with one warp per line (any D up to 4096, any
// direction set, uint16 or uint32 aggregate), winner selection with subpixel refinement, and the
// left-right check.  These are the general path; stereo_fused.cu holds the fast path for D <= 256.
//
// Reference semantics (paths relative to the reference project root):
//   census / texture     src/main/java/sgm/CensusSgm.java:523-555
//   cost modes           src/main/java/sgm/StereoCost.java:50-90
//   aggregation          src/main/java/sgm/CensusSgm.java:421-459
//   selection            src/main/java/sgm/CensusSgm.java:460-515, GpuStereo.java:631-687,758-769
//   left-right check     src/main/java/sgm/CensusSgm.java:181-201
#include "stereo_kernels.h"

#include <cfloat>
#include <climits>

namespace csgm {

// ---------------------------------------------------------------------------------------------
// Census descriptors and texture masks (CensusSgm.java:523-555), both images in one launch.
// blockIdx.z selects the image.  A 32x8 block stages its pixels plus the window apron in shared
// memory; border pixels get zero descriptors and are untextured.
constexpr int kCensusBx = 32, kCensusBy = 8, kCensusMaxR = 5;

// RX, RY: window radii (compile time, so every bit position is a constant).
template <int RX, int RY>
__global__ void __launch_bounds__(kCensusBx * kCensusBy) census_texture_kernel(CensusArgs args) {
  constexpr int TW = kCensusBx + 2 * RX, TH = kCensusBy + 2 * RY;
  __shared__ uint8_t tile[TH][TW];
  const CensusImage& im = args.image[blockIdx.z];
  const int w = args.w, h = args.h;
  const int bx0 = blockIdx.x * kCensusBx, by0 = blockIdx.y * kCensusBy;
  for (int i = threadIdx.y * kCensusBx + threadIdx.x; i < TW * TH; i += kCensusBx * kCensusBy) {
    const int ty = i / TW, tx = i % TW;
    const int gx = bx0 - RX + tx, gy = by0 - RY + ty;
    tile[ty][tx] = (gx >= 0 && gx < w && gy >= 0 && gy < h) ? im.img[(int64_t)gy * w + gx] : 0;
  }
  __syncthreads();
  const int x = bx0 + threadIdx.x, y = by0 + threadIdx.y;
  if (x >= w || y >= h) return;
  const int64_t n = (int64_t)w * h, p = (int64_t)y * w + x;
  uint64_t w0 = 0, w1 = 0;
  uint8_t textured = 0;
  if (x >= RX && x < w - RX && y >= RY && y < h - RY) {
    const uint8_t* c = &tile[threadIdx.y + RY][threadIdx.x + RX];
    const int center = *c;
    int low = 255, high = 0;
#pragma unroll
    for (int yy = -RY; yy <= RY; yy++) {
#pragma unroll
      for (int xx = -RX; xx <= RX; xx++) {
        const int v = c[yy * TW + xx];
        low = min(low, v);
        high = max(high, v);
        // Row-major bit index over the window, skipping the centre (CensusSgm.java:545-552).
        const int idx = (yy + RY) * (2 * RX + 1) + (xx + RX);
        const int center_idx = RY * (2 * RX + 1) + RX;
        if (idx == center_idx) continue;
        const int bit = idx < center_idx ? idx : idx - 1;
        const uint64_t set = v < center ? 1ull : 0ull;
        if (bit < 64)
          w0 |= set << bit;
        else
          w1 |= set << (bit - 64);
      }
    }
    textured = high - low >= 4 && (im.valid == nullptr || im.valid[p] != 0);
  }
  im.desc[p] = w0;
  if (args.words > 1) im.desc[n + p] = w1;
  im.tex[p] = textured;
}

// One cost cell per thread-lane: a warp covers one pixel's disparities (coalesced uint16 stores).
// The cost of pixel (x, y) at disparity index k: 512 when the pixel or its target lies within the
// census window's half-size of the border or is untextured, else StereoCost.value.
__device__ __forceinline__ int cost_at(const CostArgs& a, int x, int y, int k, int64_t n) {
  const int rx = a.wx / 2, ry = a.wy / 2, w = a.w;
  const int64_t p = (int64_t)y * w + x;
  if (!(x >= rx && x < w - rx && y >= ry && y < a.h - ry && a.tex_a[p])) return kInvalidCost;
  const long long disparity = (long long)a.min_disparity + k;
  const long long target = (long long)x + (a.reverse ? disparity : -disparity);
  if (target < rx || target >= w - rx) return kInvalidCost;
  const int64_t q = (int64_t)y * w + target;
  return a.tex_b[q] ? cell_cost(a, p, q, n) : kInvalidCost;
}

__global__ void cost_volume_kernel(CostArgs a) {
  int w = a.w, h = a.h, D = a.D;
  int64_t n = (int64_t)w * h;
  int lane = threadIdx.x & 31;
  int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t first = (int64_t)a.y0 * w;
  const int64_t count = a.pixels ? a.npixels : a.rows ? (int64_t)a.rows * w : n;
  for (int64_t local = warp; local < count; local += warps) {
    const int64_t p = a.pixels ? a.pixels[local] : first + local;
    const int x = (int)(p % w), y = (int)(p / w);
    uint16_t* out = a.out + local * D;
    for (int k = lane; k < D; k += 32) out[k] = (uint16_t)cost_at(a, x, y, k, n);
  }
}

// ---------------------------------------------------------------------------------------------
// Path aggregation, one warp per line (CensusSgm.java:421-459; the reference GPU kernel walks a
// line per work-group in the same way, GpuStereo.java:732-757).  The line state lives in shared
// memory as int32, so any D <= 4096 and any penalty fit.  Each lane owns disparities k = lane +
// 32 j.  The aggregate is read-modify-written once per direction.
template <typename SumT>
__global__ void paths_line_kernel(PathArgs a, SumT* __restrict__ sum) {
  extern __shared__ int smem[];
  int D = a.D, w = a.w, h = a.h;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  int* prev = smem + (size_t)warp * 2 * D;
  int* cur = prev + D;
  // Lines of the strip (y strip-local); the whole image is one strip when rows is 0.
  const int rows = a.rows ? a.rows : h, y0 = a.y0;
  const int ady = a.dy < 0 ? -a.dy : a.dy;
  int64_t lines = line_count(w, rows, a.dx, a.dy);
  for (int64_t line = (int64_t)blockIdx.x * warps + warp; line < lines;
       line += (int64_t)gridDim.x * warps) {
    int x, y;
    line_start(line, w, rows, a.dx, a.dy, x, y);
    int64_t prev_p = -1;
    if (a.carry_in && y >= 0 && y < rows) {
      // The line's first pixel follows a pixel of the previous strip in path order: its state
      // is carry row j (the previous strip's rows that this strip's first |dy| rows follow).
      const int px = x - a.dx, yp = y - a.dy, gy = y0 + yp;
      if (px >= 0 && px < w && gy >= 0 && gy < h && (yp < 0 || yp >= rows)) {
        const int j = yp < 0 ? yp + ady : yp - rows;
        const int32_t* src = a.carry_in + ((int64_t)j * w + px) * D;
        for (int k = lane; k < D; k += 32) prev[k] = src[k];
        __syncwarp();
        prev_p = (int64_t)gy * w + px;
      }
    }
    while (x >= 0 && x < w && y >= 0 && y < rows) {
      int64_t p = (int64_t)(y0 + y) * w + x;
      bool has = prev_p >= 0 && a.tex[prev_p];
      int minimum = 0, local_p2 = a.p2;
      if (has) {
        int m = INT_MAX;
        for (int k = lane; k < D; k += 32) m = min(m, prev[k]);
        minimum = (int)__reduce_min_sync(0xffffffffu, (unsigned)m);
        local_p2 = path_p2(a.p1, a.p2, a.edge_scale, a.gray[p], a.gray[prev_p]);
      }
      const int64_t local = (int64_t)y * w + x;
      const uint16_t* c = a.cost + local * D;
      SumT* s = sum + local * D;
      // Rows the next strip in path order follows: the last |dy| (dy > 0) or first |dy| (dy < 0).
      int32_t* out = nullptr;
      if (a.carry_out && a.dy != 0) {
        const int j = a.dy > 0 ? y - (rows - ady) : y;
        if (j >= 0 && j < ady) out = a.carry_out + ((int64_t)j * w + x) * D;
      }
      for (int k = lane; k < D; k += 32) {
        int v = c[k];
        if (has) {
          int t = min(prev[k], minimum + local_p2);
          if (k > 0) t = min(t, prev[k - 1] + a.p1);
          if (k + 1 < D) t = min(t, prev[k + 1] + a.p1);
          v += t - minimum;
        }
        cur[k] = v;
        s[k] = (SumT)(s[k] + (SumT)v);
        if (out) out[k] = v;
      }
      __syncwarp();
      int* swap = prev;
      prev = cur;
      cur = swap;
      prev_p = p;
      x += a.dx;
      y += a.dy;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------------------------
// cost_at for the Census cost (the only one compact SGM plans for), with the pixel's own terms
// (border, texture, descriptor words) taken once per pixel instead of once per disparity.
// The target of disparity k is x0 + step * k (step = +1 for the right view, -1 for the left).
struct CensusPixel {
  bool inside;
  uint64_t w0, w1;
  const uint64_t *b0, *b1;  // the target row's descriptor words
  const uint8_t* tb;        // the target row's texture flags
  long long x0;
  int step, lo, hi;  // valid targets lo <= t < hi
  __device__ __forceinline__ CensusPixel(const CostArgs& a, int x, int y, int64_t n) {
    const int rx = a.wx / 2, ry = a.wy / 2;
    const int64_t row = (int64_t)y * a.w, p = row + x;
    inside = x >= rx && x < a.w - rx && y >= ry && y < a.h - ry && a.tex_a[p];
    w0 = inside ? a.desc_a[p] : 0;
    w1 = inside && a.words > 1 ? a.desc_a[n + p] : 0;
    b0 = a.desc_b + row;
    b1 = a.desc_b + n + row;
    tb = a.tex_b + row;
    step = a.reverse ? 1 : -1;
    x0 = (long long)x + (long long)step * a.min_disparity;
    lo = rx;
    hi = a.w - rx;
  }
  __device__ __forceinline__ int at(const CostArgs& a, int k) const {
    const long long t = x0 + (long long)step * k;
    if (!inside || t < lo || t >= hi || !tb[t]) return kInvalidCost;
    int hamming = __popcll(w0 ^ b0[t]);
    if (a.words > 1) hamming += __popcll(w1 ^ b1[t]);
    return hamming;
  }
};

// *at += v as a 32-bit atomic add on the word that holds *at (exact while no 16-bit sum wraps).
__device__ __forceinline__ void add_u16(uint16_t* at, unsigned v) {
  const uintptr_t address = (uintptr_t)at;
  atomicAdd((unsigned*)(address & ~(uintptr_t)3), v << ((address & 2) ? 16 : 0));
}

// Compact SGM (GpuCandidateStereo.java:53-167, the path kernel hooks :401-479).  One warp per line
// as in paths_line_kernel, each pixel's costs computed from the descriptors (no cost volume), and
// every direction of a phase in one launch (blockIdx.y = direction, plus the direction count for
// a pair's mirrored view); at every pixel, after the path state L:
//  PHASE 0: `pool` separated proposals of the path: the valid disparity of least L (ties: the
//   smaller), then the least among those more than one away from every proposal so far;
//  PHASE 1 (all directions' proposals known): L at every proposal - 1, proposal, proposal + 1 is
//   added to the pixel's compact aggregates, and the least L over the valid disparities no
//   proposal covers (within one) to the pixel's lower bound of the aggregate there (or the bound
//   is marked empty when every valid disparity is covered, which no direction changes);
//  PHASE 2 (exact pass): L is added to the full aggregate row of each listed pixel.
// The directions' additions to a pixel are atomic 32-bit adds of a 16-bit value shifted into its
// half of the word.  They are exact in any order: the plan allows 16-bit aggregates only while
// directions x (512 + P2) <= 65535, and one path's L never exceeds 512 + P2, so no 16-bit sum
// carries into its neighbour (the reference adds the directions one after another with the same
// wrap-free values, GpuCandidateStereo.java:437-444).
template <int PHASE>
__global__ void esgm_paths_kernel(EsgmArgs a) {
  extern __shared__ int smem[];
  CostArgs ca = a.cost;
  const int D = ca.D, w = ca.w, h = ca.h, C = a.C;
  const int64_t n = (int64_t)w * h;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  const int dir = blockIdx.y % a.directions;
  if (blockIdx.y >= a.directions) {  // the mirrored view
    const uint64_t* d = ca.desc_a;
    ca.desc_a = ca.desc_b;
    ca.desc_b = d;
    const uint8_t* t = ca.tex_a;
    ca.tex_a = ca.tex_b;
    ca.tex_b = t;
    t = ca.gray_a;
    ca.gray_a = ca.gray_b;
    ca.gray_b = t;
    ca.reverse = !ca.reverse;
    a.cand += n * C;
    a.compact += 3 * n * C;
    a.outside += n;
    a.slots += n;
    a.sum = a.sum2;
    a.slot_lo = a.slot_lo2;
    a.slot_hi = a.slot_hi2;
  }
  int dx, dy;
  direction(dir, dx, dy);
  // StereoCost.pathP2 by the gray difference of a pixel and its predecessor.
  __shared__ int p2_of[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) p2_of[i] = path_p2(a.p1, a.p2, a.edge_scale, i, 0);
  __syncthreads();
  int* prev = smem + (size_t)warp * 4 * D;
  int* cur = prev + D;
  int* cost = cur + D;
  int* covered = cost + D;  // PHASE 1: proposals within one of k (cleared after each pixel)
  const int64_t lines = line_count(w, h, dx, dy);
  if (PHASE == 1)
    for (int k = lane; k < D; k += 32) covered[k] = 0;
  __syncwarp();
  for (int64_t line = (int64_t)blockIdx.x * warps + warp; line < lines;
       line += (int64_t)gridDim.x * warps) {
    int x, y;
    line_start(line, w, h, dx, dy, x, y);
    int64_t prev_p = -1;
    while (x >= 0 && x < w && y >= 0 && y < h) {
      const int64_t p = (int64_t)y * w + x;
      const bool has = prev_p >= 0 && ca.tex_a[prev_p];
      int minimum = 0, local_p2 = a.p2;
      if (has) {
        int m = INT_MAX;
        for (int k = lane; k < D; k += 32) m = min(m, prev[k]);
        minimum = (int)__reduce_min_sync(0xffffffffu, (unsigned)m);
        local_p2 = p2_of[abs((int)ca.gray_a[p] - (int)ca.gray_a[prev_p])];
      }
      // PHASE 1: proposal lane + 32 r of the pixel in prop[r] (C <= 64).
      int prop[2] = {65535, 65535};
      if (PHASE == 1)
        for (int r = 0; r < 2; r++)
          if (lane + 32 * r < C) {
            prop[r] = a.cand[p * C + lane + 32 * r];
            for (int k = max(prop[r] - 1, 0); k <= prop[r] + 1 && k < D; k++)
              atomicAdd(&covered[k], 1);
          }
      const CensusPixel pixel(ca, x, y, n);
      for (int k = lane; k < D; k += 32) {
        const int c = pixel.at(ca, k);
        int v = c;
        if (has) {
          int t = min(prev[k], minimum + local_p2);
          if (k > 0) t = min(t, prev[k - 1] + a.p1);
          if (k + 1 < D) t = min(t, prev[k + 1] + a.p1);
          v += t - minimum;
        }
        cur[k] = v;
        cost[k] = c;
      }
      __syncwarp();
      if constexpr (PHASE == 0) {
        // Keys (L << 12) | k order as the reference's L * (D + 1) + k (k < D <= 4096, and
        // L <= 512 + P2 <= 65535 within the 16-bit bound).
        int chosen[4] = {65535, 65535, 65535, 65535};
#pragma unroll
        for (int choice = 0; choice < 4; choice++) {
          if (choice >= a.pool) break;
          unsigned key = 0xffffffffu;
          for (int k = lane; k < D; k += 32)
            if (cost[k] != kInvalidCost) {
              bool eligible = true;
#pragma unroll
              for (int j = 0; j < choice; j++) eligible &= abs(k - chosen[j]) > 1;
              if (eligible) key = min(key, ((unsigned)cur[k] << 12) | (unsigned)k);
            }
          key = __reduce_min_sync(0xffffffffu, key);
          chosen[choice] = key == 0xffffffffu ? 65535 : (int)(key & 4095u);
          if (lane == 0) a.cand[p * C + dir * a.pool + choice] = (uint16_t)chosen[choice];
        }
      } else if constexpr (PHASE == 1) {
        for (int base = 0; base < 3 * C; base += 32) {  // uniform trip count: shuffles below
          const int j = base + lane, source = min(j, 3 * C - 1) / 3;
          const int low = __shfl_sync(0xffffffffu, prop[0], source & 31);
          const int high = __shfl_sync(0xffffffffu, prop[1], source & 31);
          const int k = (source < 32 ? low : high) + j % 3 - 1;
          if (j < 3 * C && k >= 0 && k < D) add_u16(a.compact + p * C * 3 + j, (unsigned)cur[k]);
        }
        unsigned lower = 0x7fffffffu;
        for (int k = lane; k < D; k += 32)
          if (cost[k] != kInvalidCost && covered[k] == 0) lower = min(lower, (unsigned)cur[k]);
        lower = __reduce_min_sync(0xffffffffu, lower);
        if (lane == 0) {
          if (lower == 0x7fffffffu)
            atomicOr(a.outside + p, 0x80000000u);
          else
            atomicAdd(a.outside + p, lower);
        }
        __syncwarp();
        for (int r = 0; r < 2; r++)
          if (lane + 32 * r < C)
            for (int k = max(prop[r] - 1, 0); k <= prop[r] + 1 && k < D; k++)
              atomicSub(&covered[k], 1);
      } else {
        const int slot = a.slots[p];
        if (slot >= a.slot_lo && slot < a.slot_hi) {
          uint16_t* row = a.sum + (int64_t)(slot - a.slot_lo) * D;
          for (int k = lane; k < D; k += 32) add_u16(row + k, (unsigned)cur[k]);
        }
      }
      __syncwarp();
      int* swap = prev;
      prev = cur;
      cur = swap;
      prev_p = p;
      x += dx;
      y += dy;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------------------------
// Winner selection (CensusSgm.java:460-515) with the winners record of GpuStereo.java:758-769
// and the arithmetic of the host select (GpuStereo.java:644-686).  One warp per pixel.
__device__ void select_pixel(const SelectArgs& a, int64_t p, int best, int value, int second,
                             int before, int after, int flags, unsigned long long* counts) {
  if (best < 0) return;
  bool full = flags == 3;
  if (full) {
    counts[1]++;
    if (a.boundary) a.boundary[p] = 4;
  }
  if (best == 0 || best == a.D - 1) {
    counts[2]++;
    if (a.reasons) a.reasons[p] = 2;
    if (full && best == 0) {
      counts[0]++;
      if (a.boundary) a.boundary[p] |= 1;
    }
    if (full && best == a.D - 1) {
      counts[3]++;
      if (a.boundary) a.boundary[p] |= 2;
    }
    return;
  }
  if (second != INT_MAX) {
    double slack = fmax(1.0, __dmul_rn((double)value, a.uniqueness));
    if ((double)(second - value) <= slack) {
      counts[4]++;
      if (a.reasons) a.reasons[p] = 3;
      return;
    }
  }
  double offset = 0;
  if (before >= 0 && after >= 0) {
    double curvature =
        __dsub_rn(__dadd_rn((double)before, (double)after), __dmul_rn(2.0, (double)value));
    if (curvature > 0) {
      double o = __ddiv_rn(__dmul_rn(0.5, __dsub_rn((double)before, (double)after)), curvature);
      offset = fmax(-0.5, fmin(0.5, o));
    }
  }
  a.out[p] = __double2float_rn(__dadd_rn((double)(a.min_disparity + best), offset));
  counts[5]++;
  if (a.reasons) a.reasons[p] = 0;
}

template <typename SumT>
__global__ void winners_kernel(SelectArgs a, const SumT* __restrict__ sum) {
  int w = a.w, h = a.h, D = a.D, rx = a.wx / 2, ry = a.wy / 2;
  int64_t n = (int64_t)w * h;
  int lane = threadIdx.x & 31;
  int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long counts[6] = {0, 0, 0, 0, 0, 0};
  const int64_t first = (int64_t)a.y0 * w;
  const int64_t count = a.pixels ? a.npixels : a.rows ? (int64_t)a.rows * w : n;
  for (int64_t local = warp; local < count; local += warps) {
    // A listed pixel (compact SGM's exact pass) has its cost and sum in row `local`.
    const int64_t p = a.pixels ? a.pixels[local] : first + local;
    int x = (int)(p % w), y = (int)(p / w);
    const uint16_t* c = a.cost + local * D;
    const SumT* s = sum + local * D;
    int flags = (c[0] != kInvalidCost ? 1 : 0) | (c[D - 1] != kInvalidCost ? 2 : 0);
    bool region = x >= rx && x < w - rx && y >= ry && y < h - ry;
    int best = -1, value = INT_MAX, second = INT_MAX, before = -1, after = -1;
    if (region) {
      unsigned long long key = ~0ull;
      for (int k = lane; k < D; k += 32)
        if (c[k] != kInvalidCost) {
          unsigned long long kk = ((unsigned long long)(uint32_t)s[k] << 32) | (uint32_t)k;
          key = kk < key ? kk : key;
        }
      key = shfl_min_u64(key);
      if (key != ~0ull) {
        best = (int)(key & 0xffffffffu);
        value = (int)(key >> 32);
        unsigned m = INT_MAX;
        for (int k = lane; k < D; k += 32)
          if (abs(k - best) > 1 && c[k] != kInvalidCost) m = min(m, (unsigned)s[k]);
        second = (int)__reduce_min_sync(0xffffffffu, m);
        if (best > 0 && c[best - 1] != kInvalidCost) before = (int)s[best - 1];
        if (best + 1 < D && c[best + 1] != kInvalidCost) after = (int)s[best + 1];
      }
    }
    if (lane == 0) {
      if (a.summary) {
        int32_t* r = a.summary + 6 * p;
        r[0] = best;
        r[1] = value;
        r[2] = second;
        r[3] = before;
        r[4] = after;
        r[5] = flags;
      }
      a.out[p] = __int_as_float(0x7fc00000);
      if (region) select_pixel(a, p, best, value, second, before, after, flags, counts);
    }
  }
  if (lane == 0 && a.stats) {
    if (counts[0]) atomicAdd(&a.stats->lower_boundary_rejected, counts[0]);
    if (counts[1]) atomicAdd(&a.stats->full_interval_pixels, counts[1]);
    if (counts[2]) atomicAdd(&a.stats->boundary_rejected, counts[2]);
    if (counts[3]) atomicAdd(&a.stats->upper_boundary_rejected, counts[3]);
    if (counts[4]) atomicAdd(&a.stats->ambiguity_rejected, counts[4]);
    if (counts[5]) atomicAdd(&a.stats->selected, counts[5]);
  }
}

// ---------------------------------------------------------------------------------------------
// Compact SGM selection (the esgm_select kernel, GpuCandidateStereo.java:448-478, and the
// certification of execute, :78-100).  A thread per pixel: the winners record from the compact
// aggregates (best = least aggregate over the proposals, ties to the smaller disparity; before /
// after its neighbours; second the least over the compact cells more than one away), then the
// outcome is certified when the lower bound elsewhere exceeds the best and every known other
// aggregate does, and the uniqueness test is decided either way by the known values.  A certified
// pixel is selected at once; the others are listed for the exact pass.
__global__ void esgm_select_kernel(EsgmSelectArgs a) {
  const SelectArgs& s = a.sel;
  const int w = s.w, h = s.h, D = s.D, C = a.C, rx = s.wx / 2, ry = s.wy / 2;
  const int64_t n = (int64_t)w * h;
  unsigned long long counts[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(p % w), y = (int)(p / w);
    auto valid = [&](int k) {
      return k >= 0 && k < D && cost_at(a.cost, x, y, k, n) != kInvalidCost;
    };
    const uint16_t* cand = a.cand + p * C;
    const uint16_t* compact = a.compact + p * C * 3;
    int best = -1, value = INT_MAX, second = INT_MAX, before = -1, after = -1, owner = -1;
    for (int j = 0; j < C; j++) {
      const int k = cand[j], v = compact[3 * j + 1];
      if (k < D && (v < value || (v == value && (best < 0 || k < best)))) {
        best = k;
        value = v;
        owner = j;
      }
    }
    if (owner >= 0) {
      if (valid(best - 1)) before = compact[3 * owner];
      if (valid(best + 1)) after = compact[3 * owner + 2];
      for (int j = 0; j < 3 * C; j++) {
        const int k = (int)cand[j / 3] + j % 3 - 1;
        if (abs(k - best) > 1 && valid(k)) second = min(second, (int)compact[j]);
      }
    }
    const int flags = (valid(0) ? 1 : 0) | (valid(D - 1) ? 2 : 0);
    bool trusted = true;
    if (best >= 0) {
      const unsigned bound = a.outside[p];
      const long long lower = (bound & 0x80000000u) ? 65535 : min(bound, 65535u);
      const bool winner = lower > value && (before < 0 || before > value) &&
                          (after < 0 || after > value) && second > value;
      const double margin = fmax(1.0, value * s.uniqueness);
      trusted = winner && (best == 0 || best == D - 1 || (double)second - (double)value <= margin ||
                           (double)(lower - value) > margin);
    }
    s.out[p] = __int_as_float(0x7fc00000);
    if (trusted) {
      a.slots[p] = -1;
      if (s.summary) {
        int32_t* r = s.summary + 6 * p;
        r[0] = best;
        r[1] = value;
        r[2] = second;
        r[3] = before;
        r[4] = after;
        r[5] = flags;
      }
      if (x >= rx && x < w - rx && y >= ry && y < h - ry)
        select_pixel(s, p, best, value, second, before, after, flags, counts);
    } else {
      const int slot = atomicAdd(a.count, 1);
      a.slots[p] = slot;
      a.pixels[slot] = (int32_t)p;
    }
  }
  if (s.stats) {
#pragma unroll
    for (int i = 0; i < 6; i++)
      for (int o = 16; o > 0; o /= 2) counts[i] += __shfl_down_sync(0xffffffffu, counts[i], o);
    if ((threadIdx.x & 31) == 0) {
      if (counts[0]) atomicAdd(&s.stats->lower_boundary_rejected, counts[0]);
      if (counts[1]) atomicAdd(&s.stats->full_interval_pixels, counts[1]);
      if (counts[2]) atomicAdd(&s.stats->boundary_rejected, counts[2]);
      if (counts[3]) atomicAdd(&s.stats->upper_boundary_rejected, counts[3]);
      if (counts[4]) atomicAdd(&s.stats->ambiguity_rejected, counts[4]);
      if (counts[5]) atomicAdd(&s.stats->selected, counts[5]);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Left-right check (CensusSgm.java:181-201).
__global__ void lr_check_kernel(LrArgs a) {
  int64_t n = (int64_t)a.w * a.h;
  int rx = a.wx / 2, ry = a.wy / 2;
  int rejected = 0;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    int x = (int)(p % a.w), y = (int)(p / a.w);
    float result = __int_as_float(0x7fc00000);
    if (x >= rx && x < a.w - rx && y >= ry && y < a.h - ry) {
      float d = a.dl[p];
      if (isfinite(d)) {
        int xr = java_round_float(__fsub_rn((float)x, d));
        if (xr < rx || xr >= a.w - rx) {
          if (a.reasons) a.reasons[p] = 4;
        } else {
          float other = a.dr[(int64_t)y * a.w + xr];
          if (isfinite(other) && (double)fabsf(__fsub_rn(d, other)) <= a.threshold)
            result = d;
          else {
            rejected++;
            if (a.reasons) a.reasons[p] = 4;
          }
        }
      }
    }
    a.out[p] = result;
  }
  if (a.stats) {
    int lane = threadIdx.x & 31;
    unsigned total = __reduce_add_sync(0xffffffffu, (unsigned)rejected);
    if (lane == 0 && total) atomicAdd(&a.stats->lr_rejected, (unsigned long long)total);
  }
}

// ---------------------------------------------------------------------------------------------
// Launchers.
static int grid_for(int64_t work, int threads, int max_blocks) {
  int64_t blocks = (work + threads - 1) / threads;
  if (blocks < 1) blocks = 1;
  return (int)(blocks < max_blocks ? blocks : max_blocks);
}

cudaError_t launch_census_texture(const CensusArgs& a, int images, cudaStream_t stream) {
  dim3 block(kCensusBx, kCensusBy);
  dim3 grid((a.w + kCensusBx - 1) / kCensusBx, (a.h + kCensusBy - 1) / kCensusBy, images);
  const int rx = a.wx / 2, ry = a.wy / 2;
  if (rx < 1 || rx > kCensusMaxR || ry < 1 || ry > kCensusMaxR) return cudaErrorInvalidValue;
  using Kernel = void (*)(CensusArgs);
  // [rx - 1][ry - 1]
  static const Kernel table[5][5] = {
      {census_texture_kernel<1, 1>, census_texture_kernel<1, 2>, census_texture_kernel<1, 3>,
       census_texture_kernel<1, 4>, census_texture_kernel<1, 5>},
      {census_texture_kernel<2, 1>, census_texture_kernel<2, 2>, census_texture_kernel<2, 3>,
       census_texture_kernel<2, 4>, census_texture_kernel<2, 5>},
      {census_texture_kernel<3, 1>, census_texture_kernel<3, 2>, census_texture_kernel<3, 3>,
       census_texture_kernel<3, 4>, census_texture_kernel<3, 5>},
      {census_texture_kernel<4, 1>, census_texture_kernel<4, 2>, census_texture_kernel<4, 3>,
       census_texture_kernel<4, 4>, census_texture_kernel<4, 5>},
      {census_texture_kernel<5, 1>, census_texture_kernel<5, 2>, census_texture_kernel<5, 3>,
       census_texture_kernel<5, 4>, census_texture_kernel<5, 5>}};
  table[rx - 1][ry - 1]<<<grid, block, 0, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_cost_volume(const CostArgs& a, int sm_count, cudaStream_t stream) {
  int64_t n = a.pixels ? a.npixels : (int64_t)a.w * (a.rows ? a.rows : a.h);
  cost_volume_kernel<<<grid_for(n * 32, 256, sm_count * 32), 256, 0, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_paths_line(const PathArgs& a, void* sum, int sum_bytes, int sm_count,
                              cudaStream_t stream) {
  const int warps = 4;
  size_t shared = (size_t)warps * 2 * a.D * sizeof(int);
  int64_t lines = line_count(a.w, a.rows ? a.rows : a.h, a.dx, a.dy);
  int grid = grid_for(lines, warps, sm_count * 64);
  if (sum_bytes == 2) {
    if (shared > 48 * 1024)
      cudaFuncSetAttribute(paths_line_kernel<uint16_t>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shared);
    paths_line_kernel<uint16_t><<<grid, warps * 32, shared, stream>>>(a, (uint16_t*)sum);
  } else {
    if (shared > 48 * 1024)
      cudaFuncSetAttribute(paths_line_kernel<uint32_t>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shared);
    paths_line_kernel<uint32_t><<<grid, warps * 32, shared, stream>>>(a, (uint32_t*)sum);
  }
  return cudaGetLastError();
}

cudaError_t launch_esgm_paths(const EsgmArgs& a, int phase, int sm_count, cudaStream_t stream) {
  const int warps = a.cost.D > 2048 ? 2 : 4;  // 4 D-int rows per warp within 227 KB
  const size_t shared = (size_t)warps * 4 * a.cost.D * sizeof(int);
  int64_t lines = 0;
  for (int d = 0; d < a.directions; d++) {
    int dx, dy;
    direction(d, dx, dy);
    lines = std::max(lines, line_count(a.cost.w, a.cost.h, dx, dy));
  }
  const dim3 grid(grid_for(lines, warps, sm_count * 64), a.directions * a.views);
  auto kernel = phase == 0 ? esgm_paths_kernel<0>
                : phase == 1 ? esgm_paths_kernel<1>
                             : esgm_paths_kernel<2>;
  if (shared > 48 * 1024)
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shared);
  kernel<<<grid, warps * 32, shared, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_esgm_select(const EsgmSelectArgs& a, int sm_count, cudaStream_t stream) {
  const int64_t n = (int64_t)a.sel.w * a.sel.h;
  const int grid = grid_for(n, 256, sm_count * 16);
  esgm_select_kernel<<<grid, 256, 0, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_winners(const SelectArgs& a, const void* sum, int sum_bytes, int sm_count,
                           cudaStream_t stream) {
  int64_t n = a.pixels ? a.npixels : (int64_t)a.w * (a.rows ? a.rows : a.h);
  int grid = grid_for(n * 32, 256, sm_count * 16);
  if (sum_bytes == 2)
    winners_kernel<uint16_t><<<grid, 256, 0, stream>>>(a, (const uint16_t*)sum);
  else
    winners_kernel<uint32_t><<<grid, 256, 0, stream>>>(a, (const uint32_t*)sum);
  return cudaGetLastError();
}

// 16-byte words where both buffers allow them (workspace buffers are 256-byte aligned), bytes for
// the tail; one flag store per thread that found a difference.
__global__ void bytes_differ_kernel(const uint8_t* a, const uint8_t* b, size_t bytes, int* differ) {
  const size_t words = bytes / 16;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  bool diff = false;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) {
    const uint4 x = __ldcs((const uint4*)a + i), y = __ldcs((const uint4*)b + i);
    diff |= (x.x != y.x) | (x.y != y.y) | (x.z != y.z) | (x.w != y.w);
  }
  if (blockIdx.x == 0 && threadIdx.x < bytes % 16) {
    const size_t i = words * 16 + threadIdx.x;
    diff |= a[i] != b[i];
  }
  if (diff) *differ = 1;
}

cudaError_t launch_bytes_differ(const void* a, const void* b, size_t bytes, int* differ,
                                int sm_count, cudaStream_t stream) {
  if (bytes == 0) return cudaSuccess;
  if (((uintptr_t)a | (uintptr_t)b) % 16) return cudaErrorMisalignedAddress;
  bytes_differ_kernel<<<grid_for((int64_t)(bytes / 16) + 1, 256, sm_count * 4), 256, 0, stream>>>(
      (const uint8_t*)a, (const uint8_t*)b, bytes, differ);
  return cudaGetLastError();
}

cudaError_t launch_lr_check(const LrArgs& a, int sm_count, cudaStream_t stream) {
  int64_t n = (int64_t)a.w * a.h;
  lr_check_kernel<<<grid_for(n, 256, sm_count * 8), 256, 0, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace csgm
