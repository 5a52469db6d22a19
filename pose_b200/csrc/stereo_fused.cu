// stereo_fused.cu - fast path of the matcher for D <= 256, 4/8 paths, uint16 aggregate.
//
// Reference semantics: cost CensusSgm.java:405-420 + StereoCost.java:50-90; aggregation
// CensusSgm.java:421-459; selection CensusSgm.java:460-515.  Results are bit-identical to the
// general kernels (stereo_kernels.cu) and to the CPU reference.
//
// Design (B200):
//  * cost_pair_kernel writes both views' cost volumes once, as uint8 [H][W][Dp] with
//    Dp = D rounded up to 64 and 0x80 marking the reference's invalid cost 512.
//  * sweep_kernel runs two wavefront streams in one launch, each over both views: "down"
//    processes rows top to bottom, pixels left to right, and owns the paths whose predecessor
//    lies above or to the left: (1,0), (0,1), (1,1), (-1,1); "up" is the same code on the image
//    mirrored in x and y and owns the four opposite paths.
//  * One CTA = R consecutive image rows; warp w holds row w of BOTH views (lanes 0-15 the left
//    view, lanes 16-31 the right view) and processes pixel x at step x + 2w, all warps in lock
//    step (one CTA barrier per step).  The (0,1), (1,1), (-1,1) path states of a row reach the
//    next row through a shared-memory ring; the (1,0) state stays in registers.  The last row of
//    a CTA also writes a global carry row that the next CTA of the stream reads
//    (release/acquire progress counter).
//  * Each stream stores its partial aggregate (uint16, 4 paths); the down stream marks cells whose
//    cost is invalid with 0xffff (a valid 4-path partial sum stays below 0x8000).  The streams
//    never wait for each other.
//  * wta_kernel streams both partial aggregates through shared memory (bulk copies), adds them
//    and runs winner-take-all, uniqueness and the parabolic sub-pixel step with one thread per
//    pixel.
//  * Disparities live in registers as packed uint16 pairs (REGS registers per lane per path,
//    16 lanes per view-row); the min-plus step uses the DPX instructions __vimin3_u16x2 /
//    __viaddmin_u16x2, and the per-row minima of two paths share one 16-lane shuffle butterfly
//    on packed uint16 pairs.
//  * Cost, partial-aggregate and carry slices are staged in shared memory by cp.async.bulk with
//    mbarrier completion (no multicast).  Every wait is bounded; a wait that runs out sets an
//    error flag that the host turns into CSGM_E_TIMEOUT.
//  * CTAs take tickets in launch order; a CTA only waits on lower tickets, so the schedule cannot
//    deadlock even when not every CTA is resident.
#include <climits>

#include "stereo_fused.h"
#include "stereo_kernels.h"

namespace csgm {

namespace {


__host__ __device__ inline int padded_d(int D) { return (D + 63) / 64 * 64; }

// ---------------------------------------------------------------------------------------------
// PTX helpers: shared-memory mbarriers and bulk copies (single CTA, no multicast).
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// PRMT in the generic mode: selector nibbles with bit 3 set replicate the selected byte's sign.
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
  return d;
}

// Bounded waits.  `error` short-circuits every later wait unless `shortcut` is false (the final
// drain, which must see its copies land).  A wait that runs out stores `code` (the wait site:
// 1 sweep cost chunk, 3 carry chunk, 4 selection tile, 5 drain; the sweep's producer warp
// stores 6 when it made no progress for the limit).
__device__ __forceinline__ void wait_bar(uint64_t* bar, uint32_t parity, int* error,
                                         long long limit, int code, bool shortcut = true) {
  long long start = clock64();
  while (!mbar_test(bar, parity)) {
    if (shortcut && *(volatile int*)error) break;
    if (clock64() - start > limit) {
      atomicExch(error, code);
      break;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Cost volumes of both views (uint8, 0x80 = invalid), StereoCost.value semantics
// (StereoCost.java:50-90) with CensusSgm.java:405-420 validity.  A CTA handles a segment of
// kCostSeg pixels of one row of one view: the segment's descriptors, textures and grays (with the
// disparity range of the target view) are staged in shared memory; one thread computes one
// pixel's Dp costs into a per-warp staging tile that the warp then writes out as coalesced
// 16-byte stores.  ZNCC (FP64 window sums) stays on the general per-cell path.
struct CostPairArgs {
  CostArgs view[2];  // per view: a = matching image, b = target image, reverse 0/1
  uint8_t* out[2];
  int Dp;
};

constexpr int kCostSeg = 128;  // pixels per CTA segment (4 warps x 32 pixels)

__global__ void __launch_bounds__(kCostSeg) cost_rows_kernel(CostPairArgs a) {
  extern __shared__ __align__(16) uint8_t csm[];
  const CostArgs& c = a.view[blockIdx.y];
  uint8_t* out = a.out[blockIdx.y];
  const int w = c.w, h = c.h, D = c.D, Dp = a.Dp, words = c.words;
  const int rx = c.wx / 2, ry = c.wy / 2;
  const int segs = (w + kCostSeg - 1) / kCostSeg;
  // Target columns of a segment [x0, x0+seg): left view q = x - d, right view q = x + d.
  const int span = kCostSeg + D;  // staged target pixels
  uint64_t* da = (uint64_t*)csm;                       // [words][kCostSeg]
  uint64_t* db = da + 2 * kCostSeg;                    // [words][span]
  uint8_t* stage = (uint8_t*)(db + 2 * span);          // [4 warps][32][Dp]
  uint8_t* ta = stage + 4 * 32 * Dp;                   // [kCostSeg]
  uint8_t* tb = ta + kCostSeg;                         // [span]
  uint8_t* ga = tb + span;                             // [3][kCostSeg + 2] rows y-1..y+1, x0-1..
  uint8_t* gb = ga + 3 * (kCostSeg + 2);               // [3][span + 2]
  const int64_t n = (int64_t)w * h;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t item = blockIdx.x; item < (int64_t)h * segs; item += gridDim.x) {
    const int y = (int)(item / segs), x0 = (int)(item % segs) * kCostSeg;
    const int qlo = c.reverse ? x0 + c.min_disparity : x0 - c.min_disparity - (D - 1);
    const bool row_inside = y >= ry && y < h - ry;
    __syncthreads();
    // Stage the segment.
    for (int i = threadIdx.x; i < kCostSeg; i += blockDim.x) {
      const int x = x0 + i;
      const bool ok = x < w;
      const int64_t p = (int64_t)y * w + x;
      for (int j = 0; j < words; j++) da[j * kCostSeg + i] = ok ? c.desc_a[j * n + p] : 0;
      ta[i] = ok ? c.tex_a[p] : 0;
    }
    for (int i = threadIdx.x; i < span; i += blockDim.x) {
      const int q = qlo + i;
      const bool ok = q >= 0 && q < w;
      const int64_t p = (int64_t)y * w + q;
      for (int j = 0; j < words; j++) db[j * span + i] = ok ? c.desc_b[j * n + p] : 0;
      tb[i] = ok ? c.tex_b[p] : 0;
    }
    if (c.mode == CSGM_COST_AD_CENSUS || c.mode == CSGM_COST_CENSUS_GRADIENT) {
      for (int i = threadIdx.x; i < 3 * (kCostSeg + 2); i += blockDim.x) {
        const int r = i / (kCostSeg + 2), x = x0 - 1 + i % (kCostSeg + 2), yy = y - 1 + r;
        ga[i] = (yy >= 0 && yy < h && x >= 0 && x < w) ? c.gray_a[(int64_t)yy * w + x] : 0;
      }
      for (int i = threadIdx.x; i < 3 * (span + 2); i += blockDim.x) {
        const int r = i / (span + 2), x = qlo - 1 + i % (span + 2), yy = y - 1 + r;
        gb[i] = (yy >= 0 && yy < h && x >= 0 && x < w) ? c.gray_b[(int64_t)yy * w + x] : 0;
      }
    }
    __syncthreads();
    // One pixel per thread.
    const int xi = threadIdx.x, x = x0 + xi;
    uint8_t* mine = stage + (warp * 32 + lane) * Dp;
    const bool inside = x < w && row_inside && x >= rx && x < w - rx && ta[xi];
    const int ax = inside && c.mode == CSGM_COST_CENSUS_GRADIENT
                       ? (int)ga[(kCostSeg + 2) + xi + 2] - (int)ga[(kCostSeg + 2) + xi] : 0;
    const int ay = inside && c.mode == CSGM_COST_CENSUS_GRADIENT
                       ? (int)ga[2 * (kCostSeg + 2) + xi + 1] - (int)ga[xi + 1] : 0;
    const int gav = inside ? (int)ga[(kCostSeg + 2) + xi + 1] : 0;
    const int denominator = 1000 * (c.mode == CSGM_COST_AD_CENSUS ? c.ad_cap : c.grad_cap);
    for (int k0 = 0; k0 < Dp; k0 += 4) {
      uint32_t packed = 0;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int k = k0 + j;
        int value = 0x80;
        if (inside && k < D) {
          const long long disparity = (long long)c.min_disparity + k;
          const long long target = (long long)x + (c.reverse ? disparity : -disparity);
          if (target >= rx && target < w - rx) {
            const int qi = (int)(target - qlo);
            if (tb[qi]) {
              int ham = __popcll(da[xi] ^ db[qi]);
              if (words > 1) ham += __popcll(da[kCostSeg + xi] ^ db[span + qi]);
              value = ham;
              if (c.mode == CSGM_COST_AD_CENSUS || c.mode == CSGM_COST_CENSUS_GRADIENT) {
                int difference, cap;
                if (c.mode == CSGM_COST_AD_CENSUS) {
                  difference = abs(gav - (int)gb[(span + 2) + qi + 1]);
                  cap = c.ad_cap;
                } else {
                  const int bx = (int)gb[(span + 2) + qi + 2] - (int)gb[(span + 2) + qi];
                  const int by = (int)gb[2 * (span + 2) + qi + 1] - (int)gb[qi + 1];
                  difference = abs(ax - bx) + abs(ay - by);
                  cap = c.grad_cap;
                }
                value = (c.weight * ham * cap + (1000 - c.weight) * min(difference, cap) * c.bits +
                         denominator / 2) /
                        denominator;
              }
            }
          }
        }
        packed |= (uint32_t)value << (8 * j);
      }
      *(uint32_t*)(mine + k0) = packed;
    }
    __syncwarp();
    // Coalesced write-out of the warp's 32 pixels (contiguous in memory).
    const int wx0 = x0 + warp * 32;
    const int npx = max(0, min(32, w - wx0));
    const int64_t base = ((int64_t)y * w + wx0) * Dp;
    const uint8_t* tile = stage + warp * 32 * Dp;
    for (int b = lane * 16; b < npx * Dp; b += 32 * 16)
      *(uint4*)(out + base + b) = *(const uint4*)(tile + b);
  }
}

size_t cost_rows_shared(int D, int Dp) {
  const int span = kCostSeg + D;
  return 2 * kCostSeg * 8 + 2 * (size_t)span * 8 + 4 * 32 * (size_t)Dp + kCostSeg + span +
         3 * (kCostSeg + 2) + 3 * ((size_t)span + 2) + 16;
}

// ZNCC and other fallbacks: one warp per pixel, lanes own contiguous disparity groups.
__global__ void cost_pair_kernel(CostPairArgs a) {
  const CostArgs& c = a.view[blockIdx.y];
  uint8_t* out = a.out[blockIdx.y];
  int w = c.w, h = c.h, D = c.D, Dp = a.Dp;
  int64_t n = (int64_t)w * h;
  int rx = c.wx / 2, ry = c.wy / 2;
  int lane = threadIdx.x & 31;
  int per = Dp / 32;  // 2..8 cells per lane
  int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t p = warp; p < n; p += warps) {
    int x = (int)(p % w), y = (int)(p / w);
    bool inside = x >= rx && x < w - rx && y >= ry && y < h - ry && c.tex_a[p];
    uint64_t packed = 0;
    for (int j = 0; j < per; j++) {
      int k = lane * per + j;
      int value = 0x80;
      if (inside && k < D) {
        long long disparity = (long long)c.min_disparity + k;
        long long target = (long long)x + (c.reverse ? disparity : -disparity);
        if (target >= rx && target < w - rx) {
          int64_t q = (int64_t)y * w + target;
          if (c.tex_b[q]) {
            int v = cell_cost(c, p, q, n);
            value = v == kInvalidCost ? 0x80 : v;
          }
        }
      }
      packed |= (uint64_t)value << (8 * j);
    }
    uint8_t* dst = out + p * Dp + lane * per;
    if (per == 8)
      *(uint64_t*)dst = packed;
    else if (per == 4)
      *(uint32_t*)dst = (uint32_t)packed;
    else if (per == 2)
      *(uint16_t*)dst = (uint16_t)packed;
    else
      for (int j = 0; j < per; j++) dst[j] = (uint8_t)(packed >> (8 * j));
  }
}

// ---------------------------------------------------------------------------------------------
struct SweepArgs {
  const uint8_t* cost[2];  // [H][W][Dp] per view
  const uint8_t* gray[2];  // matching-view image per view
  const uint8_t* tex[2];   // matching-view texture per view
  uint16_t* sum[2][2];     // [stream][view] partial aggregate [H][W][Dp]
  uint8_t* carry;          // [2 streams][nb][W][2 views][slot] bytes
  int* progress;           // [2][nb]
  int* ticket;
  int* error;
  int W, H, D, nb, Hp, p1, p2, edge_scale;
  long long timeout;
};

constexpr int kViews = 2;   // views per warp
constexpr int kLanes = 16;  // lanes per view-row

// Shared-memory layout (byte offsets), compile-time for a kernel instance.
template <int REGS, int K, int R>
struct SweepLayout {
  static constexpr int RING = 4;  // ring slots between consecutive rows
  static constexpr int NB = 4;    // cost chunk slots per row warp
  static constexpr int CS = 4;    // carry chunk slots
  static constexpr int Dp = 2 * kLanes * REGS;
  static constexpr int slot = 3 * Dp * 2 + 16;             // 3 paths x Dp uint16 + 4 minima
  static constexpr int vslot = kViews * slot;              // both views of one pixel
  static constexpr int lut = 0;                            // 256 x uint32
  static constexpr int bars = lut + 256 * 4;               // full[R][NB], carry_full[CS]
  static constexpr int counters = bars + (R * NB + CS) * 8;  // consumed[R], carry, published
  static constexpr int cost = (counters + (R + 2) * 4 + 127) / 128 * 128;
  static constexpr int ring = cost + R * NB * kViews * K * Dp;  // cost slots [R][NB][view][K][Dp]
  static constexpr int carry = ring + R * RING * vslot;          // row-to-row rings
  static constexpr int total = carry + CS * K * vslot;           // carry chunk slots
};

// The (P2' - P1) table of StereoCost.pathP2 for every |gray difference|, replicated to u16x2.
__device__ __forceinline__ uint32_t lut_value(int p1, int p2, int scale, int diff) {
  int v = scale == 0 ? p2 : max(p1 + 1, (int)(((long long)p2 * scale) / (scale + diff)));
  uint32_t d = (uint32_t)(v - p1);
  return d | (d << 16);
}

__device__ __forceinline__ int ld_acquire_cta(const int* p) {
  int v;
  asm volatile("ld.acquire.cta.shared::cta.b32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_cta(int* p, int v) {
  asm volatile("st.release.cta.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(p)), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// Barrier among the R row warps only (the producer warp does not take part).
__device__ __forceinline__ void rows_barrier(int threads) {
  asm volatile("bar.sync 1, %0;" ::"r"(threads) : "memory");
}

template <int REGS>
struct PathState {
  uint32_t v[REGS];
  uint32_t m;  // replicated minimum
};

// All paths of one pixel (each lane: its view's 2*REGS disparities), phase by phase so the
// independent per-path latency chains overlap.  Disparities >= D carry costs >= 0x8000, so they
// never win a minimum and never wrap (valid path costs stay below 16384 under the uint16 bound).
//   prev  predecessor path costs (zeros = no predecessor: the result is then the cost itself)
//   q     min(prev) + P2' - P1 (replicated), c the pixel's costs, p1x2 = P1 replicated.
template <int REGS, int NP>
__device__ __forceinline__ void paths_step(const PathState<REGS> (&prev)[NP],
                                           const uint32_t (&q)[NP], uint32_t p1x2,
                                           const uint32_t (&c)[REGS], int sl, int view,
                                           PathState<REGS> (&out)[NP]) {
  uint32_t below[NP], above[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    below[i] = __shfl_up_sync(0xffffffffu, prev[i].v[REGS - 1], 1, kLanes);
    above[i] = __shfl_down_sync(0xffffffffu, prev[i].v[0], 1, kLanes);
  }
#pragma unroll
  for (int i = 0; i < NP; i++) {
    if (sl == 0) below[i] = 0xffffffffu;
    if (sl == kLanes - 1) above[i] = 0xffffffffu;
    uint32_t e[REGS];
#pragma unroll
    for (int j = 0; j < REGS; j++)
      e[j] = __byte_perm(prev[i].v[j], j + 1 < REGS ? prev[i].v[j + 1] : above[i], 0x5432);
    const uint32_t dn0 = __byte_perm(below[i], prev[i].v[0], 0x5432);
    uint32_t mm = 0xffffffffu;
#pragma unroll
    for (int j = 0; j < REGS; j++) {
      const uint32_t dn = j == 0 ? dn0 : e[j - 1];
      const uint32_t m3 = __vimin3_u16x2(dn, e[j], q[i]);
      const uint32_t t = __viaddmin_u16x2(m3, p1x2, prev[i].v[j]);
      const uint32_t L = t + c[j] - prev[i].m;
      out[i].v[j] = L;
      mm = __vminu2(mm, L);
    }
    // Row minimum of this view: lane minimum, then one full-warp reduction per view with the
    // other view's lanes contributing ~0 (a reduction over a half-warp member mask measured more
    // than twice as slow, a 16-lane butterfly about a quarter slower).
    const uint32_t lm = __vminu2(mm, __byte_perm(mm, 0, 0x1032)) & 0xffffu;
    const uint32_t r0 = __reduce_min_sync(0xffffffffu, view == 0 ? lm : 0xffffffffu);
    const uint32_t r1 = __reduce_min_sync(0xffffffffu, view == 1 ? lm : 0xffffffffu);
    const uint32_t r = view ? r1 : r0;
    out[i].m = r | (r << 16);
  }
}

template <int REGS>
__device__ __forceinline__ void load_state(const uint8_t* slot, int path, int sl,
                                           PathState<REGS>& s) {
  constexpr int Dp = 2 * kLanes * REGS;
  const uint32_t* src = (const uint32_t*)(slot + 2 * (path * Dp + sl * 2 * REGS));
  if (REGS % 4 == 0) {
#pragma unroll
    for (int j = 0; j < REGS; j += 4) {
      const uint4 v = *(const uint4*)(src + j);
      s.v[j] = v.x;
      s.v[j + 1 < REGS ? j + 1 : 0] = v.y;
      s.v[j + 2 < REGS ? j + 2 : 0] = v.z;
      s.v[j + 3 < REGS ? j + 3 : 0] = v.w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < REGS; j += 2) {
      const uint2 v = *(const uint2*)(src + j);
      s.v[j] = v.x;
      s.v[j + 1 < REGS ? j + 1 : 0] = v.y;
    }
  }
  s.m = ((const uint32_t*)(slot + 6 * Dp))[path];
}

template <int REGS>
__device__ __forceinline__ void store_state(uint8_t* slot, int path, int sl,
                                            const PathState<REGS>& s) {
  constexpr int Dp = 2 * kLanes * REGS;
  uint32_t* dst = (uint32_t*)(slot + 2 * (path * Dp + sl * 2 * REGS));
  if (REGS % 4 == 0) {
#pragma unroll
    for (int j = 0; j < REGS; j += 4)
      *(uint4*)(dst + j) = make_uint4(s.v[j], s.v[j + 1 < REGS ? j + 1 : 0],
                                      s.v[j + 2 < REGS ? j + 2 : 0], s.v[j + 3 < REGS ? j + 3 : 0]);
  } else {
#pragma unroll
    for (int j = 0; j < REGS; j += 2)
      *(uint2*)(dst + j) = make_uint2(s.v[j], s.v[j + 1 < REGS ? j + 1 : 0]);
  }
  if (sl == 0) ((uint32_t*)(slot + 6 * Dp))[path] = s.m;
}

template <int REGS>
__device__ __forceinline__ void zero_state(PathState<REGS>& s) {
#pragma unroll
  for (int j = 0; j < REGS; j++) s.v[j] = 0;
  s.m = 0;
}

// One CTA = R row warps + 1 producer warp.
//  * Row warp w holds image row b*R + w (stream order) of both views and processes stream pixel
//    xs = step - 2w; the row warps meet at a named barrier once per step.  They only wait on
//    mbarriers of copies the producer issued ahead of time, and tell the producer through
//    shared-memory counters (release/acquire) which slots they have finished.
//  * The producer warp (one lane) bulk-copies cost chunks into each row warp's NB slots, fetches
//    the previous CTA's carry row chunk by chunk once its progress counter covers it, and
//    publishes this CTA's own carry progress after the last row warp has written a chunk.
// K: pixels per chunk (power of two); R: row warps; MINB: CTAs per SM.
template <int REGS, int NPATH, int K, int R, int MINB>
__global__ void __launch_bounds__((R + 1) * 32, MINB) sweep_kernel(const SweepArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  using L = SweepLayout<REGS, K, R>;
  constexpr int Dp = L::Dp, RING = L::RING, NB = L::NB, CS = L::CS;
  uint32_t* lut = (uint32_t*)(smem + L::lut);
  uint64_t* full = (uint64_t*)(smem + L::bars);  // [R][NB]
  uint64_t* carry_full = full + R * NB;          // [CS]
  int* consumed = (int*)(smem + L::counters);    // cost chunks finished, per row warp
  int* carry_consumed = consumed + R;            // carry chunks no longer needed by row warp 0
  int* published = consumed + R + 1;             // carry chunks written by row warp R-1
  uint8_t* carry_buf = smem + L::carry;
  __shared__ int s_ticket;

  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int W = a.W, H = a.H;
  if (threadIdx.x == 0) {
    s_ticket = atomicAdd(a.ticket, 1);
    for (int i = 0; i < R * NB + CS; i++) mbar_init(&full[i], 1);
    for (int i = 0; i < R + 2; i++) consumed[i] = 0;
  }
  for (int i = threadIdx.x; i < 256; i += blockDim.x) lut[i] = lut_value(a.p1, a.p2, a.edge_scale, i);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();

  const int ticket = s_ticket;
  const int stream = ticket & 1, b = ticket >> 1;
  const bool mirror = stream != 0;
  const bool has_next = b + 1 < a.nb;
  const long long limit = a.timeout;
  const int nchunks = (W + K - 1) / K;
  auto chunk_n = [&](int c) { return min(K, W - c * K); };
  auto chunk_first = [&](int c) { return mirror ? W - c * K - chunk_n(c) : c * K; };
  auto row_of = [&](int r) { return mirror ? a.Hp - 1 - (b * R + r) : b * R + r; };
  const uint8_t* carry_in = a.carry + (int64_t)(stream * a.nb + b - 1) * W * L::vslot;

  if (w == R) {
    // ------------------------------------------------------------------ producer warp
    if (lane != 0) return;
    int next[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int y = row_of(r);
      next[r] = (y >= 0 && y < H) ? 0 : nchunks;  // rows beyond the image get no chunks
    }
    int next_carry = b > 0 ? 0 : nchunks;
    int done_pub = has_next ? 0 : nchunks;
    const int* prev_progress = &a.progress[stream * a.nb + b - 1];
    int* my_progress = &a.progress[stream * a.nb + b];
    long long last = clock64();
    while (true) {
      bool pending = false, did = false;
#pragma unroll
      for (int r = 0; r < R; r++) {
        const int c = next[r];
        if (c >= nchunks) continue;
        pending = true;
        if (c - ld_acquire_cta(&consumed[r]) >= NB) continue;
        const int64_t off = ((int64_t)row_of(r) * W + chunk_first(c)) * Dp;
        const uint32_t bytes = (uint32_t)(chunk_n(c) * Dp);
        uint64_t* bar = &full[r * NB + c % NB];
        uint8_t* dst = smem + L::cost + ((r * NB + c % NB) * kViews) * K * Dp;
        fence_proxy_async_shared();
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                     "r"(2 * bytes)
                     : "memory");
#pragma unroll
        for (int vv = 0; vv < kViews; vv++)
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
              "[%3];" ::"r"(smem_u32(dst + vv * K * Dp)),
              "l"(a.cost[vv] + off), "r"(bytes), "r"(smem_u32(bar))
              : "memory");
        next[r] = c + 1;
        did = true;
      }
      if (next_carry < nchunks) {
        pending = true;
        const int ch = next_carry;
        if (ch - ld_acquire_cta(carry_consumed) < CS &&
            ld_acquire_gpu(prev_progress) >= min(W, (ch + 1) * K)) {
          fence_proxy_async_global();
          fence_proxy_async_shared();
          bulk_load(carry_buf + (ch % CS) * K * L::vslot, carry_in + (int64_t)ch * K * L::vslot,
                    (uint32_t)(chunk_n(ch) * L::vslot), &carry_full[ch % CS]);
          next_carry = ch + 1;
          did = true;
        }
      }
      if (done_pub < nchunks) {
        pending = true;
        const int done = ld_acquire_cta(published);
        if (done > done_pub) {
          __threadfence();  // the carry rows the row warps wrote are visible GPU-wide first
          atomicExch(my_progress, min(W, done * K));
          done_pub = done;
          did = true;
        }
      }
      if (!pending) break;
      if (did) {
        last = clock64();
      } else {
        if (*(volatile int*)a.error) break;
        if (clock64() - last > limit) {
          atomicExch(a.error, 6);
          break;
        }
        __nanosleep(32);
      }
    }
    // Every copy issued above lands before the CTA's shared memory is released (normally all
    // have landed already; after an error this bounds the exit).
    const long long drain = limit / 4;
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int y = row_of(r);
      if (y < 0 || y >= H) continue;
      for (int c = max(0, next[r] - NB); c < next[r]; c++)
        wait_bar(&full[r * NB + c % NB], (c / NB) & 1, a.error, drain, 5, false);
    }
    if (b > 0)
      for (int ch = max(0, next_carry - CS); ch < next_carry; ch++)
        wait_bar(&carry_full[ch % CS], (ch / CS) & 1, a.error, drain, 5, false);
    return;
  }

  // -------------------------------------------------------------------- row warps
  const int v = lane / kLanes, sl = lane % kLanes;  // view and lane within the view-row
  const int yp = b * R + w;                         // row in stream coordinates
  const int y = row_of(w);
  const bool exists = y >= 0 && y < H;
  const int steps = W + 2 * (R - 1);
  if (!exists) {
    // Rows beyond the image: nobody reads them, but the warp takes part in every step barrier.
    for (int step = 0; step < steps; step++) rows_barrier(R * 32);
    return;
  }
  const int ya = mirror ? y + 1 : y - 1;  // image row of the row above (stream order)
  const bool above_exists = yp >= 1 && ya >= 0 && ya < H;
  const bool use_carry = w == 0 && b > 0;  // the row above lives in the previous CTA
  const bool from_ring = above_exists && w > 0;
  const bool from_above = from_ring || use_carry;
  const bool publish = w == R - 1 && has_next;
  const int dir = mirror ? -1 : 1;
  const int x0 = mirror ? W - 1 : 0;       // image column of stream pixel 0

  const uint8_t* gray_v = v ? a.gray[1] : a.gray[0];
  const uint8_t* tex_v = v ? a.tex[1] : a.tex[0];
  uint16_t* sum_v = mirror ? (v ? a.sum[1][1] : a.sum[1][0]) : (v ? a.sum[0][1] : a.sum[0][0]);
  const uint8_t* gray_row = gray_v + (int64_t)y * W + x0;
  const uint8_t* tex_row = tex_v + (int64_t)y * W + x0;
  const uint8_t* gray_up = gray_v + (int64_t)(above_exists ? ya : y) * W + x0;
  uint16_t* sum_mine = sum_v + (int64_t)y * W * Dp;
  const uint8_t* cost_mine = smem + L::cost + (w * NB * kViews + v) * K * Dp;  // + slot * 2*K*Dp
  uint8_t* ring = smem + L::ring + w * RING * L::vslot + v * L::slot;
  const uint8_t* ring_up = smem + L::ring + (w - 1) * RING * L::vslot + v * L::slot;
  uint8_t* carry_out = a.carry + (int64_t)(stream * a.nb + b) * W * L::vslot + v * L::slot;
  const uint8_t* carry_view = carry_buf + v * L::slot;

  // Costs of disparities >= D are lifted from 512 to 0x8000 (see paths_step).
  uint32_t padadd[REGS];
#pragma unroll
  for (int j = 0; j < REGS; j++) {
    const int k = sl * 2 * REGS + 2 * j;
    padadd[j] = (k >= a.D ? 0x7e00u : 0u) | (k + 1 >= a.D ? 0x7e000000u : 0u);
  }
  const uint32_t p1x2 = (uint32_t)a.p1 | ((uint32_t)a.p1 << 16);

  // Per-chunk pixel data, lane sl < K of each view-row <-> pixel c*K + sl of that view:
  // gray | tex << 8 | gray above << 16 | gray above of the next pixel << 24.
  auto chunk_pixels = [&](int cc) -> uint32_t {
    const int xs_l = cc * K + sl;
    uint32_t d = 0;
    if (sl < K && xs_l < W) {
      d = (uint32_t)__ldg(gray_row + dir * xs_l) | ((uint32_t)(__ldg(tex_row + dir * xs_l) != 0) << 8);
      if (above_exists) {
        d |= (uint32_t)__ldg(gray_up + dir * xs_l) << 16;
        if (xs_l + 1 < W) d |= (uint32_t)__ldg(gray_up + dir * (xs_l + 1)) << 24;
      }
    }
    return d;
  };
  uint32_t px_cur = chunk_pixels(0);
  uint32_t px_next = nchunks > 1 ? chunk_pixels(1) : 0u;

  PathState<REGS> horiz;  // (1,0) path in stream coordinates
  zero_state(horiz);
  // Penalty-table values and texture flag of the pixel about to be processed.
  uint32_t lutv[NPATH];
  bool textured;
  int g_prev, ga_prev;  // gray of the previous pixel, gray above of the previous pixel
  {
    const uint32_t pxv = __shfl_sync(0xffffffffu, px_cur, v * kLanes);
    const int g = pxv & 0xff, ga = (pxv >> 16) & 0xff, gr = pxv >> 24;
    textured = (pxv >> 8) & 1;
    lutv[0] = lut[g];  // no left neighbour: the value is unused (zero predecessor)
    if (NPATH > 1) lutv[1 % NPATH] = lut[abs(g - ga)];
    if (NPATH > 2) lutv[2 % NPATH] = lut[0];
    if (NPATH > 3) lutv[3 % NPATH] = lut[abs(g - gr)];
    g_prev = g;
    ga_prev = ga;
  }
  int off = 0, c = 0, n_c = chunk_n(0), carry_ready = 0, carry_rel = 0;

  for (int step = 0; step < steps; step++) {
    const int xs = step - 2 * w;
    if (xs < 0 || xs >= W) {
      rows_barrier(R * 32);
      continue;
    }
    if (use_carry) {
      const int need_chunk = min(nchunks - 1, (xs + 1) / K);
      while (carry_ready <= need_chunk) {
        wait_bar(&carry_full[carry_ready % CS], (carry_ready / CS) & 1, a.error, limit, 3);
        carry_ready++;
      }
    }
    if (off == 0) wait_bar(&full[w * NB + c % NB], (c / NB) & 1, a.error, limit, 1);
    const int slot_off = (c % NB) * kViews * K * Dp;
    const int pos = mirror ? n_c - 1 - off : off;
    const int x = x0 + dir * xs;
    // Predecessor states: ring (row above in this CTA) or carry (row above in the previous CTA).
    PathState<REGS> prev[NPATH];
    prev[0] = horiz;
    const int nbr[3] = {xs, xs - 1, xs + 1};
#pragma unroll
    for (int i = 0; i < NPATH - 1; i++) {
      const int xx = nbr[i];
      if (from_above && xx >= 0 && xx < W) {
        const uint8_t* src = from_ring ? ring_up + (xx & (RING - 1)) * L::vslot
                                       : carry_view + (xx & (CS * K - 1)) * L::vslot;
        load_state<REGS>(src, i, sl, prev[i + 1]);
      } else {
        zero_state(prev[i + 1]);
      }
    }
    // Costs: 2*REGS bytes per lane -> REGS packed uint16 pairs, 0x80 -> 512.
    const uint8_t* cb = cost_mine + slot_off + pos * Dp + sl * 2 * REGS;
    uint32_t cst[REGS], words[REGS / 2];
#pragma unroll
    for (int j = 0; j < REGS; j += 2) {
      words[j / 2] = ((const uint32_t*)cb)[j / 2];
      cst[j] = (prmt(words[j / 2], 0, 0x9180u) & 0x027f027fu) + padadd[j];
      cst[j + 1] = (prmt(words[j / 2], 0, 0xb3a2u) & 0x027f027fu) + padadd[j + 1];
    }
    uint32_t q[NPATH];
#pragma unroll
    for (int i = 0; i < NPATH; i++) q[i] = prev[i].m + lutv[i];
    PathState<REGS> out[NPATH];
    paths_step<REGS, NPATH>(prev, q, p1x2, cst, sl, v, out);
    // Partial aggregate of this stream's paths; the down stream marks invalid costs 0xffff.
    uint32_t s[REGS];
#pragma unroll
    for (int j = 0; j < REGS; j++) {
      uint32_t acc = out[0].v[j];
#pragma unroll
      for (int i = 1; i < NPATH; i++) acc += out[i].v[j];
      s[j] = acc;
    }
    if (!mirror) {
#pragma unroll
      for (int j = 0; j < REGS; j += 2) {
        s[j] |= prmt(words[j / 2], 0, 0x9988u);
        s[j + 1] |= prmt(words[j / 2], 0, 0xbbaau);
      }
    }
    // Outputs for the row below: the three vertical paths, zeros if this pixel is untextured
    // (the zeroing only runs in warps that hold an untextured pixel).
    uint8_t* out_slot = ring + (xs & (RING - 1)) * L::vslot;
    if (!__all_sync(0xffffffffu, textured)) {
#pragma unroll
      for (int i = 0; i < NPATH; i++)
        if (!textured) zero_state(out[i]);
    }
#pragma unroll
    for (int i = 0; i < NPATH - 1; i++) {
      store_state<REGS>(out_slot, i, sl, out[i + 1]);
      if (publish) store_state<REGS>(carry_out + (int64_t)xs * L::vslot, i, sl, out[i + 1]);
    }
    horiz = out[0];
    uint32_t* dst = (uint32_t*)(sum_mine + (int64_t)x * Dp + sl * 2 * REGS);
    if (REGS % 4 == 0) {
#pragma unroll
      for (int j = 0; j < REGS; j += 4)
        *(uint4*)(dst + j) = make_uint4(s[j], s[j + 1 < REGS ? j + 1 : 0],
                                        s[j + 2 < REGS ? j + 2 : 0], s[j + 3 < REGS ? j + 3 : 0]);
    } else {
#pragma unroll
      for (int j = 0; j < REGS; j += 2)
        *(uint2*)(dst + j) = make_uint2(s[j], s[j + 1 < REGS ? j + 1 : 0]);
    }
    // Next pixel's pixel data, penalty-table values and texture flag (off the critical path).
    if (off + 1 == n_c) {
      // End of chunk c: hand the slot back, publish carry progress, move to chunk c+1.
      __syncwarp();
      if (lane == 0) {
        st_release_cta(&consumed[w], c + 1);
        if (publish) st_release_cta(published, c + 1);
      }
      off = 0;
      c++;
      if (c < nchunks) {
        n_c = chunk_n(c);
        px_cur = px_next;
        px_next = c + 1 < nchunks ? chunk_pixels(c + 1) : 0u;
      }
    } else {
      off++;
    }
    if (xs + 1 < W) {
      const uint32_t pxv = __shfl_sync(0xffffffffu, px_cur, v * kLanes + off);
      const int g = pxv & 0xff, ga = (pxv >> 16) & 0xff, gr = pxv >> 24;
      textured = (pxv >> 8) & 1;
      lutv[0] = lut[abs(g - g_prev)];
      if (NPATH > 1) lutv[1 % NPATH] = lut[abs(g - ga)];
      if (NPATH > 2) lutv[2 % NPATH] = lut[abs(g - ga_prev)];
      if (NPATH > 3) lutv[3 % NPATH] = lut[abs(g - gr)];
      g_prev = g;
      ga_prev = ga;
    }
    if (use_carry && xs / K > carry_rel) {
      carry_rel = xs / K;  // chunks before the one holding pixel xs are no longer needed
      __syncwarp();
      if (lane == 0) st_release_cta(carry_consumed, carry_rel);
    }
    rows_barrier(R * 32);
  }
}

// ---------------------------------------------------------------------------------------------
// Winner-take-all, uniqueness and sub-pixel selection of both views (CensusSgm.java:460-515).
// A warp owns a tile of 32 consecutive pixels of one row of one view; lane 0 bulk-copies the
// tile's two partial aggregates (down, up) into shared memory (double-buffered across tiles) and
// every lane then selects one pixel.  Lane t reads its pixel's words starting at word t, so the
// 32 lanes hit 32 different banks although the pixels are Dp words apart.
struct WtaArgs {
  const uint16_t* down[2];  // per view; 0xffff = invalid cost
  const uint16_t* up[2];
  float* disp[2];
  uint8_t* reasons;    // left view only
  uint8_t* boundary;   // left view only
  DeviceStats* stats;  // left view only
  int* error;
  int W, H, D, min_disparity, rx, ry;
  double uniqueness;
  long long timeout;
};

template <int DP>
struct WtaLayout {
  static constexpr int warps = DP <= 64 ? 8 : DP <= 128 ? 6 : DP <= 192 ? 4 : 3;
  static constexpr int tile = 32 * DP * 2;             // bytes of one stream's tile
  static constexpr int per_warp = 2 * 2 * tile;        // 2 buffers x (down, up)
  static constexpr int bars = 0;                        // warps x 2 mbarriers
  static constexpr int tiles = 128;
  static constexpr int total = tiles + warps * per_warp;
};

// Selection of one pixel from its winners record (CensusSgm.java:471-513).
__device__ __forceinline__ void select_pixel_record(int best, int value, int second, int before,
                                                    int after, int flags, int D, int min_disparity,
                                                    double uniqueness, float* out,
                                                    uint8_t* reasons, uint8_t* boundary,
                                                    unsigned (&counts)[6], bool count) {
  float result = __int_as_float(0x7fc00000);
  if (best >= 0) {
    const bool full = flags == 3;
    bool done = false;
    if (full) {
      counts[1] += count;
      if (boundary) *boundary = 4;
    }
    if (best == 0 || best == D - 1) {
      counts[2] += count;
      if (reasons) *reasons = 2;
      if (full && best == 0) {
        counts[0] += count;
        if (boundary) *boundary |= 1;
      }
      if (full && best == D - 1) {
        counts[3] += count;
        if (boundary) *boundary |= 2;
      }
      done = true;
    }
    if (!done && second != INT_MAX) {
      const double slack = fmax(1.0, __dmul_rn((double)value, uniqueness));
      if ((double)(second - value) <= slack) {
        counts[4] += count;
        if (reasons) *reasons = 3;
        done = true;
      }
    }
    if (!done) {
      double offset = 0;
      if (before >= 0 && after >= 0) {
        const double curvature =
            __dsub_rn(__dadd_rn((double)before, (double)after), __dmul_rn(2.0, (double)value));
        if (curvature > 0) {
          const double o =
              __ddiv_rn(__dmul_rn(0.5, __dsub_rn((double)before, (double)after)), curvature);
          offset = fmax(-0.5, fmin(0.5, o));
        }
      }
      result = __double2float_rn(__dadd_rn((double)(min_disparity + best), offset));
      counts[5] += count;
      if (reasons) *reasons = 0;
    }
  }
  *out = result;
}

template <int DP>
__global__ void __launch_bounds__(WtaLayout<DP>::warps * 32) wta_kernel(const WtaArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  using L = WtaLayout<DP>;
  constexpr int NW = DP / 2;  // 32-bit words per pixel and stream
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t* bars = (uint64_t*)(smem + L::bars) + warp * 2;
  uint8_t* tiles = smem + L::tiles + warp * L::per_warp;
  if (lane == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncwarp();

  const int W = a.W, H = a.H, D = a.D;
  const int per_row = (W + 31) / 32;
  const int64_t items = 2LL * H * per_row;  // (view, row, tile)
  const int64_t stride = (int64_t)gridDim.x * L::warps;
  int64_t item = (int64_t)blockIdx.x * L::warps + warp;
  auto decode = [&](int64_t it, int& view, int& y, int& x0) {
    view = (int)(it / ((int64_t)H * per_row));
    const int64_t r = it - (int64_t)view * H * per_row;
    y = (int)(r / per_row);
    x0 = (int)(r - (int64_t)y * per_row) * 32;
  };
  auto issue = [&](int64_t it, int buf) {
    if (lane == 0) {
      int view, y, x0;
      decode(it, view, y, x0);
      const uint32_t bytes = (uint32_t)(min(32, W - x0) * DP * 2);
      const int64_t off = ((int64_t)y * W + x0) * DP;
      fence_proxy_async_shared();
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                       smem_u32(&bars[buf])),
                   "r"(2 * bytes)
                   : "memory");
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
          "[%3];" ::"r"(smem_u32(tiles + (buf * 2) * L::tile)),
          "l"((view ? a.down[1] : a.down[0]) + off), "r"(bytes), "r"(smem_u32(&bars[buf]))
          : "memory");
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
          "[%3];" ::"r"(smem_u32(tiles + (buf * 2 + 1) * L::tile)),
          "l"((view ? a.up[1] : a.up[0]) + off), "r"(bytes), "r"(smem_u32(&bars[buf]))
          : "memory");
    }
    __syncwarp();  // no lane may spin on the barrier before lane 0 has armed it
  };

  unsigned counts[6] = {0, 0, 0, 0, 0, 0};
  int it = 0;
  if (item < items) issue(item, 0);
  for (; item < items; item += stride, it++) {
    const int buf = it & 1;
    if (item + stride < items) issue(item + stride, buf ^ 1);
    wait_bar(&bars[buf], (it >> 1) & 1, a.error, a.timeout, 4);
    int view, y, x0;
    decode(item, view, y, x0);
    const int x = x0 + lane;
    if (x < W) {
      const uint32_t* pa = (const uint32_t*)(tiles + (buf * 2) * L::tile) + lane * NW;
      const uint32_t* pb = (const uint32_t*)(tiles + (buf * 2 + 1) * L::tile) + lane * NW;
      const uint16_t* ha = (const uint16_t*)pa;
      const uint16_t* hb = (const uint16_t*)pb;
      const bool inside = y >= a.ry && y < H - a.ry && x >= a.rx && x < W - a.rx;
      int best = -1, value = 0, second = INT_MAX, before = -1, after = -1, flags = 0;
      if (inside) {
        // Pass 1: first strict minimum among valid disparities, as key = total << 8 | k.
        uint32_t key = 0xffffffffu;
        int wi = lane;
        for (int i = 0; i < NW; i++) {
          const uint32_t wa = pa[wi], wb = pb[wi];
          const uint32_t bad = prmt(wa, 0, 0xbb99u);  // 0xffff where the cost is invalid
          const uint32_t tot = ((wa & ~bad) + wb) | bad;
          const uint32_t k = 2 * wi;
          key = min(key, min(((tot & 0xffffu) << 8) | k, ((tot >> 8) & 0xffff00u) | (k + 1)));
          if (++wi == NW) wi = 0;
        }
        if ((key >> 8) != 0xffffu) {
          best = (int)(key & 0xffu);
          value = (int)(key >> 8);
          // Pass 2: minimum over valid disparities outside best-1..best+1.
          uint32_t sec = 0xffffu;
          wi = lane;
          for (int i = 0; i < NW; i++) {
            const uint32_t wa = pa[wi], wb = pb[wi];
            const uint32_t bad = prmt(wa, 0, 0xbb99u);
            const uint32_t tot = ((wa & ~bad) + wb) | bad;
            const int k = 2 * wi;
            if ((unsigned)(k - best + 1) > 2u) sec = min(sec, tot & 0xffffu);
            if ((unsigned)(k - best + 2) > 2u) sec = min(sec, tot >> 16);
            if (++wi == NW) wi = 0;
          }
          second = sec == 0xffffu ? INT_MAX : (int)sec;
          if (best >= 1 && !(ha[best - 1] & 0x8000u)) before = ha[best - 1] + hb[best - 1];
          if (best + 1 < D && !(ha[best + 1] & 0x8000u)) after = ha[best + 1] + hb[best + 1];
          flags = (!(ha[0] & 0x8000u) ? 1 : 0) | (!(ha[D - 1] & 0x8000u) ? 2 : 0);
        }
      }
      const int64_t p = (int64_t)y * W + x;
      select_pixel_record(best, value, second, before, after, flags, D, a.min_disparity,
                          a.uniqueness, (view ? a.disp[1] : a.disp[0]) + p,
                          view == 0 && a.reasons ? a.reasons + p : nullptr,
                          view == 0 && a.boundary ? a.boundary + p : nullptr, counts, view == 0);
    }
    __syncwarp();
  }
  // Every issued tile was waited for above; after a timed-out wait, give the copy a bounded
  // second chance to land before the CTA's shared memory is released.
  for (int j = max(0, it - 2); j < it; j++)
    wait_bar(&bars[j & 1], (j >> 1) & 1, a.error, a.timeout / 4, 5, false);
  if (a.stats) {
    unsigned long long* dst[6] = {&a.stats->lower_boundary_rejected,
                                  &a.stats->full_interval_pixels, &a.stats->boundary_rejected,
                                  &a.stats->upper_boundary_rejected,
                                  &a.stats->ambiguity_rejected, &a.stats->selected};
#pragma unroll
    for (int i = 0; i < 6; i++) {
      const unsigned total = __reduce_add_sync(0xffffffffu, counts[i]);
      if (lane == 0 && total) atomicAdd(dst[i], (unsigned long long)total);
    }
  }
}

template <int DP>
cudaError_t launch_wta(const WtaArgs& a, int sm_count, cudaStream_t stream) {
  using L = WtaLayout<DP>;
  cudaError_t e =
      cudaFuncSetAttribute(wta_kernel<DP>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::total);
  if (e != cudaSuccess) return e;
  const int64_t items = 2LL * a.H * ((a.W + 31) / 32);
  const int grid = (int)std::min<int64_t>((items + L::warps - 1) / L::warps, sm_count);
  wta_kernel<DP><<<grid, L::warps * 32, L::total, stream>>>(a);
  return cudaGetLastError();
}

template <int REGS, int NPATH, int K, int R, int MINB>
cudaError_t launch_sweep(const SweepArgs& a, cudaStream_t stream) {
  auto kernel = sweep_kernel<REGS, NPATH, K, R, MINB>;
  const int shared = SweepLayout<REGS, K, R>::total;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, shared);
  if (e != cudaSuccess) return e;
  kernel<<<2 * a.nb, (R + 1) * 32, shared, stream>>>(a);
  return cudaGetLastError();
}

// Per-register-count configuration: chunk pixels, rows per CTA (shared-memory fit), CTAs per SM.
constexpr int chunk_for(int regs) { return regs >= 6 ? 2 : 4; }
constexpr int rows_for(int regs) { return regs <= 4 ? 16 : 8; }
constexpr int minb_for(int) { return 1; }

struct FusedLayout {
  size_t cost, sum, carry, flags, total;
  int Dp, nb, slot, rows;
  FusedLayout(const csgm_params& p, int w, int h) {
    Dp = padded_d(p.disparities);
    rows = rows_for(Dp / (2 * kLanes));
    nb = (h + rows - 1) / rows;
    slot = 3 * Dp * 2 + 16;
    size_t n = (size_t)w * h;
    cost = n * Dp;
    sum = n * Dp * 2;
    carry = (size_t)2 * nb * w * kViews * slot;
    flags = ((size_t)2 * nb + 8) * sizeof(int);
    total = 2 * cost + 4 * sum + carry + flags + 6 * 256;
  }
};

}  // namespace

bool fused_supported(const csgm_params& p) {
  if (p.disparities > 256 || p.aggregate_bytes != 2) return false;
  if (p.directions != 4 && p.directions != 8) return false;
  if (512 + 2 * (int64_t)p.p2 + p.p1 > 65535) return false;
  return true;
}

size_t fused_workspace_bytes(const csgm_params& p, int w, int h) {
  return FusedLayout(p, w, h).total;
}

int run_views_fused(Context& ctx, const csgm_params& p, const FusedViews& v, int w, int h,
                    int** error_flag) {
  int status = CSGM_OK;
  FusedLayout F(p, w, h);
  uint8_t* cost_l = (uint8_t*)ctx.ws->get(kCostL, F.cost, &status);
  if (!cost_l) return status;
  uint8_t* cost_r = (uint8_t*)ctx.ws->get(kCostR, F.cost, &status);
  if (!cost_r) return status;
  uint16_t* sums[4];
  const int sum_slots[4] = {kSum, kSumR, kSumUp, kSumUpR};
  for (int i = 0; i < 4; i++) {
    sums[i] = (uint16_t*)ctx.ws->get(sum_slots[i], F.sum, &status);
    if (!sums[i]) return status;
  }
  uint8_t* carry = (uint8_t*)ctx.ws->get(kCarry, F.carry, &status);
  if (!carry) return status;
  int* flags = (int*)ctx.ws->get(kFlags, F.flags, &status);
  if (!flags) return status;

  int words = (p.window_x * p.window_y - 1 + 63) / 64;
  CostPairArgs ca{};
  ca.view[0] = CostArgs{v.desc_l, v.desc_r, v.tex_l, v.tex_r, v.gray_l, v.gray_r, nullptr, w, h,
                        p.disparities, p.min_disparity, 0, p.window_x, p.window_y, words,
                        p.cost_mode, p.census_weight_milli, p.ad_truncation,
                        p.gradient_truncation, p.window_x * p.window_y - 1};
  ca.view[1] = ca.view[0];
  ca.view[1].desc_a = v.desc_r;
  ca.view[1].desc_b = v.desc_l;
  ca.view[1].tex_a = v.tex_r;
  ca.view[1].tex_b = v.tex_l;
  ca.view[1].gray_a = v.gray_r;
  ca.view[1].gray_b = v.gray_l;
  ca.view[1].reverse = 1;
  ca.out[0] = cost_l;
  ca.out[1] = cost_r;
  ca.Dp = F.Dp;
  {
    cudaError_t le;
    ctx.prof->kernel_begin();
    if (p.cost_mode == CSGM_COST_ZNCC) {
      int64_t n = (int64_t)w * h;
      int64_t blocks = (n * 32 + 255) / 256;
      int grid = (int)std::min<int64_t>(blocks, (int64_t)ctx.sm_count * 32);
      cost_pair_kernel<<<dim3(grid, 2), 256, 0, ctx.stream>>>(ca);
      le = cudaGetLastError();
    } else {
      const size_t shared = cost_rows_shared(p.disparities, F.Dp);
      le = cudaFuncSetAttribute(cost_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)shared);
      if (le == cudaSuccess) {
        const int64_t items = (int64_t)h * ((w + kCostSeg - 1) / kCostSeg);
        const int grid = (int)std::min<int64_t>(items, (int64_t)ctx.sm_count * 16);
        cost_rows_kernel<<<dim3(grid, 2), kCostSeg, shared, ctx.stream>>>(ca);
        le = cudaGetLastError();
      }
    }
    if (le != cudaSuccess) return cuda_fail(le, "cost kernel launch");
    ctx.prof->kernel_end("cost_pair");
  }
  cudaError_t e = cudaMemsetAsync(flags, 0, F.flags, ctx.stream);
  if (e != cudaSuccess) return cuda_fail(e, "flag clear");

  SweepArgs a{};
  a.cost[0] = cost_l;
  a.cost[1] = cost_r;
  a.gray[0] = v.gray_l;
  a.gray[1] = v.gray_r;
  a.tex[0] = v.tex_l;
  a.tex[1] = v.tex_r;
  a.sum[0][0] = sums[0];
  a.sum[0][1] = sums[1];
  a.sum[1][0] = sums[2];
  a.sum[1][1] = sums[3];
  a.carry = carry;
  a.progress = flags;
  a.ticket = flags + 2 * F.nb;
  a.error = a.ticket + 1;
  *error_flag = a.error;
  a.W = w;
  a.H = h;
  a.D = p.disparities;
  a.nb = F.nb;
  a.Hp = F.nb * F.rows;
  a.p1 = p.p1;
  a.p2 = p.p2;
  a.edge_scale = p.edge_scale;
  a.timeout = 4000000000LL;  // ~2 s at 2 GHz
  const int regs = F.Dp / (2 * kLanes);
  const bool eight = p.directions == 8;
  ctx.prof->kernel_begin();
  switch (regs * 2 + (eight ? 1 : 0)) {
#define CSGM_SWEEP_CASE(R_, NP_)                                                             \
  case R_ * 2 + (NP_ == 4 ? 1 : 0):                                                         \
    e = launch_sweep<R_, NP_, chunk_for(R_), rows_for(R_), minb_for(R_)>(a, ctx.stream);     \
    break;
    CSGM_SWEEP_CASE(2, 2)
    CSGM_SWEEP_CASE(2, 4)
    CSGM_SWEEP_CASE(4, 2)
    CSGM_SWEEP_CASE(4, 4)
    CSGM_SWEEP_CASE(6, 2)
    CSGM_SWEEP_CASE(6, 4)
    CSGM_SWEEP_CASE(8, 2)
    CSGM_SWEEP_CASE(8, 4)
#undef CSGM_SWEEP_CASE
    default: return fail(CSGM_E_UNSUPPORTED, "fused path: unsupported D");
  }
  if (e != cudaSuccess) return cuda_fail(e, "sweep kernel launch");
  ctx.prof->kernel_end("sweep");

  WtaArgs t{};
  t.down[0] = sums[0];
  t.down[1] = sums[1];
  t.up[0] = sums[2];
  t.up[1] = sums[3];
  t.disp[0] = v.disp_l;
  t.disp[1] = v.disp_r;
  t.reasons = v.reasons;
  t.boundary = v.boundary;
  t.stats = v.stats;
  t.error = a.error;
  t.W = w;
  t.H = h;
  t.D = p.disparities;
  t.min_disparity = p.min_disparity;
  t.rx = p.window_x / 2;
  t.ry = p.window_y / 2;
  t.uniqueness = p.uniqueness;
  t.timeout = a.timeout;
  ctx.prof->kernel_begin();
  switch (F.Dp) {
    case 64: e = launch_wta<64>(t, ctx.sm_count, ctx.stream); break;
    case 128: e = launch_wta<128>(t, ctx.sm_count, ctx.stream); break;
    case 192: e = launch_wta<192>(t, ctx.sm_count, ctx.stream); break;
    case 256: e = launch_wta<256>(t, ctx.sm_count, ctx.stream); break;
    default: return fail(CSGM_E_UNSUPPORTED, "fused path: unsupported D");
  }
  if (e != cudaSuccess) return cuda_fail(e, "wta kernel launch");
  ctx.prof->kernel_end("wta");
  return CSGM_OK;
}

}  // namespace csgm
