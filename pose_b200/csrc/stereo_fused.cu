// stereo_fused.cu - fast path of the matcher for D <= 256, 4/8 paths, uint16 aggregate.
//
// Reference semantics: cost CensusSgm.java:405-420 + StereoCost.java:50-90; aggregation
// CensusSgm.java:421-459; selection CensusSgm.java:460-515.  Results are bit-identical to the
// general kernels (stereo_kernels.cu) and to the CPU reference.
//
// Design (B200):
//  * cost_rows_kernel (census modes) / cost_pair_kernel (ZNCC) write both views' cost volumes
//    once, as uint8 [H][W][Dp] with Dp = D rounded up to 64 and 0x80 marking the reference's
//    invalid cost 512.  penalty_kernel writes one record of per-path P2' - P1 per stream pixel.
//  * lines_kernel aggregates the two anti-diagonal paths (-1,1) and (1,-1): the lines x + y = s
//    are independent, one warp walks a line forward and back and stores their sum as the lines
//    partial aggregate.
//  * sweep_kernel runs two wavefront streams in one launch, each over both views: "down"
//    processes rows top to bottom, pixels left to right, and owns (1,0), (0,1), (1,1); "up" is
//    the same code on the image mirrored in x and y and owns the three opposite paths.
//  * One sweep CTA = R consecutive image rows; warp w holds row w of BOTH views (each register
//    packs a disparity's left-view value in its low and right-view value in its high 16 bits)
//    and processes pixel x at step x + w, all row warps in lock step (one named barrier per
//    step).  The (0,1) and (1,1) states of a row reach the next row through a shared-memory
//    ring; the (1,0) state stays in registers.  The last row of a CTA also writes a global carry
//    row that the next CTA of the stream reads (release/acquire progress counter).
//  * Each stream stores its partial aggregate (uint16 pairs, 3 paths).  No cell is marked
//    invalid: a valid path cost stays below 512 and an invalid one is at least 512, so a total of
//    at least directions x 512 is an invalid cell.  The streams never wait for each other.
//  * wta_kernel adds the partial aggregates (a warp per pixel, both views at once) and runs
//    winner-take-all, uniqueness and the parabolic sub-pixel step, lane v selecting view v.
//  * The min-plus step uses the DPX instructions __vimin3_u16x2 / __viaddmin_u16x2 on the
//    packed pairs; the row minima of both views are two redux.sync.min per path.
//  * Sweep cost chunks and carry rows are staged in shared memory by cp.async.bulk with mbarrier
//    completion (no multicast); the line kernel prefetches with cp.async.  Every wait is
//    bounded; a wait that runs out sets an error flag that the host turns into CSGM_E_TIMEOUT.
//  * Sweep CTAs take tickets in launch order; a CTA only waits on lower tickets, so the schedule
//    cannot deadlock even when not every CTA is resident.
#include <climits>
#include <cstdlib>
#include <type_traits>

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

// Non-suspending probe of an mbarrier phase.
__device__ __forceinline__ bool mbar_probe(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
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

// Bounded waits.  `error` short-circuits every later wait unless `shortcut` is false (the drains,
// which must see their copies land).  A wait that runs out stores `code` (the wait site: 1 sweep
// cost chunk, 3 carry chunk, 5 drain; the sweep's carry-in and publisher warps store 6 when they
// made no progress for the limit).  Returns true once the phase has completed, false when the
// wait gave up (the copy may still be in flight: its slot must not be refilled).
__device__ __forceinline__ bool mbar_probe(uint64_t* bar, uint32_t parity);
__device__ __forceinline__ bool wait_bar(uint64_t* bar, uint32_t parity, int* error,
                                         long long limit, int code, bool shortcut = true) {
  if (mbar_probe(bar, parity)) return true;  // the common case: the copy has landed
  const long long start = clock64();
  for (unsigned spin = 1;; spin++) {
    if (mbar_test(bar, parity)) return true;
    if ((spin & 15) == 0) {  // the error flag and the clock only every 16th probe
      if (shortcut && *(volatile int*)error) return false;
      if (clock64() - start > limit) {
        atomicExch(error, code);
        return false;
      }
    }
  }
}

// Bound of the drains: a bulk copy from this GPU's own memory always completes (nothing it waits
// for can stall), so its wait is bounded by the copy engine's progress alone and runs out only if
// the device itself stops; the configurable limit does not shorten it.
constexpr long long kDrainLimit = 1LL << 32;
constexpr long long kDefaultWaitLimit = 4000000000LL;  // ~2 s at 2 GHz

// ---------------------------------------------------------------------------------------------
// Cost volumes of both views (uint8, 0x80 = invalid), StereoCost.value semantics
// (StereoCost.java:50-90) with CensusSgm.java:405-420 validity.  The right view's cost of pixel
// x' at disparity index k is the left view's cost of pixel x' + min_disparity + k at k: the same
// two descriptors, the same validity (both pixels inside [r, w-r) and textured, the row inside)
// and a symmetric cost.  So each cell is computed once: a CTA takes one image row, computes the
// left view in segments of kCostSeg pixels into a shared-memory ring of left-view cost rows, writes
// them out, and gathers each right-view segment from the ring's diagonals as soon as every left
// pixel it needs is in the ring.  Per left segment the segment's descriptors and the target
// view's descriptors over the disparity span are staged in shared memory, each target with a
// validity byte and, for the blended modes, its gray value or packed central-difference
// gradient.  Thread t computes pixel t % kCostSeg for a slice of disparity groups (consecutive
// threads read consecutive targets: no bank conflicts).  All stores are coalesced 16-byte
// stores.  The blended modes divide by 1000 * cap through an exact 64-bit reciprocal
// (floor(n * ceil(2^64 / d) / 2^64) == n / d for n, d < 2^32).  ZNCC (FP64 window sums) stays on
// the general per-cell path.
struct CostPairArgs {
  CostArgs view[2];  // per view: a = matching image, b = target image, reverse 0/1
  uint8_t* out[2];
  int Dp;
  unsigned long long recip;  // ceil(2^64 / (1000 * cap)) of the blended modes
};

constexpr int kCostSeg = 64;       // pixels per left-view segment
constexpr int kCostThreads = 256;  // 4 threads per pixel

template <int DP>
struct CostLayout {
  // Ring of left-view cost rows, a power of two >= DP + 127 pixels: a right-view segment needs
  // the 64 + DP - 1 left pixels from x' + min_disparity on, and becomes complete one segment
  // after its last one is computed.  The row pitch DP + 4 spreads a warp's diagonal reads over
  // the 32 banks.
  static constexpr int ring_px = DP + 127 <= 256 ? 256 : 512;
  static constexpr int pitch = DP + 4;
  static constexpr int ring = 0;                           // [ring_px][pitch] cost bytes
  static constexpr int da = ring + ring_px * pitch;        // [2][kCostSeg] u64
  static constexpr int span = kCostSeg + DP;               // staged targets (>= seg + DP - 1)
  static constexpr int db = da + 2 * kCostSeg * 8;         // [2][span] u64
  static constexpr int aux = db + 2 * span * 8;            // [span] u32 gray / gradient of targets
  static constexpr int valid = aux + span * 4;             // [span] u8
  static constexpr int inside = valid + span;              // [kCostSeg] u8
  static constexpr int aaux = inside + kCostSeg;           // [kCostSeg] u32 of the segment pixels
  static constexpr int total = (aaux + kCostSeg * 4 + 15) / 16 * 16;
  static_assert(da % 8 == 0, "u64 staging alignment");
};

// Packed central-difference gradient (dx | dy << 16, each as int16) of pixel (x, y).
__device__ __forceinline__ uint32_t gradient_of(const uint8_t* g, int w, int h, int x, int y) {
  if (x < 1 || x >= w - 1 || y < 1 || y >= h - 1) return 0;
  const int64_t p = (int64_t)y * w + x;
  const int dx = (int)g[p + 1] - (int)g[p - 1];
  const int dy = (int)g[p + w] - (int)g[p - w];
  return (uint32_t)(dx & 0xffff) | ((uint32_t)dy << 16);
}

template <int DP, int MODE, int WORDS>
__global__ void __launch_bounds__(kCostThreads) cost_rows_kernel(const CostPairArgs a) {
  extern __shared__ __align__(16) uint8_t csm[];
  using L = CostLayout<DP>;
  constexpr int G = DP / 16;                    // 16-disparity groups per pixel
  constexpr int TPP = kCostThreads / kCostSeg;  // threads per pixel
  constexpr int RMASK = L::ring_px - 1;
  uint8_t* ring = csm + L::ring;
  uint64_t* da = (uint64_t*)(csm + L::da);
  uint64_t* db = (uint64_t*)(csm + L::db);
  uint32_t* aux = (uint32_t*)(csm + L::aux);
  uint8_t* valid = csm + L::valid;
  uint8_t* inside = csm + L::inside;
  uint32_t* aaux = (uint32_t*)(csm + L::aaux);
  const CostArgs& c = a.view[0];  // left view: matching image left, targets right
  const int w = c.w, h = c.h, D = c.D, mind = c.min_disparity;
  const int rx = c.wx / 2, ry = c.wy / 2;
  const int segs = (w + kCostSeg - 1) / kCostSeg;
  const int64_t n = (int64_t)w * h;
  for (int y = blockIdx.x; y < h; y += gridDim.x) {
    const bool row_inside = y >= ry && y < h - ry;
    const int64_t row = (int64_t)y * w;
    int next_r = 0;  // next right-view segment to gather
    for (int s = 0; s < segs; s++) {
      const int x0 = s * kCostSeg;
      // Target of (x0 + i, k): qlo + i + DP - 1 - k.
      const int qlo = x0 - mind - (DP - 1);
      __syncthreads();  // the previous segment's staging and gathers are done
      for (int i = threadIdx.x; i < kCostSeg; i += kCostThreads) {
        const int x = x0 + i;
        const bool ok = x < w;
#pragma unroll
        for (int j = 0; j < WORDS; j++) da[j * kCostSeg + i] = ok ? c.desc_a[j * n + row + x] : 0;
        inside[i] = ok && row_inside && x >= rx && x < w - rx && c.tex_a[row + x];
        if (MODE == CSGM_COST_AD_CENSUS) aaux[i] = ok ? c.gray_a[row + x] : 0;
        if (MODE == CSGM_COST_CENSUS_GRADIENT) aaux[i] = ok ? gradient_of(c.gray_a, w, h, x, y) : 0;
      }
      for (int i = threadIdx.x; i < kCostSeg + DP - 1; i += kCostThreads) {
        const int q = qlo + i;
        const bool ok = q >= rx && q < w - rx;
#pragma unroll
        for (int j = 0; j < WORDS; j++) db[j * L::span + i] = ok ? c.desc_b[j * n + row + q] : 0;
        valid[i] = ok && c.tex_b[row + q] ? 0xff : 0;
        if (MODE == CSGM_COST_AD_CENSUS) aux[i] = ok ? c.gray_b[row + q] : 0;
        if (MODE == CSGM_COST_CENSUS_GRADIENT) aux[i] = ok ? gradient_of(c.gray_b, w, h, q, y) : 0;
      }
      __syncthreads();
      {
        const int i = threadIdx.x % kCostSeg;
        const bool in = inside[i];
        const uint64_t a0 = da[i], a1 = WORDS > 1 ? da[kCostSeg + i] : 0;
        const uint32_t av = aaux[i];
        const int cap = MODE == CSGM_COST_AD_CENSUS ? c.ad_cap : c.grad_cap;
        const uint32_t wh = (uint32_t)(c.weight * cap), wd = (uint32_t)((1000 - c.weight) * c.bits);
        const uint32_t half = (uint32_t)(1000 * cap / 2);
        uint32_t* dst_row = (uint32_t*)(ring + ((x0 + i) & RMASK) * L::pitch);
        for (int g = threadIdx.x / kCostSeg; g < G; g += TPP) {
          uint32_t word[4] = {0x80808080u, 0x80808080u, 0x80808080u, 0x80808080u};
          if (in) {
#pragma unroll
            for (int m = 0; m < 4; m++) {
              uint32_t v[4];
#pragma unroll
              for (int b = 0; b < 4; b++) {
                const int k = g * 16 + m * 4 + b;
                const int qi = i + DP - 1 - k;  // inside the staged span
                uint32_t ham = __popcll(a0 ^ db[qi]);
                if (WORDS > 1) ham += __popcll(a1 ^ db[L::span + qi]);
                uint32_t cost = ham;
                if (MODE != CSGM_COST_CENSUS) {
                  uint32_t diff;
                  if (MODE == CSGM_COST_AD_CENSUS) {
                    diff = (uint32_t)abs((int)av - (int)aux[qi]);
                  } else {
                    const uint32_t d2 = __vabsdiffs2(av, aux[qi]);
                    diff = (d2 & 0xffffu) + (d2 >> 16);
                  }
                  const uint32_t num = wh * ham + wd * min(diff, (uint32_t)cap) + half;
                  cost = (uint32_t)__umul64hi((unsigned long long)num, a.recip);
                }
                // valid[] is 0x00 / 0xff: cost where the target is valid, 0x80 elsewhere.
                const uint32_t keep = (uint32_t)(int32_t)(int8_t)valid[qi];
                v[b] = (cost & keep) | (0x80u & ~keep);
              }
              word[m] = __byte_perm(__byte_perm(v[0], v[1], 0x0040), __byte_perm(v[2], v[3], 0x0040),
                                    0x5410);
            }
            if (g * 16 + 16 > D) {  // disparities >= D are invalid
#pragma unroll
              for (int m = 0; m < 4; m++)
#pragma unroll
                for (int b = 0; b < 4; b++)
                  if (g * 16 + m * 4 + b >= D) word[m] = (word[m] & ~(0xffu << (8 * b))) | (0x80u << (8 * b));
            }
          }
#pragma unroll
          for (int m = 0; m < 4; m++) dst_row[g * 4 + m] = word[m];
        }
      }
      __syncthreads();
      // Left view: the segment's rows, coalesced.
      {
        const int npx = min(kCostSeg, w - x0);
        uint8_t* dst = a.out[0] + (row + x0) * DP;
        for (int t = threadIdx.x; t < npx * G; t += kCostThreads) {
          const int i = t / G, g = t % G;
          const uint32_t* src = (const uint32_t*)(ring + ((x0 + i) & RMASK) * L::pitch) + g * 4;
          __stcs((uint4*)(dst + (int64_t)i * DP + g * 16), make_uint4(src[0], src[1], src[2], src[3]));
        }
      }
      // Right view: every segment whose left pixels are all in the ring (all of them after the
      // last left segment; left pixels outside the image give 0x80).
      const int x_end = min(w - 1, x0 + kCostSeg - 1);
      const bool last = s == segs - 1;
      for (; next_r < segs &&
             (last || next_r * kCostSeg + kCostSeg - 1 + mind + DP - 1 <= x_end);
           next_r++) {
        const int xr0 = next_r * kCostSeg;
        const int npx = min(kCostSeg, w - xr0);
        uint8_t* dst = a.out[1] + (row + xr0) * DP;
        for (int t = threadIdx.x; t < npx * G; t += kCostThreads) {
          const int i = t / G, g = t % G;
          const int xb = xr0 + i + mind + g * 16;  // left pixel of k = 16g; k = 16g + m at xb + m
          uint32_t b[16];
          if (xb >= 0 && xb + 15 < w && (xb & RMASK) + 15 <= RMASK) {
            const uint8_t* src = ring + (xb & RMASK) * L::pitch + g * 16;
#pragma unroll
            for (int m = 0; m < 16; m++) b[m] = src[m * (L::pitch + 1)];
          } else {
#pragma unroll
            for (int m = 0; m < 16; m++) {
              const int x = xb + m;
              b[m] = x >= 0 && x < w ? ring[(x & RMASK) * L::pitch + g * 16 + m] : 0x80u;
            }
          }
          uint32_t word[4];
#pragma unroll
          for (int q = 0; q < 4; q++)
            word[q] = __byte_perm(__byte_perm(b[4 * q], b[4 * q + 1], 0x0040),
                                  __byte_perm(b[4 * q + 2], b[4 * q + 3], 0x0040), 0x5410);
          __stcs((uint4*)(dst + (int64_t)i * DP + g * 16),
                 make_uint4(word[0], word[1], word[2], word[3]));
        }
      }
    }
  }
}

template <int DP, int MODE, int WORDS>
cudaError_t launch_cost_rows_t(const CostPairArgs& a, int sm_count, cudaStream_t stream) {
  using L = CostLayout<DP>;
  auto kernel = cost_rows_kernel<DP, MODE, WORDS>;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, L::total);
  if (e != cudaSuccess) return e;
  // One CTA per image row (rows are equal work; the block scheduler balances them).
  (void)sm_count;
  kernel<<<a.view[0].h, kCostThreads, L::total, stream>>>(a);
  return cudaGetLastError();
}

template <int DP>
cudaError_t launch_cost_rows_dp(const CostPairArgs& a, int sm_count, cudaStream_t stream) {
  const int mode = a.view[0].mode, words = a.view[0].words;
  if (mode == CSGM_COST_CENSUS)
    return words > 1 ? launch_cost_rows_t<DP, CSGM_COST_CENSUS, 2>(a, sm_count, stream)
                     : launch_cost_rows_t<DP, CSGM_COST_CENSUS, 1>(a, sm_count, stream);
  if (mode == CSGM_COST_AD_CENSUS)
    return words > 1 ? launch_cost_rows_t<DP, CSGM_COST_AD_CENSUS, 2>(a, sm_count, stream)
                     : launch_cost_rows_t<DP, CSGM_COST_AD_CENSUS, 1>(a, sm_count, stream);
  return words > 1 ? launch_cost_rows_t<DP, CSGM_COST_CENSUS_GRADIENT, 2>(a, sm_count, stream)
                   : launch_cost_rows_t<DP, CSGM_COST_CENSUS_GRADIENT, 1>(a, sm_count, stream);
}

cudaError_t launch_cost_rows(const CostPairArgs& a, int sm_count, cudaStream_t stream) {
  switch (a.Dp) {
    case 64: return launch_cost_rows_dp<64>(a, sm_count, stream);
    case 128: return launch_cost_rows_dp<128>(a, sm_count, stream);
    case 192: return launch_cost_rows_dp<192>(a, sm_count, stream);
    case 256: return launch_cost_rows_dp<256>(a, sm_count, stream);
    default: return cudaErrorInvalidValue;
  }
}

// ceil(2^64 / d) for 2 <= d < 2^32.
unsigned long long reciprocal64(unsigned long long d) { return ~0ull / d + 1; }

// ---------------------------------------------------------------------------------------------
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
// Per-pixel penalty records (StereoCost.pathP2, StereoCost.java:44-48), one per stream and pixel
// in stream order (row yp, pixel xs).  Word i belongs to the stream's path i - (1,0), (0,1),
// (1,1), (-1,1) in stream coordinates - and holds pathP2 - P1 of the left view in bits 0-14 and
// of the right view in bits 16-30.  Bits 15 / 31 of word 0 flag a textured left / right pixel.
// A path without a predecessor gets P2 - P1 (its state is zero, so the value is never used).
struct PenaltyArgs {
  const uint8_t* gray[2];
  const uint8_t* tex[2];
  uint4* out;      // [2 streams][H][W]
  uint32_t* info;  // optional [H][W] pixel records of the 16-path line walks (KnightArgs::info)
  int W, H, p1, p2, edge_scale;
};

__global__ void penalty_kernel(const PenaltyArgs a) {
  // StereoCost.pathP2 depends on the gray difference only: a table of its 256 values replaces the
  // 64-bit division per path, view and pixel.
  __shared__ int step_p2[256];
  for (int d = threadIdx.x; d < 256; d += blockDim.x)
    step_p2[d] = path_p2(a.p1, a.p2, a.edge_scale, d, 0);
  __syncthreads();
  const int yp = blockIdx.y, s = blockIdx.z;
  const int W = a.W, H = a.H;
  // Several pixels of the row per thread, so that the table above is filled once per 1024 pixels.
  for (int xs = blockIdx.x * blockDim.x + threadIdx.x; xs < W; xs += gridDim.x * blockDim.x) {
    const int step = s ? -1 : 1;  // image offset of one stream step, in x and in y
    const int x = s ? W - 1 - xs : xs, y = s ? H - 1 - yp : yp;
    const int px[4] = {x - step, x, x - step, x + step};
    const int py[4] = {y, y - step, y - step, y - step};
    uint32_t word[4] = {0, 0, 0, 0};
#pragma unroll
    for (int v = 0; v < 2; v++) {
      const uint8_t* g = a.gray[v];
      const int center = g[(int64_t)y * W + x];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        int value = a.p2;
        if (px[i] >= 0 && px[i] < W && py[i] >= 0 && py[i] < H)
          value = step_p2[abs(center - (int)g[(int64_t)py[i] * W + px[i]])];
        word[i] |= (uint32_t)(value - a.p1) << (16 * v);
      }
      if (a.tex[v][(int64_t)y * W + x]) word[0] |= 0x8000u << (16 * v);
    }
    a.out[((int64_t)s * H + yp) * W + xs] = make_uint4(word[0], word[1], word[2], word[3]);
    if (a.info && s == 0) {
      const int64_t p = (int64_t)y * W + x;
      a.info[p] = (uint32_t)a.gray[0][p] | (uint32_t)a.gray[1][p] << 8 |
                  (a.tex[0][p] ? 1u : 0u) << 16 | (a.tex[1][p] ? 1u : 0u) << 24;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// The anti-diagonal paths (-1,1) and (1,-1) (CensusSgm.java:421-459, direction table entries 5
// and 6) follow the lines x + y = s, which are independent of each other: one warp per line,
// both views packed as in the sweep.  The forward pass walks (-1,1) from the line's upper-right
// end and stores its path costs as the line partial; the backward pass walks (1,-1) from the
// lower-left end, adds its path costs and stores the sum.  Costs, penalty records and (backward)
// the stored forward costs are prefetched kPrefetch pixels ahead.  Word 3 of the down stream's
// penalty record of a pixel is pathP2 - P1 towards (x+1, y-1), word 3 of the up stream's record
// pathP2 - P1 towards (x-1, y+1).
struct LineArgs {
  const uint8_t* cost[2];  // [H][W][Dp] per view
  const uint4* pen;        // [2 streams][H][W] penalty records, stream order
  uint32_t* part;          // [H][W][Dp] partial aggregate of the two anti-diagonal paths
  int W, H, D, p1;
  int* next;  // queue of lines (longest first) shared with the sweep's line warps; null: a warp
              // per line
};

constexpr int kLineWarps = 8;
constexpr int kPrefetch = 8;

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
// The same copy under a predicate (no branch around it; `src` is not read when `on` is false).
__device__ __forceinline__ void cp_async16_if(uint32_t dst, const void* src, bool on) {
  asm volatile(
      "{\n .reg .pred q;\n setp.ne.b32 q, %2, 0;\n @q cp.async.cg.shared.global [%0], [%1], 16;\n}\n" ::
          "r"(dst),
      "l"(src), "r"((int)on)
      : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Per-warp ring of kPrefetch pixel slots: costs of both views (Dp bytes each), the penalty record
// (16 bytes) and, on the return pass, the stored forward costs (Dp x 4 bytes).
template <int REGS>
struct LineSlot {
  static constexpr int Dp = 32 * REGS;
  static constexpr int cost = 0, pen = 2 * Dp, part = 2 * Dp + 16;
  static constexpr int bytes = 2 * Dp + 16 + 4 * Dp;
};

// Queue position idx -> line x + y = s, longest lines first: the min(W, H)-pixel plateau, then
// the two ramps from their long ends, alternately.
__device__ __forceinline__ int line_of(int idx, int W, int H) {
  const int m = min(W, H), M = max(W, H), plateau = M - m + 1;
  if (idx < plateau) return m - 1 + idx;
  const int j = idx - plateau, k = j / 2 + 1;
  return (j & 1) ? M - 1 + k : m - 1 - k;
}
__device__ __forceinline__ int line_len_at(int idx, int W, int H) {
  const int m = min(W, H), plateau = max(W, H) - m + 1;
  return idx < plateau ? m : m - ((idx - plateau) / 2 + 1);
}

// ---------------------------------------------------------------------------------------------
// Aggregation sweep.  Both views of one image row live in one warp: every 32-bit register holds
// one disparity of the left view (low half) and the same disparity of the right view (high
// half), lane l owning disparities l*REGS .. l*REGS+REGS-1.  The d-1 / d+1 neighbours of a
// register are therefore the neighbouring registers (one shuffle per lane edge), and every
// packed DPX min / add serves both views at once.
struct SweepArgs {
  const uint8_t* cost[2];  // [H][W][Dp] per view, image order; 0x80 = invalid (512)
  const uint4* pen;        // [2 streams][H][W] penalty records, stream order
  uint32_t* sum[2];        // per stream: partial aggregate [H][W][Dp], left | right << 16
  uint8_t* carry;          // [2 streams][nb][W][vslot] last-row states of each row block
  int* progress;           // [2][nb] carry pixels published per row block
  int* ticket;
  int* error;
  int W, H, D, nb, p1;
  long long timeout;
  LineArgs line;  // the anti-diagonal lines taken by the sweep's line warps (LW > 0)
  int line_slack;  // a line warp takes a line of len pixels while 100 * len <= slack * pixels left
};

// Shared-memory layout (byte offsets) of one sweep CTA.
template <int REGS, int NPATH, int K, int R>
struct SweepLayout {
  static constexpr int Dp = 32 * REGS;
  static constexpr int NV = NPATH - 1;  // paths whose predecessor lies in the row above
  static constexpr int RING = 4;        // ring slots between consecutive row warps
  static constexpr int NB = 4;          // cost chunk slots per row warp
  static constexpr int CS = 16 / K;     // carry chunk slots (16 pixels)
  // One pixel's vertical path states as computed (NV x Dp u16x2), then their row minima (NV
  // words, padded to 16 bytes): the successor subtracts the minimum itself, as the (1,0) path
  // does with its state in registers.
  static constexpr int vmins = NV * Dp * 4;
  static constexpr int vslot = vmins + 16;
  // One cost chunk: K x Dp cost bytes of the left view, of the right view, K penalty records.
  static constexpr int cslot = K * (2 * Dp + 16);
  static constexpr int bars = 0;                            // cost_full[R][NB], carry_full[CS]
  static constexpr int counters = bars + (R * NB + CS) * 8;  // carry_consumed, published
  static constexpr int cost = (counters + 16 + 127) / 128 * 128;
  static constexpr int ring = cost + R * NB * cslot;
  static constexpr int carry = ring + R * RING * vslot;
  static constexpr int zero = carry + CS * K * vslot;  // a pixel slot of zeros
  static constexpr int total = zero + vslot;
  // Rings of the line warps, kPrefetch LineSlots each.
  static constexpr int lines = (total + 127) / 128 * 128;
  static constexpr int with_lines(int lw) { return lines + lw * kPrefetch * LineSlot<REGS>::bytes; }
};

__device__ __forceinline__ int ld_acquire_cta(const int* p) {
  int v;
  asm volatile("ld.acquire.cta.shared::cta.b32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_cta(int* p, int v) {
  asm volatile("st.release.cta.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(p)), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_relaxed_gpu(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acq_rel_gpu() {
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
}
// Barrier among the R row warps only (the producer warp does not take part).
__device__ __forceinline__ void rows_barrier(int threads) {
  asm volatile("bar.sync 1, %0;" ::"r"(threads) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// REGS consecutive 32-bit words at a 8-byte aligned address (16-byte aligned when REGS % 4 == 0).
template <int REGS>
__device__ __forceinline__ void load_words(const void* p, uint32_t (&v)[REGS]) {
  if constexpr (REGS % 4 == 0) {
#pragma unroll
    for (int j = 0; j < REGS; j += 4) {
      const uint4 t = ((const uint4*)p)[j / 4];
      v[j] = t.x;
      v[j + 1] = t.y;
      v[j + 2] = t.z;
      v[j + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < REGS; j += 2) {
      const uint2 t = ((const uint2*)p)[j / 2];
      v[j] = t.x;
      v[j + 1] = t.y;
    }
  }
}
template <int REGS>
__device__ __forceinline__ void store_words(void* p, const uint32_t (&v)[REGS]) {
  if constexpr (REGS % 4 == 0) {
#pragma unroll
    for (int j = 0; j < REGS; j += 4)
      ((uint4*)p)[j / 4] = make_uint4(v[j], v[j + 1], v[j + 2], v[j + 3]);
  } else {
#pragma unroll
    for (int j = 0; j < REGS; j += 2) ((uint2*)p)[j / 2] = make_uint2(v[j], v[j + 1]);
  }
}
// Streaming global store of a partial aggregate (not re-read before the selection kernel).
template <int REGS>
__device__ __forceinline__ void store_words_cs(uint32_t* p, const uint32_t (&v)[REGS]) {
  if constexpr (REGS % 4 == 0) {
#pragma unroll
    for (int j = 0; j < REGS; j += 4)
      __stcs((uint4*)p + j / 4, make_uint4(v[j], v[j + 1], v[j + 2], v[j + 3]));
  } else {
#pragma unroll
    for (int j = 0; j < REGS; j += 2) __stcs((uint2*)p + j / 2, make_uint2(v[j], v[j + 1]));
  }
}

// Shared-memory loads and stores through 32-bit shared-window addresses (volatile, so they keep
// their order relative to the barriers and mbarrier waits around them).
__device__ __forceinline__ uint32_t lds_u16(uint32_t a) {
  unsigned short v;
  asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ uint32_t lds_u32(uint32_t a) {
  uint32_t v;
  asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ uint2 lds_v2(uint32_t a) {
  uint2 v;
  asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(a));
  return v;
}
__device__ __forceinline__ uint4 lds_v4(uint32_t a) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(a));
  return v;
}
__device__ __forceinline__ void sts_v2(uint32_t a, uint32_t x, uint32_t y) {
  asm volatile("st.shared.v2.u32 [%0], {%1, %2};" ::"r"(a), "r"(x), "r"(y));
}
__device__ __forceinline__ void sts_v4(uint32_t a, uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
  asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(a), "r"(x), "r"(y), "r"(z), "r"(w));
}
template <int REGS>
__device__ __forceinline__ void lds_words(uint32_t a, uint32_t (&v)[REGS]) {
  if constexpr (REGS % 4 == 0) {
#pragma unroll
    for (int j = 0; j < REGS; j += 4) {
      const uint4 t = lds_v4(a + 4 * j);
      v[j] = t.x;
      v[j + 1] = t.y;
      v[j + 2] = t.z;
      v[j + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < REGS; j += 2) {
      const uint2 t = lds_v2(a + 4 * j);
      v[j] = t.x;
      v[j + 1] = t.y;
    }
  }
}
template <int REGS>
__device__ __forceinline__ void sts_words(uint32_t a, const uint32_t (&v)[REGS]) {
  if constexpr (REGS % 4 == 0) {
#pragma unroll
    for (int j = 0; j < REGS; j += 4) sts_v4(a + 4 * j, v[j], v[j + 1], v[j + 2], v[j + 3]);
  } else {
#pragma unroll
    for (int j = 0; j < REGS; j += 2) sts_v2(a + 4 * j, v[j], v[j + 1]);
  }
}

template <int REGS>
struct PathState {
  uint32_t v[REGS];
  uint32_t m;  // packed row minima (left | right << 16)
};

template <int REGS>
__device__ __forceinline__ void zero_state(PathState<REGS>& s) {
#pragma unroll
  for (int j = 0; j < REGS; j++) s.v[j] = 0;
  s.m = 0;
}

// Path `path` of the pixel slot at shared address `slot` (vslot layout with the minima at byte
// `vmins`) for the lane whose words start `lane_off` bytes in: its state and its row minimum.
template <int REGS>
__device__ __forceinline__ void load_path(uint32_t slot, uint32_t lane_off, int vmins, int path,
                                          PathState<REGS>& s) {
  lds_words<REGS>(slot + lane_off + path * (32 * REGS * 4), s.v);
  s.m = lds_u32(slot + vmins + 4 * path);
}

// Cost of the pad disparities D..Dp-1 in both halves.  A pad lane's path cost is at least 1536,
// a real one at most 512 + P2 <= 1023, so a pad lane is never a row minimum and never the
// strict minimum of a real lane's candidates (its normalised state exceeds P2 + 1); and with 16
// paths a pad total stays below 16 x (1536 + 511) < 2^16, above the invalid threshold 16 x 512.
constexpr uint32_t kPadCost = 0x06000600u;

// This lane's costs of both views as packed u16 pairs (widen_costs = load_cost_words +
// widen_words): byte j of each view widened, 0x80 -> 512, and pad[j] ORed in (disparities >= D
// are lifted to kPadCost so they never win a minimum).
template <int REGS>
struct CostWords {  // this lane's raw cost bytes of both views
  static constexpr int NW = (REGS + 3) / 4;
  uint32_t a[NW], b[NW];
};
template <int REGS>
__device__ __forceinline__ void load_cost_words(uint32_t c0, uint32_t c1, CostWords<REGS>& w) {
  uint32_t(&a)[CostWords<REGS>::NW] = w.a;
  uint32_t(&b)[CostWords<REGS>::NW] = w.b;
  if constexpr (REGS == 2) {
    a[0] = lds_u16(c0);
    b[0] = lds_u16(c1);
  } else if constexpr (REGS == 4) {
    a[0] = lds_u32(c0);
    b[0] = lds_u32(c1);
  } else if constexpr (REGS == 6) {
    a[0] = lds_u16(c0) | (lds_u16(c0 + 2) << 16);
    a[1] = lds_u16(c0 + 4);
    b[0] = lds_u16(c1) | (lds_u16(c1 + 2) << 16);
    b[1] = lds_u16(c1 + 4);
  } else {
    const uint2 t0 = lds_v2(c0), t1 = lds_v2(c1);
    a[0] = t0.x;
    a[1] = t0.y;
    b[0] = t1.x;
    b[1] = t1.y;
  }
}
template <int REGS>
__device__ __forceinline__ void widen_words(const CostWords<REGS>& w, const uint32_t (&pad)[REGS],
                                            uint32_t (&c)[REGS]) {
  const uint32_t(&a)[CostWords<REGS>::NW] = w.a;
  const uint32_t(&b)[CostWords<REGS>::NW] = w.b;
#pragma unroll
  for (int j = 0; j < REGS; j++) {
    const uint32_t i = j % 4;
    // byte i of a, its sign, byte i of b, its sign
    const uint32_t sel = i | ((i | 8) << 4) | ((4 + i) << 8) | (((4 + i) | 8) << 12);
    c[j] = (prmt(a[j / 4], b[j / 4], sel) & 0x027f027fu) | pad[j];
  }
}
template <int REGS>
__device__ __forceinline__ void widen_costs(uint32_t c0, uint32_t c1, const uint32_t (&pad)[REGS],
                                            uint32_t (&c)[REGS]) {
  CostWords<REGS> w;
  load_cost_words<REGS>(c0, c1, w);
  widen_words<REGS>(w, pad, c);
}

// Lane minimum of REGS packed pairs.
template <int REGS>
__device__ __forceinline__ uint32_t lane_min(const uint32_t (&v)[REGS]) {
  uint32_t m = v[0];
  int j = 1;
#pragma unroll
  for (; j + 1 < REGS; j += 2) m = __vimin3_u16x2(m, v[j], v[j + 1]);
  if (j < REGS) m = __vminu2(m, v[j]);
  return m;
}

// One pixel of every path of the stream (CensusSgm.java:436-457 for both views at once):
//   L(k) = C(k) + min(Lp(k), Lp(k-1) + P1, Lp(k+1) + P1, minLp + P2') - minLp,
// q = minLp + P2' - P1 (packed), with the row minimum of the new state for the next pixel.
// A zero predecessor state (no predecessor, or an untextured one) gives L = C.
template <int REGS, int NP>
__device__ __forceinline__ void paths_step(const PathState<REGS> (&prev)[NP],
                                           const uint32_t (&q)[NP], uint32_t p1x2,
                                           const uint32_t (&c)[REGS], uint32_t lo_edge,
                                           uint32_t hi_edge, PathState<REGS> (&out)[NP]) {
  uint32_t below[NP], above[NP];
#pragma unroll
  for (int i = 0; i < NP; i++) {
    below[i] = __shfl_up_sync(0xffffffffu, prev[i].v[REGS - 1], 1) | lo_edge;
    above[i] = __shfl_down_sync(0xffffffffu, prev[i].v[0], 1) | hi_edge;
  }
#pragma unroll
  for (int i = 0; i < NP; i++) {
#pragma unroll
    for (int j = 0; j < REGS; j++) {
      const uint32_t dn = j == 0 ? below[i] : prev[i].v[j - 1];
      const uint32_t up = j == REGS - 1 ? above[i] : prev[i].v[j + 1];
      const uint32_t t =
          __viaddmin_u16x2(__vimin3_u16x2(dn, up, q[i]), p1x2, prev[i].v[j]);
      out[i].v[j] = t + c[j] - prev[i].m;  // t >= minLp in both halves: no borrow
    }
    // Warp minima of both halves: the high 16 bits of a 32-bit minimum are the minimum of the
    // high halves, so one reduction of mm and one of mm << 16 give both.
    const uint32_t mm = lane_min<REGS>(out[i].v);
    const uint32_t hi = __reduce_min_sync(0xffffffffu, mm);
    const uint32_t lo = __reduce_min_sync(0xffffffffu, mm << 16);
    out[i].m = __byte_perm(lo, hi, 0x7632);
  }
}

// One warp walks line x + y = `line` forward and back; `ring` is the warp's shared-memory ring of
// kPrefetch LineSlots.  Returns with no copy in flight.
template <int REGS>
__device__ __forceinline__ void walk_line(const LineArgs& a, int line, uint32_t ring, int lane) {
  constexpr int Dp = 32 * REGS, CH = Dp / 16;  // 16-byte chunks per view's cost line
  using S = LineSlot<REGS>;
  const int W = a.W, H = a.H;
  const int x0 = min(line, W - 1), y0 = line - x0;  // upper-right end of the line
  const int len = min(x0 + 1, H - y0);               // pixel i: (x0 - i, y0 + i)
  const uint32_t lo_edge = lane == 0 ? 0xffffffffu : 0u;
  const uint32_t hi_edge = lane == 31 ? 0xffffffffu : 0u;
  uint32_t pad[REGS];
#pragma unroll
  for (int j = 0; j < REGS; j++) pad[j] = lane * REGS + j >= a.D ? kPadCost : 0u;
  const uint32_t p1x2 = (uint32_t)a.p1 * 0x10001u;
  uint32_t* part = a.part + lane * REGS;
  const int64_t step = (int64_t)W - 1;  // pixel-index step along the line (down-left)
  const int64_t p0 = (int64_t)y0 * W + x0;
  // Per lane, once per line: lanes 0 .. 2 CH - 1 copy one 16-byte chunk of a view's costs, lane
  // 31 the penalty record.  The up stream's record of pixel i sits at pen_up0 - i * step (its
  // stream coordinates mirror the image in x and y).  Along the line every address advances by a
  // fixed step per pixel, so the copies and stores use running pointers.
  const bool cost_lane = lane < 2 * CH;
  const uint32_t cost_dst = S::cost + (cost_lane ? (lane / CH) * Dp + (lane % CH) * 16 : 0);
  const uint8_t* cost_src =
      (cost_lane && lane >= CH ? a.cost[1] : a.cost[0]) + (cost_lane ? (lane % CH) * 16 : 0);
  const int64_t pen_up0 = ((int64_t)2 * H - 1 - y0) * W + (W - 1 - x0);
  const int64_t cost_stride = step * Dp;  // bytes of a cost volume per pixel along the line
  const int64_t part_stride = step * Dp;  // words of the partial per pixel along the line

  // Position of the next pixel to fetch (its copies' sources) and of the pixel being stored.
  struct Cursor {
    const uint8_t* cost;
    const uint4* pen;
    const uint32_t* part;
  };
  // Issues the copies of the cursor's pixel into ring slot `slot` as one commit group (empty if
  // `on` is false, so the group count stays in step).
  auto fetch = [&](int slot, const Cursor& f, bool on, bool back) {
    const uint32_t s = ring + slot * S::bytes;
    cp_async16_if(s + cost_dst, f.cost, on && cost_lane);
    cp_async16_if(s + S::pen, f.pen, on && lane == 31);
    if (back) {
#pragma unroll
      for (int c = lane; c < Dp / 4; c += 32) cp_async16_if(s + S::part + c * 16, f.part + c * 4, on);
    }
    cp_async_commit();
  };
  // Consumes ring slot `slot`: this lane's widened costs, penalty and texture words.
  auto take = [&](int slot, uint32_t (&c)[REGS], uint32_t& pq, uint32_t& pt) {
    const uint32_t s = ring + slot * S::bytes;
    widen_costs<REGS>(s + S::cost + lane * REGS, s + S::cost + Dp + lane * REGS, pad, c);
    const uint4 r = lds_v4(s + S::pen);
    pq = r.w;
    pt = r.x;
  };

  PathState<REGS> cur;
  // Forward: (-1,1), pixel i's predecessor is pixel i - 1.
  {
    zero_state(cur);
    Cursor f{cost_src + p0 * Dp, a.pen + p0, nullptr};  // pixel 0
    uint32_t* out_ptr = part + p0 * Dp;
    auto advance = [&](Cursor& c) {
      c.cost += cost_stride;
      c.pen += step;
    };
#pragma unroll
    for (int k = 0; k < kPrefetch; k++) {
      fetch(k, f, k < len, false);
      advance(f);
    }
    // One pixel (ring slot k) while `i < len`.
    auto pixel = [&](int k, int i, auto guarded) {
      if (decltype(guarded)::value && i >= len) return;
      cp_async_wait<kPrefetch - 1>();
      __syncwarp();
      uint32_t c[REGS], pq, pt;
      take(k, c, pq, pt);
      __syncwarp();  // every lane has read the slot before it is refilled
      fetch(k, f, i + kPrefetch < len, false);
      advance(f);
      const uint32_t q[1] = {cur.m + (pq & 0x7fff7fffu)};
      const uint32_t keep = prmt(pt, 0, 0xbb99u);
      PathState<REGS> prev[1] = {cur}, out[1];
      paths_step<REGS, 1>(prev, q, p1x2, c, lo_edge, hi_edge, out);
      store_words<REGS>(out_ptr, out[0].v);
      out_ptr += part_stride;
      cur = out[0];
      if (keep != 0xffffffffu) {
#pragma unroll
        for (int j = 0; j < REGS; j++) cur.v[j] &= keep;
        cur.m &= keep;
      }
    };
    for (int base = 0; base < len; base += kPrefetch) {
#pragma unroll
      for (int k = 0; k < kPrefetch; k++) pixel(k, base + k, std::true_type{});
    }
    cp_async_wait<0>();
  }
  // The return pass copies the stored forward costs back from L2 (cp.async.cg), some of them
  // written by other lanes just now: every lane's stores reach L2 before any lane copies.
  __threadfence();
  __syncwarp();
  // Backward: (1,-1), pixel i's predecessor is pixel i + 1; adds to the stored forward costs.
  {
    zero_state(cur);
    const int64_t pl = p0 + (int64_t)(len - 1) * step;  // pixel len - 1
    Cursor f{cost_src + pl * Dp, a.pen + (pen_up0 - (int64_t)(len - 1) * step),
             a.part + pl * Dp};
    uint32_t* out_ptr = part + pl * Dp;
    auto advance = [&](Cursor& c) {
      c.cost -= cost_stride;
      c.pen += step;
      c.part -= part_stride;
    };
#pragma unroll
    for (int k = 0; k < kPrefetch; k++) {
      fetch(k, f, k < len, true);
      advance(f);
    }
    // Pixel len - 1 - n (ring slot k), the n-th of the pass.
    auto pixel = [&](int k, int n, auto guarded) {
      if (decltype(guarded)::value && n >= len) return;
      cp_async_wait<kPrefetch - 1>();
      __syncwarp();
      uint32_t c[REGS], pq, pt, fwd[REGS];
      take(k, c, pq, pt);
      lds_words<REGS>(ring + k * S::bytes + S::part + lane * REGS * 4, fwd);
      __syncwarp();
      fetch(k, f, n + kPrefetch < len, true);
      advance(f);
      const uint32_t q[1] = {cur.m + (pq & 0x7fff7fffu)};
      const uint32_t keep = prmt(pt, 0, 0xbb99u);
      PathState<REGS> prev[1] = {cur}, out[1];
      paths_step<REGS, 1>(prev, q, p1x2, c, lo_edge, hi_edge, out);
      uint32_t sum[REGS];
#pragma unroll
      for (int j = 0; j < REGS; j++) sum[j] = fwd[j] + out[0].v[j];
      store_words_cs<REGS>(out_ptr, sum);
      out_ptr -= part_stride;
      cur = out[0];
      if (keep != 0xffffffffu) {
#pragma unroll
        for (int j = 0; j < REGS; j++) cur.v[j] &= keep;
        cur.m &= keep;
      }
    };
    for (int base = 0; base < len; base += kPrefetch) {
#pragma unroll
      for (int k = 0; k < kPrefetch; k++) pixel(k, base + k, std::true_type{});
    }
  }
  cp_async_wait<0>();
}

template <int REGS>
__global__ void __launch_bounds__(kLineWarps * 32) lines_kernel(const LineArgs a) {
  extern __shared__ __align__(16) uint8_t lsm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t ring = smem_u32(lsm) + warp * kPrefetch * LineSlot<REGS>::bytes;
  const int lines = a.W + a.H - 1;
  if (!a.next) {
    const int line = blockIdx.x * kLineWarps + warp;
    if (line < lines) walk_line<REGS>(a, line, ring, lane);
    return;
  }
  // The lines the sweep's line warps left: taken from the queue until it is empty.
  for (;;) {
    int idx = 0;
    if (lane == 0) idx = atomicAdd(a.next, 1);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= lines) return;
    walk_line<REGS>(a, line_of(idx, a.W, a.H), ring, lane);
  }
}

// ---------------------------------------------------------------------------------------------
// The 16-path extension's eight paths (+-1,+-2), (+-2,+-1) (direction table entries 8..15): four
// families of independent lines, family (dx, dy) with dy > 0 covering the paths (dx, dy) and
// (-dx, -dy).  A line starts at a pixel whose predecessor (x - dx, y - dy) is outside the image
// and visits start + i * (dx, dy).  One warp walks a line forward (path (dx, dy)) and back (path
// (-dx, -dy)), both views packed as in the sweep, and each pass adds its path costs to the lines
// partial aggregate: the families run one after another after the anti-diagonal lines, so every
// read-modify-write of a pixel's partial is ordered.  Per pixel the warp's ring brings both views'
// costs, the pixel's record (both grays and texture flags) and the partial, kPrefetch pixels
// ahead; pathP2 - P1 (StereoCost.java:44-48) comes from a per-CTA table over |gray difference|.
struct KnightArgs {
  const uint8_t* cost[2];  // [H][W][Dp] per view
  const uint32_t* info;    // [H][W] gray_l | gray_r << 8 | textured_l << 16 | textured_r << 24
  uint32_t* part;          // [H][W][Dp] lines partial, accumulated
  int W, H, D, p1, p2, edge_scale, dx, dy;
};

template <int REGS>
struct KnightSlot {
  static constexpr int Dp = 32 * REGS;
  static constexpr int cost = 0, info = 2 * Dp, part = 2 * Dp + 16;
  static constexpr int bytes = 2 * Dp + 16 + 4 * Dp;
};

__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}

template <int REGS>
__global__ void __launch_bounds__(kLineWarps * 32) knight_kernel(const KnightArgs a) {
  constexpr int Dp = 32 * REGS, CH = Dp / 16;
  using S = KnightSlot<REGS>;
  extern __shared__ __align__(16) uint8_t ksm[];
  __shared__ uint32_t step_p2[256];  // pathP2 - P1 for a gray difference d
  for (int d = threadIdx.x; d < 256; d += blockDim.x)
    step_p2[d] = (uint32_t)(path_p2(a.p1, a.p2, a.edge_scale, d, 0) - a.p1);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int W = a.W, H = a.H, dx = a.dx, dy = a.dy;
  const int64_t line = (int64_t)blockIdx.x * kLineWarps + warp;
  if (line >= line_count(W, H, dx, dy)) return;
  int x0, y0;
  line_start(line, W, H, dx, dy, x0, y0);
  const int len = min((H - 1 - y0) / dy + 1, dx > 0 ? (W - 1 - x0) / dx + 1 : x0 / (-dx) + 1);
  const int64_t p0 = (int64_t)y0 * W + x0, step = (int64_t)dy * W + dx;
  const uint32_t ring = smem_u32(ksm) + warp * kPrefetch * S::bytes;
  const uint32_t lo_edge = lane == 0 ? 0xffffffffu : 0u;
  const uint32_t hi_edge = lane == 31 ? 0xffffffffu : 0u;
  uint32_t pad[REGS];
#pragma unroll
  for (int j = 0; j < REGS; j++) pad[j] = lane * REGS + j >= a.D ? kPadCost : 0u;
  const uint32_t p1x2 = (uint32_t)a.p1 * 0x10001u;
  uint32_t* part = a.part + lane * REGS;

  // Copies of pixel i into ring slot `slot`, one commit group (empty off the line).
  auto fetch = [&](int slot, int i) {
    if (i >= 0 && i < len) {
      const int64_t p = p0 + i * step;
      const uint32_t sl = ring + slot * S::bytes;
      if (lane < 2 * CH) {
        const int view = lane / CH, chunk = lane % CH;
        cp_async16(sl + S::cost + view * Dp + chunk * 16,
                   (view ? a.cost[1] : a.cost[0]) + p * Dp + chunk * 16);
      }
      if (lane == 31) cp_async4(sl + S::info, a.info + p);
#pragma unroll
      for (int c = lane; c < Dp / 4; c += 32) cp_async16(sl + S::part + c * 16, a.part + p * Dp + c * 4);
    }
    cp_async_commit();
  };
  // One pass: forward (back = false, pixel i after i - 1) or back (pixel i after i + 1).
  auto pass = [&](bool back) {
    PathState<REGS> cur;
    zero_state(cur);
    uint32_t prev_info = 0;
    auto at = [&](int k) { return back ? len - 1 - k : k; };
#pragma unroll
    for (int k = 0; k < kPrefetch; k++) fetch(k, at(k));
    for (int base = 0; base < len; base += kPrefetch) {
#pragma unroll
      for (int k = 0; k < kPrefetch; k++) {
        if (base + k < len) {
          const int i = at(base + k);
          cp_async_wait<kPrefetch - 1>();
          __syncwarp();
          const uint32_t sl = ring + k * S::bytes;
          uint32_t c[REGS], old[REGS];
          widen_costs<REGS>(sl + S::cost + lane * REGS, sl + S::cost + Dp + lane * REGS, pad, c);
          const uint32_t info = lds_u32(sl + S::info);
          lds_words<REGS>(sl + S::part + lane * REGS * 4, old);
          __syncwarp();  // every lane has read the slot before it is refilled
          fetch(k, at(base + k + kPrefetch));
          // The matching view's grays: left view in bits 0-7, right view in bits 8-15.  The first
          // pixel has a zero state, so its penalty is never used.
          const int dl = abs((int)(info & 0xffu) - (int)(prev_info & 0xffu));
          const int dr = abs((int)((info >> 8) & 0xffu) - (int)((prev_info >> 8) & 0xffu));
          const uint32_t q[1] = {cur.m + (step_p2[dl] | (step_p2[dr] << 16))};
          PathState<REGS> prev[1] = {cur}, out[1];
          paths_step<REGS, 1>(prev, q, p1x2, c, lo_edge, hi_edge, out);
          uint32_t sum[REGS];
#pragma unroll
          for (int j = 0; j < REGS; j++) sum[j] = old[j] + out[0].v[j];
          if (back)
            store_words_cs<REGS>(part + (p0 + i * step) * Dp, sum);
          else
            store_words<REGS>(part + (p0 + i * step) * Dp, sum);
          cur = out[0];
          // Successors of an untextured pixel start afresh (CensusSgm.java:432-433).
          const uint32_t keep = ((info >> 16) & 1u ? 0xffffu : 0u) | ((info >> 24) & 1u ? 0xffff0000u : 0u);
          if (keep != 0xffffffffu) {
#pragma unroll
            for (int j = 0; j < REGS; j++) cur.v[j] &= keep;
            cur.m &= keep;
          }
          prev_info = info;
        }
      }
    }
    cp_async_wait<0>();
  };
  pass(false);
  // The return pass copies the forward pass's sums back from L2 (cp.async), some of them stored
  // by other lanes just now: every lane's stores reach L2 before any lane copies.
  __threadfence();
  __syncwarp();
  pass(true);
}

template <int REGS>
cudaError_t launch_knights(KnightArgs a, cudaStream_t stream) {
  const int shared = kLineWarps * kPrefetch * KnightSlot<REGS>::bytes;
  cudaError_t e = cudaFuncSetAttribute(knight_kernel<REGS>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, shared);
  if (e != cudaSuccess) return e;
  // The four families one after another: (1,2), (2,1), (-1,2), (-2,1).
  const int family[4][2] = {{1, 2}, {2, 1}, {-1, 2}, {-2, 1}};
  for (const auto& f : family) {
    a.dx = f[0];
    a.dy = f[1];
    const int64_t lines = line_count(a.W, a.H, a.dx, a.dy);
    knight_kernel<REGS><<<(int)((lines + kLineWarps - 1) / kLineWarps), kLineWarps * 32, shared,
                           stream>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// One CTA = R row warps + a carry-in warp + a publisher warp (+ LW line warps), one row block of
// one stream.
//  * "down" (stream 0) runs rows top to bottom and pixels left to right and owns (1,0), (0,1),
//    (1,1) (NPATH = 3; (1,0), (0,1) in 4-path mode, NPATH = 2); "up" (stream 1) is the same code
//    on the image mirrored in x and y and owns the opposite paths.  The anti-diagonal paths,
//    whose predecessor lies one pixel ahead in the row above, are walked line by line: by the
//    line warps (walk_line) on the issue slots the row warps leave idle, or by lines_kernel.
//  * Row warp w holds stream row b*R + w of both views and processes stream pixel xs at step
//    xs + w; the row warps meet at a named barrier once per step.  The vertical path states of
//    a pixel reach the next row through a shared-memory ring; the (1,0) state stays in registers.
//  * Each row warp bulk-copies its own cost chunks (both views + penalty records) NB chunks
//    ahead; the last row warp also stores its vertical states as the block's carry row.
//  * The carry-in warp fetches the previous block's carry row chunk by chunk once its progress
//    counter covers the chunk; the publisher warp advances this block's progress counter after a
//    GPU-scope fence (both off the row warps' critical path).
//  * CTAs take tickets in launch order and only wait on lower tickets, so the schedule cannot
//    deadlock even when not every CTA is resident.
//  * One CTA per SM at most is planned for, so the compiler may give a thread all the registers
//    it wants (about 90 at D = 128: 2.39 ms per cfg1 sweep, against 2.71 ms at the 63 it picks
//    when asked to fit three CTAs).
template <int REGS, int NPATH, int K, int R, int LW>
__global__ void __launch_bounds__((R + 2 + LW) * 32, 1) sweep_kernel(const SweepArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  using L = SweepLayout<REGS, NPATH, K, R>;
  constexpr int Dp = L::Dp, NV = L::NV, RING = L::RING, NB = L::NB, CS = L::CS;
  uint64_t* full = (uint64_t*)(smem + L::bars);     // [R][NB]
  uint64_t* carry_full = full + R * NB;             // [CS]
  int* carry_consumed = (int*)(smem + L::counters);  // carry chunks row warp 0 no longer needs
  int* published = carry_consumed + 1;              // carry chunks row warp R-1 has written
  int* row_done = carry_consumed + 2;               // chunks row warp 0 has finished
  uint8_t* carry_buf = smem + L::carry;
  __shared__ int s_ticket;

  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    s_ticket = atomicAdd(a.ticket, 1);
    for (int i = 0; i < R * NB + CS; i++) mbar_init(&full[i], 1);
    *carry_consumed = 0;
    *published = 0;
    *row_done = 0;
  }
  for (int i = threadIdx.x; i < L::vslot / 4; i += blockDim.x) ((uint32_t*)(smem + L::zero))[i] = 0;
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();

  const int ticket = s_ticket;
  const int stream = ticket & 1, b = ticket >> 1;
  const bool mirror = stream != 0;
  const int W = a.W, H = a.H;
  const bool has_next = b + 1 < a.nb;
  const long long limit = a.timeout;
  int* const err = a.error;
  const int nchunks = (W + K - 1) / K;
  auto chunk_n = [&](int c) { return min(K, W - c * K); };

  if (w == R) {
    // --------------------------------------------------------------- carry-in warp
    // Copies the previous block's carry row into the carry ring as soon as its progress counter
    // covers a chunk, every covered chunk at once.
    if (lane != 0 || b == 0) return;
    const int* prev_progress = &a.progress[stream * a.nb + b - 1];
    const uint8_t* carry_in = a.carry + (int64_t)(stream * a.nb + b - 1) * W * L::vslot;
    int next_carry = 0, prev_seen = 0;
    long long last = clock64();
    while (next_carry < nchunks) {
      const int room = ld_acquire_cta(carry_consumed) + CS;  // chunks below this fit the ring
      if (next_carry < room && prev_seen < min(W, (next_carry + 1) * K))
        prev_seen = ld_relaxed_gpu(prev_progress);
      const int avail = min(min(room, nchunks), prev_seen >= W ? nchunks : prev_seen / K);
      if (next_carry < avail) {
        fence_acq_rel_gpu();  // the carry data behind the observed progress is visible
        fence_proxy_async_global();
        fence_proxy_async_shared();
        for (; next_carry < avail; next_carry++) {
          const int ch = next_carry;
          uint64_t* bar = &carry_full[ch % CS];
          // The slot's previous copy has landed (row warp 0 waited for it before releasing the
          // slot, unless its wait gave up after an error: then this wait sees the copy land).
          if (ch >= CS) wait_bar(bar, ((ch - CS) / CS) & 1, err, kDrainLimit, 5, false);
          const uint32_t bytes = (uint32_t)(chunk_n(ch) * L::vslot);
          mbar_expect_tx(bar, bytes);
          bulk_copy(carry_buf + (ch % CS) * K * L::vslot, carry_in + (int64_t)ch * K * L::vslot,
                    bytes, bar);
        }
        last = clock64();
      } else {
        if (*(volatile int*)err) break;
        if (clock64() - last > limit) {
          atomicExch(err, 6);
          break;
        }
        __nanosleep(32);
      }
    }
    // Every issued carry copy lands before the CTA's shared memory is released.
    for (int ch = max(0, next_carry - CS); ch < next_carry; ch++)
      wait_bar(&carry_full[ch % CS], (ch / CS) & 1, err, kDrainLimit, 5, false);
    return;
  }
  if (w >= R + 2) {
    // --------------------------------------------------------------- line warps
    // Anti-diagonal lines from the queue, longest first, while this block's rows are busy: a
    // warp takes the next line only if it is no longer than the pixels row warp 0 still has to
    // go (a line step costs well under half a sweep step), so the line work does not hold the
    // SM beyond the block's own rows.  The lines nobody took are walked after the sweep.
    if constexpr (LW > 0) {
      const uint32_t ring = smem_u32(smem) + L::lines + (w - R - 2) * kPrefetch * LineSlot<REGS>::bytes;
      const int lines = W + H - 1;
      for (;;) {
        int idx = INT_MAX;
        if (lane == 0) {
          const int head = *(volatile int*)a.line.next;
          const int left = W - K * *(volatile int*)row_done;
          if (head < lines && 100 * line_len_at(head, W, H) <= a.line_slack * left)
            idx = atomicAdd(a.line.next, 1);
        }
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= lines) break;
        walk_line<REGS>(a.line, line_of(idx, W, H), ring, lane);
      }
    }
    return;
  }
  if (w == R + 1) {
    // --------------------------------------------------------------- publisher warp
    // Makes the carry chunks the last row warp has written visible GPU-wide, then advances this
    // block's progress counter (the fence stays off the row warps' critical path).
    if (lane != 0 || !has_next) return;
    int* my_progress = &a.progress[stream * a.nb + b];
    int done_pub = 0;
    long long last = clock64();
    while (done_pub < nchunks) {
      const int done = ld_acquire_cta(published);
      if (done > done_pub) {
        __threadfence();
        atomicExch(my_progress, min(W, done * K));
        done_pub = done;
        last = clock64();
      } else {
        if (*(volatile int*)err) break;
        if (clock64() - last > limit) {
          atomicExch(err, 6);
          break;
        }
        __nanosleep(32);
      }
    }
    return;
  }

  // -------------------------------------------------------------------- row warps
  const int yp = b * R + w;  // row in stream order
  if (yp >= H) {
    // Rows beyond the image: nobody reads them, but the warp takes part in every step barrier.
    for (int step = 0; step < W + (R - 1); step++) rows_barrier(R * 32);
    return;
  }
  const int y = mirror ? H - 1 - yp : yp;
  const bool use_carry = w == 0 && b > 0;  // the row above lives in the previous CTA
  const bool publish = w == R - 1 && has_next;
  uint8_t* my_slots = smem + L::cost + w * NB * L::cslot;
  uint64_t* my_full = full + w * NB;
  // Shared-window addresses (32-bit), this lane's offset inside a pixel slot folded in.
  const uint32_t sm0 = smem_u32(smem);
  const uint32_t lane_off = lane * REGS * 4;
  const uint32_t slots_a = sm0 + L::cost + w * NB * L::cslot;
  const uint32_t ring_a = sm0 + L::ring + w * RING * L::vslot;
  const uint32_t zero_a = sm0 + L::zero;
  // Predecessor row: the ring of the warp above, the carry buffer, or (first image row) the zero
  // slot for every pixel.
  const uint32_t up_a = yp == 0     ? sm0 + L::zero
                        : use_carry ? sm0 + L::carry
                                    : sm0 + L::ring + (w - 1) * RING * L::vslot;
  const int up_mask = yp == 0 ? 0 : use_carry ? CS * K - 1 : RING - 1;
  uint8_t* carry_out = a.carry + (int64_t)(stream * a.nb + b) * W * L::vslot;
  const uint8_t* cost_row0 = a.cost[0] + (int64_t)y * W * Dp;
  const uint8_t* cost_row1 = a.cost[1] + (int64_t)y * W * Dp;
  const uint4* pen_row = a.pen + ((int64_t)stream * H + yp) * W;
  // Partial aggregate of the current stream pixel (this lane's words), advanced by sum_step.
  uint32_t* sum_ptr = (stream ? a.sum[1] : a.sum[0]) + ((int64_t)y * W + (mirror ? W - 1 : 0)) * Dp +
                      lane * REGS;
  const int sum_step = mirror ? -Dp : Dp;
  // Cost bytes of chunk pixel `off` sit at slot + cost_first + off * cost_step (image order).
  const int cost_first_full = (mirror ? (K - 1) * Dp : 0) + lane * REGS;
  const int cost_step = mirror ? -Dp : Dp;
  uint8_t* carry_ptr = carry_out;  // this row's carry slot of the current pixel

  auto issue_chunk = [&](int c) {  // lane 0
    const int n = chunk_n(c);
    const int first = mirror ? W - c * K - n : c * K;  // image column of the chunk's first byte
    uint8_t* dst = my_slots + (c % NB) * L::cslot;
    uint64_t* bar = &my_full[c % NB];
    const uint32_t cb = (uint32_t)(n * Dp);
    fence_proxy_async_shared();
    mbar_expect_tx(bar, 2 * cb + 16u * n);
    bulk_copy(dst, cost_row0 + (int64_t)first * Dp, cb, bar);
    bulk_copy(dst + K * Dp, cost_row1 + (int64_t)first * Dp, cb, bar);
    bulk_copy(dst + 2 * K * Dp, pen_row + c * K, 16u * n, bar);
  };
  int issued = min(NB, nchunks);  // chunks whose copies lane 0 has issued
  if (lane == 0)
    for (int c = 0; c < issued; c++) issue_chunk(c);
  __syncwarp();
  // Set when one of lane 0's chunk waits gave up (an error anywhere in the sweep): the copy into
  // that slot may still be in flight, so lane 0 issues no further copies.
  bool aborted = false;

  const uint32_t lo_edge = lane == 0 ? 0xffffffffu : 0u;
  const uint32_t hi_edge = lane == 31 ? 0xffffffffu : 0u;
  uint32_t pad[REGS];
#pragma unroll
  for (int j = 0; j < REGS; j++) pad[j] = lane * REGS + j >= a.D ? kPadCost : 0u;
  const uint32_t p1x2 = (uint32_t)a.p1 * 0x10001u;
  PathState<REGS> horiz;  // (1,0) in stream coordinates
  zero_state(horiz);
  int carry_ready = 0;

  // The sweep of one row.  CARRY_IN: the row above is the previous block's carry row (waited for
  // chunk by chunk); PUBLISH: this row's vertical states are also stored as this block's carry.
  // The (1,0) path of a pixel depends on this warp's registers alone, so it is computed one step
  // ahead, before the step barrier: a step issues its loads first (the row above for pixel xs,
  // the costs and record of pixel xs + 1), then the paths from the row above for xs and the (1,0)
  // path of xs + 1 side by side, then its stores.
  struct Prepared {
    uint32_t c[REGS];   // the pixel's widened costs
    uint4 pw;           // its penalty record
    PathState<REGS> h;  // its (1,0) path state
  };
  auto sweep_row = [&](auto carry_tag, auto publish_tag) {
    constexpr bool CARRY_IN = decltype(carry_tag)::value;
    constexpr bool PUBLISH = decltype(publish_tag)::value;
    constexpr int NU = NPATH - 1;  // paths from the row above
    auto wait_carry = [&](int need) {
      need = min(need, nchunks - 1);
      while (carry_ready <= need) {
        wait_bar(&carry_full[carry_ready % CS], (carry_ready / CS) & 1, err, limit, 3);
        carry_ready++;
      }
    };
    // The (1,0) path of the next pixel from its loaded cost words and record.
    auto prepare = [&](const CostWords<REGS>& cw, const uint4& pw, Prepared& n) {
      widen_words<REGS>(cw, pad, n.c);
      n.pw = pw;
      const uint32_t q[1] = {horiz.m + (pw.x & 0x7fff7fffu)};
      PathState<REGS> prev[1] = {horiz}, out[1];
      paths_step<REGS, 1>(prev, q, p1x2, n.c, lo_edge, hi_edge, out);
      n.h = out[0];
    };
    // One step: pixel xs (stream column) from its prepared part `cur`, and the next pixel's
    // prepared part from its cost bytes at ncb and record at npb (when xs + 1 < W; otherwise the
    // addresses repeat a landed slot and the result is not used).
    auto step = [&](int xs, const Prepared& cur, uint32_t ncb, uint32_t npb, Prepared& nx) {
      PathState<REGS> prev[NU];
      load_path<REGS>(up_a + (xs & up_mask) * L::vslot, lane_off, L::vmins, 0, prev[0]);
      if constexpr (NU > 1) {
        const uint32_t pd = xs > 0 ? up_a + ((xs - 1) & up_mask) * L::vslot : zero_a;
        load_path<REGS>(pd, lane_off, L::vmins, 1, prev[1]);
      }
      CostWords<REGS> cw;
      load_cost_words<REGS>(ncb, ncb + K * Dp, cw);
      const uint4 npw = lds_v4(npb);
      // Successors of an untextured pixel start afresh (CensusSgm.java:432-433): they see zeros.
      const uint32_t keep = prmt(cur.pw.x, 0, 0xbb99u);
      horiz = cur.h;
      if (keep != 0xffffffffu) {
#pragma unroll
        for (int j = 0; j < REGS; j++) horiz.v[j] &= keep;
        horiz.m &= keep;
      }
      prepare(cw, npw, nx);
      uint32_t q[NU];
      q[0] = prev[0].m + cur.pw.y;
      if constexpr (NU > 1) q[1] = prev[1].m + cur.pw.z;
      PathState<REGS> out[NU];
      paths_step<REGS, NU>(prev, q, p1x2, cur.c, lo_edge, hi_edge, out);
      // Partial aggregate of this stream's paths.
      uint32_t s[REGS];
#pragma unroll
      for (int j = 0; j < REGS; j++) {
        uint32_t acc = cur.h.v[j];
#pragma unroll
        for (int i = 0; i < NU; i++) acc += out[i].v[j];
        s[j] = acc;
      }
      store_words_cs<REGS>(sum_ptr, s);
      sum_ptr += sum_step;
      // The row below gets the states and their minima.
      if (keep != 0xffffffffu) {
#pragma unroll
        for (int i = 0; i < NU; i++) {
#pragma unroll
          for (int j = 0; j < REGS; j++) out[i].v[j] &= keep;
          out[i].m &= keep;
        }
      }
      const uint32_t o = ring_a + (xs & (RING - 1)) * L::vslot;
#pragma unroll
      for (int i = 0; i < NV; i++) {
        sts_words<REGS>(o + lane_off + i * (Dp * 4), out[i].v);
        if constexpr (PUBLISH) store_words<REGS>(carry_ptr + lane_off + i * (Dp * 4), out[i].v);
      }
      if (lane == 0) {
        if constexpr (NV == 2) {
          sts_v2(o + L::vmins, out[0].m, out[1].m);
          if constexpr (PUBLISH) *(uint2*)(carry_ptr + L::vmins) = make_uint2(out[0].m, out[1].m);
        } else {
          asm volatile("st.shared.u32 [%0], %1;" ::"r"(o + L::vmins), "r"(out[0].m));
          if constexpr (PUBLISH) *(uint32_t*)(carry_ptr + L::vmins) = out[0].m;
        }
      }
      if constexpr (PUBLISH) carry_ptr += L::vslot;
    };
    // End of chunk c: refill its slot NB chunks ahead, report carry progress / release.
    auto end_chunk = [&](int c) {
      __syncwarp();
      if (lane == 0) {
        if (c + NB < nchunks && !aborted) {
          issue_chunk(c + NB);
          issued = c + NB + 1;
        }
        if constexpr (PUBLISH) st_release_cta(published, c + 1);
        if constexpr (CARRY_IN) st_release_cta(carry_consumed, c);
        if constexpr (LW > 0)
          if (w == 0) *(volatile int*)row_done = c + 1;
      }
      __syncwarp();
    };
    auto wait_chunk = [&](int c) {
      if (!wait_bar(&my_full[c % NB], (c / NB) & 1, err, limit, 1)) aborted = true;
    };
    // Shared address of this lane's cost bytes of the first pixel of chunk c.
    auto first_cost = [&](int c) {
      return slots_a + (c % NB) * L::cslot + (mirror ? (chunk_n(c) - 1) * Dp : 0) + lane * REGS;
    };
    auto first_pen = [&](int c) { return slots_a + (c % NB) * L::cslot + 2 * K * Dp; };
    Prepared nx;
    {
      wait_chunk(0);
      CostWords<REGS> cw;
      load_cost_words<REGS>(first_cost(0), first_cost(0) + K * Dp, cw);
      prepare(cw, lds_v4(first_pen(0)), nx);
    }
    // Idle steps before this row starts (the 1-pixel lag behind the row above).
    for (int st = 0; st < w; st++) rows_barrier(R * 32);
    const int full_chunks = W / K;
    for (int c = 0; c < full_chunks; c++) {
      if constexpr (CARRY_IN) wait_carry(c);
      const uint32_t slot = slots_a + (c % NB) * L::cslot;
#pragma unroll
      for (int off = 0; off < K; off++) {
        const Prepared cur = nx;
        uint32_t ncb, npb;
        if (off + 1 < K) {
          ncb = slot + cost_first_full + (off + 1) * cost_step;
          npb = slot + 2 * K * Dp + 16 * (off + 1);
        } else if (c + 1 < nchunks) {
          wait_chunk(c + 1);
          ncb = first_cost(c + 1);
          npb = first_pen(c + 1);
        } else {
          ncb = slot + cost_first_full + off * cost_step;
          npb = slot + 2 * K * Dp + 16 * off;
        }
        step(c * K + off, cur, ncb, npb, nx);
        rows_barrier(R * 32);
      }
      end_chunk(c);
    }
    if (full_chunks < nchunks) {
      // Partial last chunk (its first pixel is prepared).
      const int c = full_chunks, n = W - c * K;
      if constexpr (CARRY_IN) wait_carry(c);
      const uint32_t slot = slots_a + (c % NB) * L::cslot;
      const int first = (mirror ? (n - 1) * Dp : 0) + lane * REGS;
      for (int off = 0; off < n; off++) {
        const Prepared cur = nx;
        const int nxt = off + 1 < n ? off + 1 : off;
        step(c * K + off, cur, slot + first + nxt * cost_step, slot + 2 * K * Dp + 16 * nxt, nx);
        rows_barrier(R * 32);
      }
      end_chunk(c);
    }
  };
  if (use_carry)
    sweep_row(std::true_type{}, std::false_type{});
  else if (publish)
    sweep_row(std::false_type{}, std::true_type{});
  else
    sweep_row(std::false_type{}, std::false_type{});

  // Idle steps after this row finished (the rows below are still running).
  for (int step = 0; step < R - 1 - w; step++) rows_barrier(R * 32);
  // Every issued chunk copy lands before the CTA's shared memory is released.  A chunk below
  // issued - NB has landed: lane 0 refilled its slot only after its wait for it succeeded.
  issued = __shfl_sync(0xffffffffu, issued, 0);
  for (int cc = max(0, issued - NB); cc < issued; cc++)
    wait_bar(&my_full[cc % NB], (cc / NB) & 1, err, kDrainLimit, 5, false);
}

template <int REGS>
cudaError_t launch_lines(const LineArgs& a, cudaStream_t stream) {
  const int lines = a.W + a.H - 1;
  const int shared = kLineWarps * kPrefetch * LineSlot<REGS>::bytes;
  cudaError_t e = cudaFuncSetAttribute(lines_kernel<REGS>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, shared);
  if (e != cudaSuccess) return e;
  lines_kernel<REGS><<<(lines + kLineWarps - 1) / kLineWarps, kLineWarps * 32, shared, stream>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Winner-take-all, uniqueness and sub-pixel selection of both views (CensusSgm.java:460-515).
// A warp takes pixels 16 at a time.  Per pixel, lane l adds the partial aggregates (down, up and
// the anti-diagonal lines) of its REGS disparities, both views packed, and the first strict
// minimum and the second minimum outside best-1..best+1 are warp reductions of (total << 8 | k)
// keys; lanes 0/1 note the record of view 0/1.  Then every lane runs the FP64 selection of one
// (pixel, view) record of the group, so the long selection chain runs 32 at a time instead of 2.
// The partials arrive through a per-warp cp.async ring two pixels deep.  A total of at least
// `invalid` (directions x 512) marks a cell whose cost is invalid: every valid total is smaller
// because each valid path cost is at most bits + P2 < 512.
struct WtaArgs {
  const uint32_t* down;  // [H][W][Dp] left | right << 16
  const uint32_t* up;
  const uint32_t* lines;  // anti-diagonal paths (8-path mode), else null
  float* disp[2];
  // Per view, each optional: reason codes and boundary flags of the pixels decided here (others
  // keep their value), selection counters (added to), winners records int32 [n][6].
  uint8_t* reasons[2];
  uint8_t* boundary[2];
  DeviceStats* stats[2];
  int32_t* summary[2];
  int W, H, D, min_disparity, rx, ry, invalid;
  double uniqueness;
};

// Selection of one pixel from its winners record (CensusSgm.java:471-513).
__device__ __forceinline__ void select_pixel_record(int best, int value, int second, int before,
                                                    int after, int flags, int D, int min_disparity,
                                                    double uniqueness, float* out,
                                                    uint8_t* reasons, uint8_t* boundary,
                                                    unsigned (&counts)[6]) {
  float result = __int_as_float(0x7fc00000);
  if (best >= 0) {
    const bool full = flags == 3;
    bool done = false;
    if (full) {
      counts[1]++;
      if (boundary) *boundary = 4;
    }
    if (best == 0 || best == D - 1) {
      counts[2]++;
      if (reasons) *reasons = 2;
      if (full && best == 0) {
        counts[0]++;
        if (boundary) *boundary |= 1;
      }
      if (full && best == D - 1) {
        counts[3]++;
        if (boundary) *boundary |= 2;
      }
      done = true;
    }
    if (!done && second != INT_MAX) {
      const double slack = fmax(1.0, __dmul_rn((double)value, uniqueness));
      if ((double)(second - value) <= slack) {
        counts[4]++;
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
      counts[5]++;
      if (reasons) *reasons = 0;
    }
  }
  *out = result;
}

constexpr int kWtaWarps = 8;

template <int REGS, int PF>
__global__ void __launch_bounds__(kWtaWarps * 32) wta_kernel(const WtaArgs a) {
  constexpr int Dp = 32 * REGS;
  constexpr int kSlot = 3 * Dp * 4;  // one pixel's down, up and lines partials
  constexpr int G = 16;              // pixels per group: 16 pixels x 2 views = one per lane
  extern __shared__ __align__(16) uint8_t wsm[];
  __shared__ __align__(16) uint32_t stage[kWtaWarps][Dp];
  __shared__ int4 rec_a[kWtaWarps][2 * G];  // best, value, second, before of (pixel, view)
  __shared__ int rec_b[kWtaWarps][2 * G];   // after | flags << 16
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t ring = smem_u32(wsm) + warp * PF * kSlot;
  const uint16_t* t16 = (const uint16_t*)stage[warp] + lane;  // view `lane` of k at t16[2k]
  const int W = a.W, H = a.H, D = a.D, invalid = a.invalid;
  const int64_t n = (int64_t)W * H;
  const int64_t stride = (int64_t)gridDim.x * kWtaWarps;
  unsigned counts[6] = {0, 0, 0, 0, 0, 0};
  // The partials of this warp's next PF pixels are in flight (cp.async into a shared-memory ring,
  // one commit group per pixel, empty past the end) while one pixel's minima are found.
  const bool three = a.lines != nullptr;
  auto fetch = [&](int slot, int64_t q) {
    if (q < n) {
      const uint32_t sl = ring + slot * kSlot;
      for (int c = lane; c < Dp / 4; c += 32) {
        cp_async16(sl + c * 16, a.down + q * Dp + c * 4);
        cp_async16(sl + Dp * 4 + c * 16, a.up + q * Dp + c * 4);
        if (three) cp_async16(sl + 2 * Dp * 4 + c * 16, a.lines + q * Dp + c * 4);
      }
    }
    cp_async_commit();
  };
  const int64_t first = (int64_t)blockIdx.x * kWtaWarps + warp;
#pragma unroll
  for (int k = 0; k < PF; k++) fetch(k, first + k * stride);
  int slot = 0;
  // Groups of G of this warp's pixels: the minima of each pixel by warp reductions (whole warp),
  // then the selection of the group's 2G (pixel, view) records, one per lane, side by side.
  for (int64_t base = first; base < n; base += G * stride) {
    for (int i = 0; i < G; i++) {
      const int64_t p = base + i * stride;
      if (p >= n) break;
      const int y = (int)(p / W), x = (int)(p - (int64_t)y * W);
      cp_async_wait<PF - 1>();
      __syncwarp();
      uint32_t tot[REGS], u[REGS], g[REGS] = {};
      const uint32_t sl = ring + slot * kSlot + lane * REGS * 4;
      lds_words<REGS>(sl, tot);
      lds_words<REGS>(sl + Dp * 4, u);
      if (three) lds_words<REGS>(sl + 2 * Dp * 4, g);
#pragma unroll
      for (int j = 0; j < REGS; j++) tot[j] += u[j] + g[j];
      __syncwarp();  // every lane has read the slot before it is refilled
      fetch(slot, p + PF * stride);
      slot = slot + 1 == PF ? 0 : slot + 1;
      int best = -1, value = 0, second = INT_MAX, before = -1, after = -1, flags = 0;
      if (y >= a.ry && y < H - a.ry && x >= a.rx && x < W - a.rx) {
        // Pass 1: first strict minimum, as key = total << 8 | k.
        uint32_t k0 = 0xffffffffu, k1 = 0xffffffffu;
#pragma unroll
        for (int j = 0; j < REGS; j++) {
          const uint32_t k = lane * REGS + j;
          k0 = min(k0, ((tot[j] << 8) & 0xffff00u) | k);
          k1 = min(k1, ((tot[j] >> 8) & 0xffff00u) | k);
        }
        k0 = __reduce_min_sync(0xffffffffu, k0);
        k1 = __reduce_min_sync(0xffffffffu, k1);
        // Pass 2: minimum outside best-1..best+1.
        const int b0 = (int)(k0 & 0xffu), b1 = (int)(k1 & 0xffu);
        uint32_t s0 = 0xffffu, s1 = 0xffffu;
#pragma unroll
        for (int j = 0; j < REGS; j++) {
          const int k = lane * REGS + j;
          if ((unsigned)(k - b0 + 1) > 2u) s0 = min(s0, tot[j] & 0xffffu);
          if ((unsigned)(k - b1 + 1) > 2u) s1 = min(s1, tot[j] >> 16);
        }
        s0 = __reduce_min_sync(0xffffffffu, s0);
        s1 = __reduce_min_sync(0xffffffffu, s1);
        store_words<REGS>(stage[warp] + lane * REGS, tot);
        __syncwarp();
        if (lane < 2) {
          const uint32_t key = lane ? k1 : k0;
          if ((int)(key >> 8) < invalid) {
            best = (int)(key & 0xffu);
            value = (int)(key >> 8);
            const int sec = (int)(lane ? s1 : s0);
            second = sec < invalid ? sec : INT_MAX;
            if (best >= 1 && t16[2 * (best - 1)] < invalid) before = t16[2 * (best - 1)];
            if (best + 1 < D && t16[2 * (best + 1)] < invalid) after = t16[2 * (best + 1)];
            flags = (t16[0] < invalid ? 1 : 0) | (t16[2 * (D - 1)] < invalid ? 2 : 0);
          }
        }
        __syncwarp();
      }
      if (lane < 2) {
        rec_a[warp][2 * i + lane] = make_int4(best, value, second, before);
        rec_b[warp][2 * i + lane] = (after & 0xffff) | flags << 16;
      }
    }
    __syncwarp();
    {
      const int i = lane >> 1, view = lane & 1;
      const int64_t p = base + i * stride;
      if (p < n) {
        const int4 r = rec_a[warp][lane];
        const int rb = rec_b[warp][lane];
        const int after = (int)(int16_t)(rb & 0xffff), flags = rb >> 16;
        uint8_t* reasons = view ? a.reasons[1] : a.reasons[0];
        uint8_t* boundary = view ? a.boundary[1] : a.boundary[0];
        select_pixel_record(r.x, r.y, r.z, r.w, after, flags, D, a.min_disparity, a.uniqueness,
                            (view ? a.disp[1] : a.disp[0]) + p, reasons ? reasons + p : nullptr,
                            boundary ? boundary + p : nullptr, counts);
        int32_t* summary = view ? a.summary[1] : a.summary[0];
        if (summary) {
          // The record of GpuStereo.java:758-769: no winner -> value INT_MAX.
          int2* rec = (int2*)(summary + 6 * p);
          rec[0] = make_int2(r.x, r.x >= 0 ? r.y : INT_MAX);
          rec[1] = make_int2(r.z, r.w);
          rec[2] = make_int2(after, flags);
        }
      }
    }
    __syncwarp();
  }
  cp_async_wait<0>();
  // Lane l selected view l & 1 throughout: the counters of each view are the sums over its lanes.
#pragma unroll
  for (int view = 0; view < 2; view++) {
    DeviceStats* st = a.stats[view];
    if (!st) continue;
    unsigned long long* dst[6] = {&st->lower_boundary_rejected, &st->full_interval_pixels,
                                  &st->boundary_rejected, &st->upper_boundary_rejected,
                                  &st->ambiguity_rejected, &st->selected};
#pragma unroll
    for (int i = 0; i < 6; i++) {
      const unsigned total = __reduce_add_sync(0xffffffffu, (lane & 1) == view ? counts[i] : 0u);
      if (lane == 0 && total) atomicAdd(dst[i], (unsigned long long)total);
    }
  }
}

template <int REGS, int PF>
cudaError_t launch_wta_t(const WtaArgs& a, int sm_count, cudaStream_t stream) {
  auto kernel = wta_kernel<REGS, PF>;
  const int shared = kWtaWarps * PF * 3 * 32 * REGS * 4;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, shared);
  if (e != cudaSuccess) return e;
  const int64_t n = (int64_t)a.W * a.H;
  const int grid = (int)std::min<int64_t>((n + kWtaWarps - 1) / kWtaWarps, (int64_t)sm_count * 8);
  kernel<<<grid, kWtaWarps * 32, shared, stream>>>(a);
  return cudaGetLastError();
}

// Two pixels in flight per warp: more (4) measured the same, and its ring costs a CTA per SM.
template <int REGS>
cudaError_t launch_wta(const WtaArgs& a, int sm_count, cudaStream_t stream) {
  return launch_wta_t<REGS, 2>(a, sm_count, stream);
}

template <int REGS, int NPATH, int K, int R, int LW>
cudaError_t launch_sweep(const SweepArgs& a, cudaStream_t stream, bool exclusive) {
  auto kernel = sweep_kernel<REGS, NPATH, K, R, LW>;
  using L = SweepLayout<REGS, NPATH, K, R>;
  // Exclusive: at least 116 KB so that one CTA holds an SM alone (two row blocks on one SM halve
  // each other's step rate, while a later block never needs an SM before an earlier one
  // finishes).  Batched pairs instead share SMs, filling each other's idle issue slots.
  const int need = LW > 0 ? L::with_lines(LW) : L::total;
  const int shared = exclusive ? std::max(need, 116 * 1024) : need;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, shared);
  if (e != cudaSuccess) return e;
  kernel<<<2 * a.nb, (R + 2 + LW) * 32, shared, stream>>>(a);
  return cudaGetLastError();
}

// Rows per sweep CTA: few enough that the rows of a block (all busy at once) spread over SMs,
// many enough that the carry hand-off between blocks stays rare, and that few row blocks wait for
// an SM (one CTA per SM: at D = 128, 1067 rows, 12 rows per CTA measured 2.84 ms per sweep
// against 2.93 with 8 and 3.04 with 16).
constexpr int kChunk = 2;  // pixels per cost chunk and per carry publication
// 193..256 disparities: 8 rows (3000x2000 D256, 16 paths: 46-48 ms per pair against 50 with 4).
constexpr int rows_default(int regs) { return regs == 4 ? 12 : 8; }

// Rows per sweep CTA: the default, or CSGM_SWEEP_ROWS (4, 8, or 12 at D <= 128) for tuning runs.
int rows_for(int regs) {
  static const int forced = [] {
    const char* e = getenv("CSGM_SWEEP_ROWS");
    const int v = e ? atoi(e) : 0;
    return v == 4 || v == 8 || v == 12 ? v : 0;
  }();
  if (forced == 12 && regs != 4) return rows_default(regs);
  return forced ? forced : rows_default(regs);
}

// Line warps per sweep CTA in 8-path mode: the anti-diagonal lines run inside the sweep's CTAs on
// the issue slots the row warps leave idle, when the line rings fit beside the sweep's shared
// memory (227 KB per CTA); 0 runs them as a separate kernel before the sweep.
// CSGM_SWEEP_LINE_WARPS (0, 4 or 8) overrides the default for tuning runs.
constexpr int kSweepLineWarps = 8;
constexpr int kMaxSharedPerBlock = 227 * 1024;

template <int REGS, int R>
int sweep_smem_with_lines(int lw) { return SweepLayout<REGS, 3, kChunk, R>::with_lines(lw); }

// `requested` (0, 4 or 8; -1 = none) takes precedence over the environment and the default.
int line_warps_for(int regs, int rows, int requested) {
  static const int forced = [] {
    const char* e = getenv("CSGM_SWEEP_LINE_WARPS");
    const int v = e ? atoi(e) : -1;
    return v == 0 || v == 4 || v == 8 ? v : -1;
  }();
  int lw = requested >= 0 ? requested : forced >= 0 ? forced : kSweepLineWarps;
  auto smem = [&](int l) {
    switch (regs * 16 + rows) {
      case 2 * 16 + 4: return sweep_smem_with_lines<2, 4>(l);
      case 2 * 16 + 8: return sweep_smem_with_lines<2, 8>(l);
      case 4 * 16 + 4: return sweep_smem_with_lines<4, 4>(l);
      case 4 * 16 + 8: return sweep_smem_with_lines<4, 8>(l);
      case 4 * 16 + 12: return sweep_smem_with_lines<4, 12>(l);
      case 6 * 16 + 4: return sweep_smem_with_lines<6, 4>(l);
      case 6 * 16 + 8: return sweep_smem_with_lines<6, 8>(l);
      case 8 * 16 + 4: return sweep_smem_with_lines<8, 4>(l);
      default: return sweep_smem_with_lines<8, 8>(l);
    }
  };
  while (lw > 0 && smem(lw) > kMaxSharedPerBlock) lw -= 4;
  return lw;
}

// How much of a block's remaining row pixels a line may take (percent): a line warp's pixel costs
// well under half a sweep step, so 100 leaves slack.  CSGM_SWEEP_LINE_SLACK overrides it for
// tuning runs.
int line_slack() {
  static const int v = [] {
    const char* e = getenv("CSGM_SWEEP_LINE_SLACK");
    const int x = e ? atoi(e) : 0;
    return x >= 10 && x <= 1000 ? x : 100;
  }();
  return v;
}

template <int REGS, int NPATH>
cudaError_t launch_sweep_for(const SweepArgs& a, cudaStream_t stream, bool exclusive, int rows,
                             int lw) {
  if constexpr (REGS == 4) {
    if (rows == 12) {
      if constexpr (NPATH == 3) {
        if (lw == 8) return launch_sweep<REGS, 3, kChunk, 12, 8>(a, stream, exclusive);
        if (lw == 4) return launch_sweep<REGS, 3, kChunk, 12, 4>(a, stream, exclusive);
      }
      return launch_sweep<REGS, NPATH, kChunk, 12, 0>(a, stream, exclusive);
    }
  }
  if constexpr (NPATH == 3) {
    if (lw == 8)
      return rows == 8 ? launch_sweep<REGS, 3, kChunk, 8, 8>(a, stream, exclusive)
                       : launch_sweep<REGS, 3, kChunk, 4, 8>(a, stream, exclusive);
    if (lw == 4)
      return rows == 8 ? launch_sweep<REGS, 3, kChunk, 8, 4>(a, stream, exclusive)
                       : launch_sweep<REGS, 3, kChunk, 4, 4>(a, stream, exclusive);
  }
  return rows == 8 ? launch_sweep<REGS, NPATH, kChunk, 8, 0>(a, stream, exclusive)
                   : launch_sweep<REGS, NPATH, kChunk, 4, 0>(a, stream, exclusive);
}

struct FusedLayout {
  size_t cost, sum, pen, info, carry, flags, total;
  int Dp, nb, vslot, rows;
  FusedLayout(const csgm_params& p, int w, int h, int rows_per_block) {
    Dp = padded_d(p.disparities);
    rows = rows_per_block;
    nb = (h + rows - 1) / rows;
    const int nv = p.directions >= 8 ? 2 : 1;
    vslot = nv * Dp * 4 + 16;  // the states and their minima (16 bytes)
    size_t n = (size_t)w * h;
    cost = n * Dp;
    sum = n * Dp * 4;
    pen = 2 * n * 16;
    info = p.directions == 16 ? n * 4 : 0;
    carry = (size_t)2 * nb * w * vslot;
    flags = ((size_t)2 * nb + 8) * sizeof(int);
    total = 2 * cost + (p.directions >= 8 ? 3 : 2) * sum + pen + info + carry + flags + 8 * 256;
  }
};

}  // namespace

bool fused_supported(const csgm_params& p) {
  if (p.disparities > 256) return false;
  if (p.directions != 4 && p.directions != 8 && p.directions != 16) return false;
  // Valid path costs stay below 512 (cost <= bits, penalty <= P2), which is what lets the
  // selection tell invalid cells by their totals.
  const int bits = p.window_x * p.window_y - 1;
  if (bits > 127 || p.p2 + bits >= 512) return false;
  // The partial aggregates are packed uint16 pairs.  They hold every sum exactly when the proved
  // bound directions x (512 + P2) fits 16 bits (StereoCost.aggregateBound, StereoCost.java:31-41),
  // which P2 + bits < 512 guarantees for up to 16 paths; a uint32 aggregate then holds the same
  // values, so aggregate_bytes 4 gives bit-identical results on these kernels.
  if ((int64_t)p.directions * (512 + p.p2) > 65535) return false;
  return true;
}

SweepTuning resolve_tuning(const csgm_params& p, const SweepTuning& want) {
  const int regs = padded_d(p.disparities) / 32;
  SweepTuning t;
  const int r = want.rows;
  t.rows = r == 4 || r == 8 || (r == 12 && regs == 4) ? r : rows_for(regs);
  const int lw = want.line_warps == 0 || want.line_warps == 4 || want.line_warps == 8
                     ? want.line_warps
                     : -1;
  t.line_warps = p.directions >= 8 ? line_warps_for(regs, t.rows, lw) : 0;
  t.line_slack = want.line_slack >= 10 && want.line_slack <= 1000 ? want.line_slack : line_slack();
  return t;
}

size_t fused_workspace_bytes(const csgm_params& p, int w, int h, const SweepTuning& tuning) {
  return FusedLayout(p, w, h, resolve_tuning(p, tuning).rows).total;
}

int run_views_fused(Context& ctx, const csgm_params& p, const FusedViews& v, int w, int h,
                    int** error_flag) {
  int status = CSGM_OK;
  if (h > 65535) return fail(CSGM_E_UNSUPPORTED, "fused path: image taller than 65535 rows");
  const SweepTuning T = resolve_tuning(p, ctx.tuning);
  FusedLayout F(p, w, h, T.rows);
  uint8_t* cost_l = (uint8_t*)ctx.ws->get(kCostL, F.cost, &status);
  if (!cost_l) return status;
  uint8_t* cost_r = (uint8_t*)ctx.ws->get(kCostR, F.cost, &status);
  if (!cost_r) return status;
  uint32_t* sum_down = (uint32_t*)ctx.ws->get(kSum, F.sum, &status);
  if (!sum_down) return status;
  uint32_t* sum_up = (uint32_t*)ctx.ws->get(kSumUp, F.sum, &status);
  if (!sum_up) return status;
  uint32_t* sum_lines = nullptr;
  if (p.directions >= 8) {
    sum_lines = (uint32_t*)ctx.ws->get(kSumLines, F.sum, &status);
    if (!sum_lines) return status;
  }
  uint32_t* info = nullptr;
  if (p.directions == 16) {
    info = (uint32_t*)ctx.ws->get(kPixelInfo, F.info, &status);
    if (!info) return status;
  }
  uint4* pen = (uint4*)ctx.ws->get(kPen, F.pen, &status);
  if (!pen) return status;
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
      const int cap = p.cost_mode == CSGM_COST_AD_CENSUS ? p.ad_truncation : p.gradient_truncation;
      ca.recip = p.cost_mode == CSGM_COST_CENSUS ? 0 : reciprocal64(1000ull * (unsigned)cap);
      le = launch_cost_rows(ca, ctx.sm_count, ctx.stream);
    }
    if (le != cudaSuccess) return cuda_fail(le, "cost kernel launch");
    ctx.prof->kernel_end("cost_pair");
  }
  {
    PenaltyArgs pa{{v.gray_l, v.gray_r}, {v.tex_l, v.tex_r}, pen, info, w, h, p.p1, p.p2,
                   p.edge_scale};
    ctx.prof->kernel_begin();
    penalty_kernel<<<dim3((w + 1023) / 1024, h, 2), 128, 0, ctx.stream>>>(pa);
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) return cuda_fail(le, "penalty kernel launch");
    ctx.prof->kernel_end("penalty");
  }
  const int regs = F.Dp / 32;
  // The anti-diagonal lines: inside the sweep's CTAs (line warps), or as their own kernel on the
  // pair's stream before the sweep (beside the sweep on a second stream they slowed it by more
  // than their own run time: 4.63 ms per pair against 4.47 ms one after the other).
  const int line_warps = sum_lines && ctx.lines_in_sweep ? T.line_warps : 0;
  LineArgs la{{cost_l, cost_r}, pen, sum_lines, w, h, p.disparities, p.p1,
              line_warps ? flags + 2 * F.nb + 2 : nullptr};
  auto run_lines = [&](cudaStream_t stream) {
    switch (regs) {
      case 2: return launch_lines<2>(la, stream);
      case 4: return launch_lines<4>(la, stream);
      case 6: return launch_lines<6>(la, stream);
      default: return launch_lines<8>(la, stream);
    }
  };
  // 16 paths: the knight-move line families add to the lines partial once the anti-diagonal
  // lines have written it.
  KnightArgs ka{{cost_l, cost_r}, info, sum_lines, w, h, p.disparities, p.p1, p.p2, p.edge_scale,
                0, 0};
  auto run_knights = [&](cudaStream_t stream) -> int {
    if (!info) return CSGM_OK;
    ctx.prof->kernel_begin();
    cudaError_t ke;
    switch (regs) {
      case 2: ke = launch_knights<2>(ka, stream); break;
      case 4: ke = launch_knights<4>(ka, stream); break;
      case 6: ke = launch_knights<6>(ka, stream); break;
      default: ke = launch_knights<8>(ka, stream); break;
    }
    if (ke != cudaSuccess) return cuda_fail(ke, "knight line kernel launch");
    ctx.prof->kernel_end("knights");
    return CSGM_OK;
  };
  if (sum_lines && !line_warps) {
    cudaError_t le;
    ctx.prof->kernel_begin();
    le = run_lines(ctx.stream);
    if (le != cudaSuccess) return cuda_fail(le, "line kernel launch");
    ctx.prof->kernel_end("lines");
    status = run_knights(ctx.stream);
    if (status) return status;
  }
  cudaError_t e = cudaMemsetAsync(flags, 0, F.flags, ctx.stream);
  if (e != cudaSuccess) return cuda_fail(e, "flag clear");

  SweepArgs a{};
  a.cost[0] = cost_l;
  a.cost[1] = cost_r;
  a.pen = pen;
  a.sum[0] = sum_down;
  a.sum[1] = sum_up;
  a.carry = carry;
  a.progress = flags;
  a.ticket = flags + 2 * F.nb;
  a.error = a.ticket + 1;
  *error_flag = a.error;
  a.W = w;
  a.H = h;
  a.D = p.disparities;
  a.nb = F.nb;
  a.p1 = p.p1;
  a.timeout = ctx.wait_limit > 0 ? ctx.wait_limit : kDefaultWaitLimit;
  a.line = la;
  a.line_slack = T.line_slack;
  const bool eight = p.directions >= 8;  // 16 paths: the 8-path sweep plus the knight lines
  // Batched pairs launch the sweep on a high-priority stream: its pending CTAs then take SMs ahead
  // of other pairs' bandwidth-bound kernels, so a pair's chain of row blocks is not held up.
  cudaStream_t sweep_stream = ctx.stream;
  if (ctx.sweep_stream) {
    e = cudaEventRecord(ctx.sweep_ready, ctx.stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx.sweep_stream, ctx.sweep_ready, 0);
    if (e != cudaSuccess) return cuda_fail(e, "sweep stream ordering");
    sweep_stream = ctx.sweep_stream;
  }
  ctx.prof->kernel_begin();
  switch (regs * 2 + (eight ? 1 : 0)) {
    case 2 * 2: e = launch_sweep_for<2, 2>(a, sweep_stream, ctx.exclusive_sweep, F.rows, 0); break;
    case 2 * 2 + 1: e = launch_sweep_for<2, 3>(a, sweep_stream, ctx.exclusive_sweep, F.rows, line_warps); break;
    case 4 * 2: e = launch_sweep_for<4, 2>(a, sweep_stream, ctx.exclusive_sweep, F.rows, 0); break;
    case 4 * 2 + 1: e = launch_sweep_for<4, 3>(a, sweep_stream, ctx.exclusive_sweep, F.rows, line_warps); break;
    case 6 * 2: e = launch_sweep_for<6, 2>(a, sweep_stream, ctx.exclusive_sweep, F.rows, 0); break;
    case 6 * 2 + 1: e = launch_sweep_for<6, 3>(a, sweep_stream, ctx.exclusive_sweep, F.rows, line_warps); break;
    case 8 * 2: e = launch_sweep_for<8, 2>(a, sweep_stream, ctx.exclusive_sweep, F.rows, 0); break;
    case 8 * 2 + 1: e = launch_sweep_for<8, 3>(a, sweep_stream, ctx.exclusive_sweep, F.rows, line_warps); break;
    default: return fail(CSGM_E_UNSUPPORTED, "fused path: unsupported D");
  }
  if (e != cudaSuccess) return cuda_fail(e, "sweep kernel launch");
  ctx.prof->kernel_end("sweep");
  if (line_warps) {
    // The lines the sweep's line warps did not take (a queue that is already empty costs one
    // short launch).
    ctx.prof->kernel_begin();
    e = run_lines(sweep_stream);
    if (e != cudaSuccess) return cuda_fail(e, "line kernel launch");
    ctx.prof->kernel_end("lines_rest");
    status = run_knights(sweep_stream);
    if (status) return status;
  }
  if (ctx.sweep_stream) {
    e = cudaEventRecord(ctx.sweep_done, ctx.sweep_stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx.stream, ctx.sweep_done, 0);
    if (e != cudaSuccess) return cuda_fail(e, "sweep stream ordering");
  }

  WtaArgs t{};
  t.down = sum_down;
  t.up = sum_up;
  t.lines = sum_lines;
  t.disp[0] = v.disp_l;
  t.disp[1] = v.disp_r;
  for (int view = 0; view < 2; view++) {
    t.reasons[view] = v.reasons[view];
    t.boundary[view] = v.boundary[view];
    t.stats[view] = v.stats[view];
    t.summary[view] = v.summary[view];
  }
  t.W = w;
  t.H = h;
  t.D = p.disparities;
  t.min_disparity = p.min_disparity;
  t.rx = p.window_x / 2;
  t.ry = p.window_y / 2;
  t.invalid = 512 * p.directions;
  t.uniqueness = p.uniqueness;
  ctx.prof->kernel_begin();
  switch (regs) {
    case 2: e = launch_wta<2>(t, ctx.sm_count, ctx.stream); break;
    case 4: e = launch_wta<4>(t, ctx.sm_count, ctx.stream); break;
    case 6: e = launch_wta<6>(t, ctx.sm_count, ctx.stream); break;
    case 8: e = launch_wta<8>(t, ctx.sm_count, ctx.stream); break;
    default: return fail(CSGM_E_UNSUPPORTED, "fused path: unsupported D");
  }
  if (e != cudaSuccess) return cuda_fail(e, "wta kernel launch");
  ctx.prof->kernel_end("wta");
  return CSGM_OK;
}

}  // namespace csgm
