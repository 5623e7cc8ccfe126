// Dense stereo hot path for B200 (sm_100a): census -> graded cost -> four-pass
// recursive edge-aware filter -> per-pixel top-2 -> MASDA row solve.
//
// Arithmetic is the reference's, bit for bit (mayio/doubleeye
// core/tools/de_dense.cpp, core/include/doubleeye/dense_solve.hpp); the work
// decomposition is this file's own:
//
//   k_census_rows / k_census_generic
//             shared-memory tiles with a halo, both images at once; a thread owns
//             four vertically adjacent pixels, whose windows share rows (7x7 and
//             9x7), or one pixel (other windows).  Writes a 64-bit census word that
//             also carries the pixel byte (bits 52..59) when the window fits in 48
//             bits, so the cost kernel gets Hamming and absolute-difference inputs
//             in one load, plus the two Q15 coefficient planes of the left image.
//   k_rows    one CTA per image row, a thread per PAIR of adjacent disparities
//             (int16x2 in one 32-bit register): graded score fused with the
//             horizontal forward pass, then the backward pass, both sequential in
//             x as integer rounding demands; the row's census words live in
//             shared memory, the forward result comes back through a ring of bulk
//             copies.
//   k_cols    a column is a group of lanes, each lane KT disparities: vertical
//             forward pass written in place, vertical backward pass fused with the
//             top-2 (packed keys, merged over the group by recursive halving) and
//             the winner's neighbour costs; rows stream through per-lane rings (in
//             shared memory filled by cp.async at 8 disparities per lane, else in
//             registers), with no block-wide step.
//   k_solve   one CTA per row: candidate buckets by right pixel, damped max-sum
//             iterations, belief, and the one-to-one claim done in parallel as a
//             per-right-pixel arg-max (each pixel claims exactly one right pixel,
//             so "first in belief order wins" is that arg-max), sub-pixel fit,
//             reverse-match residuals, confidence.
//
// All kernels take the batch descriptor table by value, so one set of launches
// covers any mix of pair shapes and needs no host-to-device copies (CUDA-graph
// capturable).  Compiled with --fmad=false: the solve's float arithmetic must not
// be contracted, to match the reference's x86-64 single-precision results.

#include <algorithm>
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

#include "de_internal.h"

namespace de {
namespace {

constexpr float kNegBig = -1e30f;

__device__ __forceinline__ int find_pair(const int* prefix, int n, int item) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= item) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// One recursive-filter step (core/tools/de_dense.cpp:419): int32 carry, +2^14
// rounding, arithmetic shift.
__device__ __forceinline__ int32_t rf_step(int32_t c, int32_t f, int32_t a) {
  return c + ((a * (f - c) + (1 << 14)) >> 15);
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }

__device__ __forceinline__ uint32_t pack2(int32_t lo, int32_t hi) {
  return (uint32_t(uint16_t(lo))) | (uint32_t(hi) << 16);
}
__device__ __forceinline__ int32_t lo16(uint32_t v) { return int32_t(int16_t(v & 0xFFFFu)); }
__device__ __forceinline__ int32_t hi16(uint32_t v) { return int32_t(int16_t(v >> 16)); }

// ---------------------------------------------------------------------------------
// Census words + coefficient planes.
// core/tools/de_dense.cpp:94-129,186-227 (census), :531-561 (rf_coeffs).
constexpr int kCTX = 32, kCTY = 8, kMaxHalf = 4;

// Packed census words (windows of <= 48 bits): lo32 = bits 0..31; hi32 = bits
// 32..47 | guard bit 19 (left words only) | pixel byte at bits 20..27.  Then
// (left.hi - right.hi) >> 20 is exactly L - R: the guard keeps the census bits from
// borrowing into the pixel field.  (left ^ right) masked to the census bits gives the
// Hamming input as before.
constexpr uint32_t kCensusHiMask = 0xFFFFu;
constexpr uint32_t kGuard = 1u << 19;
constexpr int kPixShift = 20;

__device__ __forceinline__ void census_generic(const uint8_t (*sL)[kCTX + 2 * kMaxHalf],
                                               const uint8_t (*sR)[kCTX + 2 * kMaxHalf],
                                               int cx, int cy, int hw, int hh, uint64_t& wl,
                                               uint64_t& wr) {
  const uint8_t cl = sL[cy][cx], cr = sR[cy][cx];
  wl = wr = 0;
  int bit = 0;
  for (int dy = -hh; dy <= hh; ++dy)
    for (int dx = -hw; dx <= hw; ++dx) {
      if (dx == 0 && dy == 0) continue;
      wl |= uint64_t(sL[cy + dy][cx + dx] < cl) << bit;
      wr |= uint64_t(sR[cy + dy][cx + dx] < cr) << bit;
      ++bit;
    }
}

// Any window up to 9x9 (runtime half-widths), one pixel a thread.
__global__ void __launch_bounds__(kCTX * kCTY) k_census_generic(DevCfg cfg, Batch b) {
  __shared__ uint8_t sL[kCTY + 2 * kMaxHalf][kCTX + 2 * kMaxHalf];
  __shared__ uint8_t sR[kCTY + 2 * kMaxHalf][kCTX + 2 * kMaxHalf];
  __shared__ uint16_t srf[256];
  const int item = blockIdx.x;
  const int pi = find_pair(b.pix_prefix, b.n, item);
  const DevPair& P = b.p[pi];
  const int W = P.W, H = P.H;
  const int t = item - b.pix_prefix[pi];
  const int tilesX = (W + kCTX - 1) / kCTX;
  const int x0 = (t % tilesX) * kCTX, y0 = (t / tilesX) * kCTY;
  const int tid = threadIdx.y * kCTX + threadIdx.x;
  for (int i = tid; i < 256; i += kCTX * kCTY) srf[i] = cfg.rf[i];
  constexpr int TW = kCTX + 2 * kMaxHalf, TH = kCTY + 2 * kMaxHalf;
  for (int i = tid; i < TW * TH; i += kCTX * kCTY) {
    const int ty = i / TW, tx = i % TW;
    const int gx = x0 + tx - kMaxHalf, gy = y0 + ty - kMaxHalf;
    const bool in = gx >= 0 && gx < W && gy >= 0 && gy < H;
    const size_t gi = size_t(gy) * W + gx;
    sL[ty][tx] = in ? P.L[gi] : 0;
    sR[ty][tx] = in ? P.R[gi] : 0;
  }
  __syncthreads();
  const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
  if (x >= W || y >= H) return;
  const int hw = cfg.hw, hh = cfg.hh;
  const int cx = threadIdx.x + kMaxHalf, cy = threadIdx.y + kMaxHalf;
  uint64_t wl = 0, wr = 0;
  if (x >= hw && x < W - hw && y >= hh && y < H - hh)
    census_generic(sL, sR, cx, cy, hw, hh, wl, wr);
  if (cfg.packed) {
    wl |= (uint64_t(kGuard) | (uint64_t(sL[cy][cx]) << kPixShift)) << 32;
    wr |= (uint64_t(sR[cy][cx]) << kPixShift) << 32;
  }
  P.cwL[size_t(y) * P.cpitch + P.lpad + x] = wl;
  P.cwR[size_t(y) * P.cpitch + x] = wr;
  const int c = sL[cy][cx];
  P.ax[size_t(y) * P.apitch + P.lpad + x] = x > 0 ? srf[abs(c - int(sL[cy][cx - 1]))] : srf[0];
  P.ay[size_t(y) * W + x] = y > 0 ? srf[abs(c - int(sL[cy - 1][cx]))] : srf[0];
}

// k_census_rows<HW>: the (2 HW + 1) x 7 census (7x7, the default, and 9x7), NR
// vertically adjacent pixels per thread.  Their windows share most of their rows, so
// each byte read from the shared tile serves up to NR pixels' compares: (6 + NR) rows
// of loads per NR pixels per image instead of 7 rows each.  Tiles are 32 x (8 NR)
// pixels; the bit order, border zeros, packed layout and coefficient planes are those
// of k_census_generic.
constexpr int kCensusNR = 4;                        // pixels per thread (rows)
constexpr int kC2Y = kCensusNR * kCTY;              // tile rows

template <int HW>
__host__ __device__ constexpr int census_bit(int dy, int dx) {   // row-major, no centre
  return (dy + 3) * (2 * HW + 1) + (dx + HW) - ((dy > 0 || (dy == 0 && dx > 0)) ? 1 : 0);
}

template <int HW>
__global__ void __launch_bounds__(kCTX * kCTY) k_census_rows(DevCfg cfg, Batch b) {
  static_assert(HW >= 1 && HW <= kMaxHalf, "half-width");
  constexpr int NR = kCensusNR;
  __shared__ uint8_t sL[kC2Y + 2 * kMaxHalf][kCTX + 2 * kMaxHalf];
  __shared__ uint8_t sR[kC2Y + 2 * kMaxHalf][kCTX + 2 * kMaxHalf];
  __shared__ uint16_t srf[256];
  const int item = blockIdx.x;
  const int pi = find_pair(b.pix_prefix, b.n, item);
  const DevPair& P = b.p[pi];
  const int W = P.W, H = P.H;
  const int t = item - b.pix_prefix[pi];
  const int tilesX = (W + kCTX - 1) / kCTX;
  const int x0 = (t % tilesX) * kCTX, y0 = (t / tilesX) * kC2Y;
  const int tid = threadIdx.y * kCTX + threadIdx.x;
  for (int i = tid; i < 256; i += kCTX * kCTY) srf[i] = cfg.rf[i];
  constexpr int TW = kCTX + 2 * kMaxHalf, TH = kC2Y + 2 * kMaxHalf;
  for (int i = tid; i < TW * TH; i += kCTX * kCTY) {
    const int ty = i / TW, tx = i % TW;
    const int gx = x0 + tx - kMaxHalf, gy = y0 + ty - kMaxHalf;
    const bool in = gx >= 0 && gx < W && gy >= 0 && gy < H;
    const size_t gi = size_t(gy) * W + gx;
    sL[ty][tx] = in ? P.L[gi] : 0;
    sR[ty][tx] = in ? P.R[gi] : 0;
  }
  __syncthreads();
  const int x = x0 + threadIdx.x, y0t = y0 + NR * threadIdx.y;
  if (x >= W || y0t >= H) return;
  const int cx = threadIdx.x + kMaxHalf, cy = NR * threadIdx.y + kMaxHalf;   // first pixel
  uint32_t cl[NR], cr[NR], l0[NR], l1[NR], r0[NR], r1[NR];
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    cl[i] = sL[cy + i][cx];
    cr[i] = sR[cy + i][cx];
    l0[i] = l1[i] = r0[i] = r1[i] = 0;
  }
#pragma unroll
  for (int w = 0; w < 6 + NR; ++w)                   // tile row cy - 3 + w
#pragma unroll
    for (int dx = -HW; dx <= HW; ++dx) {
      const uint32_t vl = sL[cy - 3 + w][cx + dx], vr = sR[cy - 3 + w][cx + dx];
#pragma unroll
      for (int i = 0; i < NR; ++i) {                 // pixel i sees this row at dy = w - 3 - i
        const int dy = w - 3 - i;
        if (dy < -3 || dy > 3 || (dy == 0 && dx == 0)) continue;
        const int bit = census_bit<HW>(dy, dx);
        const uint32_t fl = vl < cl[i], fr = vr < cr[i];
        if (bit < 32) { l0[i] |= fl << bit; r0[i] |= fr << bit; }
        else { l1[i] |= fl << (bit - 32); r1[i] |= fr << (bit - 32); }
      }
    }
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    const int y = y0t + i, cyy = cy + i;
    if (y >= H) break;
    uint64_t wl = 0, wr = 0;
    if (x >= HW && x < W - HW && y >= 3 && y < H - 3) {
      wl = (uint64_t(l1[i]) << 32) | l0[i];
      wr = (uint64_t(r1[i]) << 32) | r0[i];
    }
    if (cfg.packed) {
      wl |= (uint64_t(kGuard) | (uint64_t(cl[i]) << kPixShift)) << 32;
      wr |= (uint64_t(cr[i]) << kPixShift) << 32;
    }
    P.cwL[size_t(y) * P.cpitch + P.lpad + x] = wl;
    P.cwR[size_t(y) * P.cpitch + x] = wr;
    const int c = int(cl[i]);
    P.ax[size_t(y) * P.apitch + P.lpad + x] = x > 0 ? srf[abs(c - int(sL[cyy][cx - 1]))] : srf[0];
    P.ay[size_t(y) * W + x] = y > 0 ? srf[abs(c - int(sL[cyy - 1][cx]))] : srf[0];
  }
}

// ---------------------------------------------------------------------------------
// k_rows: graded score + horizontal forward + horizontal backward, one row.
// Score: core/tools/de_dense.cpp:1224-1233.  Horizontal passes: :411-430.
//
// Thread t owns disparities k0 = 2t and k1 = 2t+1 of the row.  The right census
// word chain k1 needs at x is the one chain k0 used at x-1, so each step loads one
// right word.  Lanes before their own valid start (x < hw + d) carry exact zeros,
// which is what the reference's zero-filled plane gives there, so a warp can start
// at its first lane's start.  Values left of a plane's valid window never reach a
// valid output (the vertical passes stay within a column and the top-2 masks
// k > x - hw - dmin), so they are not computed exactly and not needed.
// Score table: (h, m) -> Q14 score, h = Hamming distance, m = |L - R| clamped to
// TS-1 (exact: the AD score saturates at ad_trunc < TS).  Stored m-major with 64
// h-entries per row, so the many lookups that share the saturated m read adjacent
// entries, not one bank.
template <int TS, int CP>
struct ScoreTable {
  __host__ __device__ static constexpr size_t bytes() { return size_t(TS) * 64 * 2; }
};

template <bool PACKED, int TS, int CP>
__device__ __forceinline__ int32_t graded(uint64_t lw, uint64_t rw, const void* tab,
                                          const uint8_t* sLp, const uint8_t* sRp, int xl,
                                          int xr) {
  int h, ad;
  if (PACKED) {
    const uint32_t lh = uint32_t(lw >> 32), rh = uint32_t(rw >> 32);
    h = __popc(uint32_t(lw) ^ uint32_t(rw)) + __popc((lh ^ rh) & kCensusHiMask);
    ad = abs((int32_t(lh) - int32_t(rh)) >> kPixShift);
  } else {
    h = __popcll(lw ^ rw);
    ad = abs(int(sLp[xl]) - int(sRp[xr]));
  }
  if (TS == 16) ad = min(ad, 15);
  return static_cast<const int16_t*>(tab)[ad * 64 + h];
}

// Bulk asynchronous copies (cp.async.bulk, the TMA engine's 1-D form) with
// mbarrier completion.  Every wait is bounded: if a phase never completes the
// kernel records it in the batch status word and runs on to its end.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return uint32_t(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
constexpr int kWaitLimit = 1 << 22;                  // try_wait rounds before giving up
__device__ __forceinline__ void mbar_wait(uint64_t* bar, uint32_t parity, int* err,
                                          int limit = kWaitLimit) {
  for (int i = 0; i < limit; ++i)
    if (mbar_test(bar, parity)) return;
  if (err) atomicExch(err, 1);
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async;" ::: "memory");
}

// One row per CTA iteration (the grid is persistent over rows); all pairs of a
// launch share Dpad = 64 G, so strides and chunk sizes are compile-time.  The row's
// census words arrive by bulk copy into a single buffer that is refilled for the
// next row while this row's backward pass runs (only the forward pass reads them);
// the x-coefficients, read by both passes, are double-buffered.  Forward results go
// to the volume with plain stores; the backward pass brings them back through a
// ring of bulk copies, so no thread waits on a global load.
// Backward ring: stages of kRowsChunk disparity-columns (x times Dpad, 4 KB), two or
// three in flight (NS).  The launcher takes two where that puts more rows in flight
// at Dpad 64, else three, which hide the copies better.  Smaller stages lose more to
// the per-stage barrier than an extra row gains (2 KB stages, nine rows per SM at
// 848x480 D=128: rows 0.935 -> 0.971 ms per 16 pairs).
constexpr int kRowsChunk = 2048;

template <bool PACKED, int TS, int G, int NS>
__global__ void __launch_bounds__(32 * G, 8 / G) k_rows(DevCfg cfg, Batch b) {
  constexpr int DP = 64 * G;                          // Dpad
  constexpr int XS = DP / 2;                          // x stride in 32-bit words
  constexpr int CH = kRowsChunk / DP;                 // x columns per backward chunk

  constexpr size_t STAGE = size_t(CH) * DP * 2;
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t bars[4 + NS];      // census, ax[2], spare, ring
  int cpm = 0, apm = 0, maxW = 0;
  for (int i = 0; i < b.n; ++i) {
    cpm = max(cpm, b.p[i].cpitch);
    apm = max(apm, b.p[i].apitch);
    maxW = max(maxW, b.p[i].W);
  }
  uint8_t* tabp = smem;
  uint8_t* cbuf = tabp + ScoreTable<TS, 1>::bytes();                 // L | R words
  uint8_t* abuf = cbuf + size_t(cpm) * 16;                            // ax x 2
  const size_t abytes = (size_t(apm) * 2 + 127) & ~size_t(127);
  uint8_t* ring = abuf + 2 * abytes;
  uint8_t* sLp = ring + NS * STAGE;
  uint8_t* sRp = sLp + maxW;
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int i = 0; i < 4 + NS; ++i) mbar_init(&bars[i], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  {
    int16_t* t16 = reinterpret_cast<int16_t*>(tabp);
    for (int i = tid; i < TS * 64; i += blockDim.x) {
      const int m = i >> 6, h = i & 63;
      t16[i] = int16_t((int32_t(cfg.tbl[h]) * (1024 - cfg.wq) + int32_t(cfg.adt[m]) * cfg.wq) >> 10);
    }
  }
  __syncthreads();
  const void* tab = static_cast<const void*>(tabp);
  const int hw = cfg.hw, dmin = cfg.dmin;
  const int total = b.rows_prefix[b.n];
  int* err = b.err;
  const uint64_t* sL = reinterpret_cast<const uint64_t*>(cbuf);       // + lpad below
  const uint64_t* sR = reinterpret_cast<const uint64_t*>(cbuf + size_t(cpm) * 8);

  auto row_of = [&](int item, int* y) -> const DevPair& {
    const int pi = find_pair(b.rows_prefix, b.n, item);
    *y = cfg.hh + (item - b.rows_prefix[pi]);
    return b.p[pi];
  };
  auto issue_census = [&](int item) {                 // thread 0
    int y;
    const DevPair& P = row_of(item, &y);
    const uint32_t cb = uint32_t(P.cpitch) * 8;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect(&bars[0], 2 * cb);
    bulk_load(cbuf, P.cwL + size_t(y) * P.cpitch, cb, &bars[0]);
    bulk_load(cbuf + size_t(cpm) * 8, P.cwR + size_t(y) * P.cpitch, cb, &bars[0]);
  };
  auto issue_ax = [&](int item, int buf) {            // thread 0
    int y;
    const DevPair& P = row_of(item, &y);
    const uint32_t ab = uint32_t(P.apitch) * 2;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect(&bars[1 + buf], ab);
    bulk_load(abuf + buf * abytes, P.ax + size_t(y) * P.apitch, ab, &bars[1 + buf]);
  };

  uint32_t phase = 0;                                 // parity bit per barrier
  auto wait_bar = [&](int i) {
    mbar_wait(&bars[i], (phase >> i) & 1u, err);
    phase ^= 1u << i;
  };
  if (tid == 0 && int(blockIdx.x) < total) { issue_census(blockIdx.x); issue_ax(blockIdx.x, 0); }
  int it = 0;
  for (int item = blockIdx.x; item < total; item += gridDim.x, ++it) {
    const int buf = it & 1;
    const int next = item + int(gridDim.x);
    if (tid == 0 && next < total) issue_ax(next, buf ^ 1);
    int y;
    const DevPair& P = row_of(item, &y);
    const int W = P.W;
    const size_t row = size_t(y) * W;
    wait_bar(0);
    wait_bar(1 + buf);
    const uint64_t* sLx = sL + P.lpad;
    const uint16_t* sax = reinterpret_cast<const uint16_t*>(abuf + buf * abytes) + P.lpad;
    if (!PACKED) {
      for (int i = tid; i < W; i += blockDim.x) { sLp[i] = P.L[row + i]; sRp[i] = P.R[row + i]; }
      __syncthreads();
    }
    const int d0 = dmin + 2 * tid;
    const int xw = hw + dmin + 2 * (tid & ~31);       // first lane's start in this warp
    const int xend = W - hw;                          // scores are 0 from here on
    uint32_t* out = reinterpret_cast<uint32_t*>(P.vol + row * DP) + tid;
    int32_t f0 = 0, f1 = 0;
    {
      uint64_t rprev = (xw - 1 - d0 >= 0) ? sR[xw - 1 - d0] : 0;    // chain k1's word
      int x = xw;
      int xramp = min(xend, xw + 64);                 // lanes may still be before their start
      xramp += (xramp - dmin) & 1;                    // the paired loop needs x - dmin even
      xramp = min(xramp, xend);
      for (; x < xramp; ++x) {
        const int32_t a = sax[x];
        const uint64_t lw = sLx[x];
        int32_t v0 = 0, v1 = 0;
        uint64_t rw = 0;
        if (x - d0 >= hw) {
          rw = sR[x - d0];
          v0 = graded<PACKED, TS, 1>(lw, rw, tab, sLp, sRp, x, x - d0);
        }
        if (x - d0 - 1 >= hw) v1 = graded<PACKED, TS, 1>(lw, rprev, tab, sLp, sRp, x, x - d0 - 1);
        rprev = rw;
        f0 = rf_step(v0, f0, a);
        f1 = rf_step(v1, f1, a);
        out[x * XS] = pack2(f0, f1);
      }
      const uint64_t* rp = sR + (x - d0);
      const uint64_t* lp = sLx + x;
      const uint16_t* ap = sax + x;
      uint32_t* op = out + x * XS;
#pragma unroll 8
      for (; x + 1 < xend; x += 2) {                  // two x per iteration
        const uint32_t a2 = *reinterpret_cast<const uint32_t*>(ap);
        const ulonglong2 l2 = *reinterpret_cast<const ulonglong2*>(lp);
        const ulonglong2 r2 = *reinterpret_cast<const ulonglong2*>(rp);
        const int32_t a0 = int32_t(a2 & 0xFFFFu), a1 = int32_t(a2 >> 16);
        const int32_t v00 = graded<PACKED, TS, 1>(l2.x, r2.x, tab, sLp, sRp, x, x - d0);
        const int32_t v01 = graded<PACKED, TS, 1>(l2.x, rprev, tab, sLp, sRp, x, x - d0 - 1);
        const int32_t v10 = graded<PACKED, TS, 1>(l2.y, r2.y, tab, sLp, sRp, x + 1, x + 1 - d0);
        const int32_t v11 = graded<PACKED, TS, 1>(l2.y, r2.x, tab, sLp, sRp, x + 1, x - d0);
        rprev = r2.y;
        f0 = rf_step(v00, f0, a0);
        f1 = rf_step(v01, f1, a0);
        op[0] = pack2(f0, f1);
        f0 = rf_step(v10, f0, a1);
        f1 = rf_step(v11, f1, a1);
        op[XS] = pack2(f0, f1);
        rp += 2; lp += 2; ap += 2; op += 2 * XS;
      }
      for (; x < xend; ++x) {                         // at most one leftover step
        const int32_t a = sax[x];
        const uint64_t lw = sLx[x];
        const uint64_t rw = sR[x - d0];
        const int32_t v0 = graded<PACKED, TS, 1>(lw, rw, tab, sLp, sRp, x, x - d0);
        const int32_t v1 = graded<PACKED, TS, 1>(lw, rprev, tab, sLp, sRp, x, x - d0 - 1);
        rprev = rw;
        f0 = rf_step(v0, f0, a);
        f1 = rf_step(v1, f1, a);
        out[x * XS] = pack2(f0, f1);
      }
      for (; x < W; ++x) {                            // right border, score 0
        const int32_t a = sax[x];
        f0 = rf_step(0, f0, a);
        f1 = rf_step(0, f1, a);
        out[x * XS] = pack2(f0, f1);
      }
    }
    // backward; the census buffer is free now, so the next row's words start loading
    fence_proxy_async();                              // our stores before the async reads
    __syncthreads();
    if (tid == 0 && next < total) issue_census(next);
    const int xlo_cta = hw + dmin;
    const int jmax = (W - 2) / CH, jmin = xlo_cta / CH;
    auto issue_chunk = [&](int j, int slot) {
      const int xa = j * CH;
      const uint32_t bytes = uint32_t(min(CH, W - xa)) * uint32_t(DP) * 2u;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // stage reads done
      mbar_expect(&bars[4 + slot], bytes);
      bulk_load(ring + slot * STAGE, P.vol + (row + xa) * DP, bytes, &bars[4 + slot]);
    };
    if (tid == 0)
      for (int q = 0; q < NS && jmax - q >= jmin; ++q) issue_chunk(jmax - q, q);
    int32_t g0 = f0, g1 = f1;                         // seed: forward value at W-1
    int slot = 0;
    for (int j = jmax; j >= jmin; --j) {
      wait_bar(4 + slot);
      const int xa = j * CH;
      const uint32_t* cb = reinterpret_cast<const uint32_t*>(ring + slot * STAGE) + tid;
      const int xhi = min(W - 2, xa + CH - 1);
      const int xlo = max(xa, xw);
      if (xhi == xa + CH - 1 && xlo == xa) {          // a full chunk: unrolled
        uint32_t* o = out + xa * XS;
        const uint16_t* a1p = sax + xa + 1;
#pragma unroll
        for (int q = CH - 1; q >= 0; --q) {
          const uint32_t c = cb[q * XS];
          const int32_t a = a1p[q];
          g0 = rf_step(lo16(c), g0, a);
          g1 = rf_step(hi16(c), g1, a);
          o[q * XS] = pack2(g0, g1);
        }
      } else {
        for (int x = xhi; x >= xlo; --x) {
          const uint32_t c = cb[(x - xa) * XS];
          const int32_t a = sax[x + 1];
          g0 = rf_step(lo16(c), g0, a);
          g1 = rf_step(hi16(c), g1, a);
          out[x * XS] = pack2(g0, g1);
        }
      }
      __syncthreads();                                // stage consumed by every thread
      if (tid == 0 && j - NS >= jmin) issue_chunk(j - NS, slot);
      slot = (slot + 1 == NS) ? 0 : slot + 1;
    }
  }
  // Test hook (knob "expire_wait_polls"): once every real wait has completed and no
  // copy is in flight, the launch's first CTA waits a bounded number of polls on the
  // spare barrier, which nothing arrives at, so the time-out path of a device wait and
  // the status it reports are exercised without a fault.
  if (cfg.expire_polls > 0 && blockIdx.x == 0 && tid == 0)
    mbar_wait(&bars[3], 0u, err, cfg.expire_polls);
}

// ---------------------------------------------------------------------------------
__device__ __forceinline__ int32_t sx16(uint32_t v) {     // sign-extended low half
  return int32_t(int16_t(uint16_t(v & 0xFFFFu)));
}
__device__ __forceinline__ int32_t hx16(uint32_t v) { return int32_t(v) >> 16; }
__device__ __forceinline__ uint32_t pk16(int32_t lo, int32_t hi) {
  return __byte_perm(uint32_t(lo), uint32_t(hi), 0x5410);
}

// k_cols: vertical forward (in place), vertical backward + top-2 + neighbours.
// Vertical passes: core/tools/de_dense.cpp:490-507.  Top-2 semantics: :1276-1292
// (ascending k, strictly greater, ties keep the smaller k), sub-pixel neighbour
// capture :1276-1285.
//
// A column is a group of TPC = Dpad/KT lanes (padded to TPCP, a power of two);
// lane s of the group owns disparities [s*KT, s*KT + KT) as int16 pairs, so one row
// of one column is 2*Dpad contiguous bytes, and adjacent columns are adjacent in
// memory.  The top-2 key (v + 32768) << 8 | (255 - k) is unique per k, so the
// strictly-greater insertion is three unsigned min/max, the merge across lanes is
// four, and any merge order gives the sequential scan's answer.  The winner's
// neighbour costs are read back from a per-group row buffer.
//
// No block-wide step: each lane reads its own 2*KT bytes of a row from global memory,
// PF rows ahead of use (the rows of a warp's columns are adjacent, so a warp's loads
// and stores of one row are contiguous), and the only synchronisation is the group's
// own merge of a column's lanes.  At 8 disparities per lane (AS) the ring is the
// lane's own 16-byte slots in shared memory, filled by cp.async and read after
// cp.async.wait_group: it needs no registers, so the kernel runs at 80 registers and
// three 256-thread CTAs per SM (two with a register ring), and a concurrent launch
// set finds room beside it (the 16-pair batch 2.53 -> 2.41 ms, 1280x720 D=256 4.76 ->
// 4.43 ms); the kernel alone times the same.  Otherwise the ring is in registers.  Warps
// therefore run at their own pace instead of meeting at a barrier every row.  A lane
// reads back only what it stored itself in the forward pass.  Only the filter state
// runs from row to row, so the backward pass merges several rows' keys together
// (one row buffer each) and their shuffle chains interleave.  KT = 4 gives one
// column per warp (the most columns in flight, for small batches); 8 and 16 trade
// columns for disparities per lane.
template <int KW>   // KW 32-bit words (2*KW disparities) per lane and row
__device__ __forceinline__ void vload(const uint32_t* p, uint32_t* w) {
  if constexpr (KW == 2) {
    const uint2 v = __ldcg(reinterpret_cast<const uint2*>(p));
    w[0] = v.x; w[1] = v.y;
  } else {
#pragma unroll
    for (int i = 0; i < KW / 4; ++i) {
      const uint4 v = __ldcg(reinterpret_cast<const uint4*>(p) + i);
      w[4 * i] = v.x; w[4 * i + 1] = v.y; w[4 * i + 2] = v.z; w[4 * i + 3] = v.w;
    }
  }
}
template <int KW>
__device__ __forceinline__ void vstore(uint32_t* p, const uint32_t* w) {
  if constexpr (KW == 2) {
    *reinterpret_cast<uint2*>(p) = make_uint2(w[0], w[1]);
  } else {
#pragma unroll
    for (int i = 0; i < KW / 4; ++i)
      reinterpret_cast<uint4*>(p)[i] = make_uint4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
  }
}

// Ampere-style asynchronous copies (cp.async) of 16 bytes into shared memory, counted
// in commit groups; each lane copies and later reads only its own slots.  The source
// operand `dep` only orders the copy after the register it names is ready (the slot's
// previous contents have been read into it).
__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t dep) {
  asm volatile("{ .reg .b32 d; mov.b32 d, %2; cp.async.cg.shared.global [%0], [%1], 16; }"
               ::"r"(smem_addr(dst)), "l"(src), "r"(dep) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int KT, int TPCP, int PF, int NT, bool AS = false>
__global__ void __launch_bounds__(NT, (AS ? 768 : 512) / NT) k_cols(DevCfg cfg, Batch b) {
  static_assert((KT == 4 || KT % 8 == 0) && TPCP >= 1 && TPCP <= 32, "shape");
  static_assert(!AS || KT == 8, "the asynchronous ring moves 16 bytes a lane and row");
  constexpr int KW = KT / 2;                         // 32-bit words per lane and row
  constexpr int NCOL = NT / TPCP;                    // columns per CTA tile
  // backward rows whose lane merges run together: 8 where the prefetch ring is 8 or
  // 16 deep (at 8 disparities per lane this spills a few bytes of loop-invariant
  // state and is still the fastest), 4 with a 4-deep ring, 2 at 16 disparities per
  // lane (more would spill)
  constexpr int kRB = KT >= 16 ? 2 : (PF >= 8 ? 8 : 4);
  __shared__ __align__(16) int16_t sbuf[NT / 32][kRB][32 * KT];   // kRB row buffers per warp
  // AS: the prefetch ring in (dynamic) shared memory, PF slots of 16 bytes per lane,
  // so it costs no registers (more warps per SM) and no barrier (a lane reads only its
  // own slots); per warp, slot j of lane l is word (j * 32 + l) * KW
  extern __shared__ __align__(16) uint32_t sring[];
  const int tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
  const int gi = tid / TPCP, sub = tid % TPCP, gbase = lane - sub;
  const unsigned gmask = (TPCP == 32) ? 0xffffffffu : (((1u << TPCP) - 1u) << gbase);
  const int tile = blockIdx.x;
  const int pi = find_pair(b.cols_prefix, b.n, tile);
  const DevPair& P = b.p[pi];
  const int W = P.W, H = P.H, D = P.D, Dpad = P.Dpad;
  const int hw = cfg.hw, hh = cfg.hh, dmin = cfg.dmin;
  const int xbase = hw + dmin + (tile - b.cols_prefix[pi]) * NCOL;
  const int ncols = min(NCOL, W - hw - xbase);
  const int x = xbase + gi;
  const int k0 = sub * KT;
  const bool colok = gi < ncols;
  const int kmax = colok ? min(D - 1, x - hw - dmin) : -1;
  // A lane whose disparities all lie past kmax (the left-edge triangle, or past D)
  // feeds neither a key nor a neighbour cost, so it is not live.
  const bool live = colok && k0 < Dpad && k0 <= kmax;
  const int nvalid = max(0, min(KT, kmax - k0 + 1));
  const int yin = H - hh;                             // rows >= yin have zero input
  const size_t grs = size_t(W) * Dpad / 2;            // image-row stride in words
  // Every lane reads a valid address, so the loads need no guard: a lane that is not
  // live reads its group's first lane's words (the same sectors, no extra traffic)
  // and never uses them; only live lanes store.
  uint32_t* gcol = reinterpret_cast<uint32_t*>(P.vol + size_t(colok ? x : xbase) * Dpad +
                                               (live ? k0 : 0));
  const uint16_t* ay = P.ay + (colok ? x : xbase);
  int32_t st[KT];
#pragma unroll
  for (int s = 0; s < KT; ++s) st[s] = 0;
  auto step = [&](const uint32_t* w, int32_t a) {
#pragma unroll
    for (int i = 0; i < KW; ++i) {
      st[2 * i] = rf_step(sx16(w[i]), st[2 * i], a);
      st[2 * i + 1] = rf_step(hx16(w[i]), st[2 * i + 1], a);
    }
  };
  auto pack_state = [&](uint32_t* w) {
#pragma unroll
    for (int i = 0; i < KW; ++i) w[i] = pk16(st[2 * i], st[2 * i + 1]);
  };
  auto fetch = [&](int y, uint32_t* dst) { vload<KW>(gcol + size_t(y) * grs, dst); };
  // The steady-state loops below run whole blocks of PF rows with no branch, so a
  // load issued PF rows ahead stays in flight until its row; a guarded tail finishes.
  uint32_t ring[AS ? 1 : PF][KW] = {};
  int32_t aring[PF] = {};
  // ring slot j: take the row it holds (AS: once its copy group has landed; one group
  // per row, rows taken in issue order, so PF - 1 newer groups may stay in flight) and
  // refill it with row y
  uint32_t* const myslot = AS ? sring + wib * (PF * 32 * KW) + lane * KW : nullptr;
  auto ring_take = [&](int j, uint32_t* c) {
    if constexpr (AS) {
      cp_async_wait<PF - 1>();
      const uint4 v = *reinterpret_cast<const uint4*>(myslot + j * 32 * KW);
      c[0] = v.x; c[1] = v.y; c[2] = v.z; c[3] = v.w;
    } else {
#pragma unroll
      for (int i = 0; i < KW; ++i) c[i] = ring[j][i];
    }
  };
  auto ring_fill = [&](int j, int y, uint32_t dep) {
    if constexpr (AS) {
      cp_async16(myslot + j * 32 * KW, gcol + size_t(y) * grs, dep);
      cp_async_commit();
    } else {
      fetch(y, ring[j]);
    }
  };
  const int ylast = clampi(yin - 1, 0, H - 1);        // last row with input
  // ---- vertical forward, rows hh..H-1, results stored in place --------------------
  auto fwd = [&](int y, int j) {
    uint32_t c[KW];
    ring_take(j, c);
    const uint32_t dep = c[0];
#pragma unroll
    for (int i = 0; i < KW; ++i) c[i] = (y < yin) ? c[i] : 0u;
    const int32_t a = aring[j];
    const int yn = y + PF;
    ring_fill(j, min(yn, ylast), dep);
    aring[j] = ay[size_t(min(yn, H - 1)) * W];
    step(c, a);
    if (live) {
      uint32_t o[KW];
      pack_state(o);
      vstore<KW>(gcol + size_t(y) * grs, o);
    }
  };
#pragma unroll
  for (int j = 0; j < PF; ++j) {
    ring_fill(j, min(hh + j, ylast), 0u);
    aring[j] = ay[size_t(min(hh + j, H - 1)) * W];
  }
  int y0 = hh;
  for (; y0 + PF <= H; y0 += PF) {
#pragma unroll
    for (int j = 0; j < PF; ++j) fwd(y0 + j, j);
  }
#pragma unroll
  for (int j = 0; j < PF; ++j)
    if (y0 + j < H) fwd(y0 + j, j);
  if constexpr (AS) cp_async_wait<0>();               // the forward's last refills land
  // ---- vertical backward from H-1 (its value is the forward one) + top-2 ----------
  // Rows yin..H-2 carry no candidates: plain steps with direct loads.
  int ys = H - 2;
  for (; ys >= yin && ys >= hh; --ys) {
    uint32_t c[KW];
    fetch(ys, c);
    step(c, ay[size_t(ys + 1) * W]);
  }
  if (ys < hh) return;
  int16_t* rowbufs[kRB];
#pragma unroll
  for (int i = 0; i < kRB; ++i) rowbufs[i] = &sbuf[wib][i][gbase * KT];
  constexpr int kRowbufLast = TPCP * KT - 1;          // the group's last rowbuf entry
  auto bwd_rows = [&](auto with_rkey) {
    constexpr bool RK = decltype(with_rkey)::value;
    // One row: the filter step, the lane's top-2 keys, and its costs into a row
    // buffer (for the winner's neighbours).
    auto row_keys = [&](int y, int j, uint32_t& pk0, uint32_t& pk1, int16_t* rowbuf) {
      uint32_t c[KW];
      ring_take(j, c);
      const int32_t a = aring[j];
      const int yn = y - PF;
      ring_fill(j, max(yn, 0), c[0]);
      aring[j] = ay[size_t(max(yn + 1, 0)) * W];
      step(c, a);
      pk0 = 0;
      pk1 = 0;                                        // key 0 never displaces a candidate
#pragma unroll
      for (int s = 0; s < KT; ++s) {
        const uint32_t key =
            (s < nvalid) ? (uint32_t(st[s] + 32768) << 8) | uint32_t(255 - k0 - s) : 0u;
        const uint32_t lo = min(pk0, key);
        pk0 = max(pk0, key);
        pk1 = max(pk1, lo);
      }
      if (RK) {
        const size_t rowo = size_t(y) * W + x - dmin - k0;
#pragma unroll
        for (int s = 0; s < KT; ++s)
          if (s < nvalid)
            atomicMax(P.rkey + rowo - s, (uint32_t(st[s] + 32768) << 8) | uint32_t(255 - k0 - s));
      }
      uint32_t o[KW];
      pack_state(o);
      vstore<KW>(reinterpret_cast<uint32_t*>(rowbuf + k0), o);
    };
    auto merge_step = [&](uint32_t& pk0, uint32_t& pk1, int off) {
      const uint32_t o0 = __shfl_xor_sync(gmask, pk0, off, TPCP);
      const uint32_t o1 = __shfl_xor_sync(gmask, pk1, off, TPCP);
      const uint32_t lo = min(pk0, o0);
      pk0 = max(pk0, o0);
      pk1 = max(max(pk1, o1), lo);
    };
    // a lane holding a row's merged keys writes them, with the winner's neighbours
    auto emit = [&](int y, uint32_t pk0, uint32_t pk1, const int16_t* rowbuf) {
      const int kw = pk0 ? 255 - int(pk0 & 255u) : -1;
      const int32_t vm = rowbuf[max(kw - 1, 0)];
      const int32_t vp = rowbuf[min(kw + 1, kRowbufLast)];
      const int32_t nm = (kw >= 1) ? vm : -32768;
      const int32_t np = (kw >= 0 && kw + 1 <= kmax) ? vp : -32768;
      const size_t i = size_t(y) * W + x;
      P.key0[i] = pk0;
      P.key1[i] = pk1;
      P.nb[i] = pk16(nm, np);
    };
    auto bwd = [&](int y, int j) {                   // one row
      uint32_t pk0, pk1;
      __syncwarp(gmask);                              // the previous rows' reads are done
      row_keys(y, j, pk0, pk1, rowbufs[0]);
#pragma unroll
      for (int off = TPCP / 2; off > 0; off >>= 1) merge_step(pk0, pk1, off);
      __syncwarp(gmask);
      if (sub == 0 && colok) emit(y, pk0, pk1, rowbufs[0]);
    };
    // kRB rows at a time, merged across the group's lanes by recursive halving: in
    // round t lanes h = TPCP >> (t + 1) apart pair up, each keeps half of the rows it
    // holds (the upper half where its bit h is set) and merges its partner's partial
    // keys for them, so after log2(kRB) rounds lane `sub` holds row sub / (TPCP /
    // kRB) alone, merged over kRB lanes; a butterfly over the remaining TPCP / kRB
    // lanes finishes it.  That is 2 kRB - 1 merges a lane (kRB log2(TPCP) with a
    // butterfly per row), and kRB lanes write the kRB rows side by side.  The merge
    // is order-free, so the result is the sequential scan's.
    static_assert(TPCP >= kRB, "each lane ends with one row");
    constexpr int kLanesPerRow = TPCP / kRB;
    auto bwdn = [&](int y, int j) {                   // rows y, y - 1, ..., y - kRB + 1
      uint32_t k0s[kRB], k1s[kRB];
      __syncwarp(gmask);
#pragma unroll
      for (int r = 0; r < kRB; ++r) row_keys(y - r, j + r, k0s[r], k1s[r], rowbufs[r]);
#pragma unroll
      for (int h = TPCP / 2, half = kRB / 2; half > 0; h >>= 1, half >>= 1) {
        const bool up = (sub & h) != 0;
#pragma unroll
        for (int i = 0; i < half; ++i) {
          const uint32_t s0 = up ? k0s[i] : k0s[i + half];
          const uint32_t s1 = up ? k1s[i] : k1s[i + half];
          const uint32_t m0 = up ? k0s[i + half] : k0s[i];
          const uint32_t m1 = up ? k1s[i + half] : k1s[i];
          const uint32_t o0 = __shfl_xor_sync(gmask, s0, h, TPCP);
          const uint32_t o1 = __shfl_xor_sync(gmask, s1, h, TPCP);
          const uint32_t lo = min(m0, o0);
          k0s[i] = max(m0, o0);
          k1s[i] = max(max(m1, o1), lo);
        }
      }
#pragma unroll
      for (int off = kLanesPerRow / 2; off > 0; off >>= 1) merge_step(k0s[0], k1s[0], off);
      __syncwarp(gmask);
      const int r = sub / kLanesPerRow;
      if (sub % kLanesPerRow == 0 && colok) emit(y - r, k0s[0], k1s[0], &sbuf[wib][r][gbase * KT]);
    };
#pragma unroll
    for (int j = 0; j < PF; ++j) {
      ring_fill(j, max(ys - j, 0), 0u);
      aring[j] = ay[size_t(max(ys - j + 1, 0)) * W];   // coefficient at y + 1
    }
    int yb = ys;
    static_assert(PF % kRB == 0, "rows are taken kRB at a time");
    for (; yb - PF + 1 >= hh; yb -= PF) {
#pragma unroll
      for (int j = 0; j < PF; j += kRB) bwdn(yb - j, j);
    }
#pragma unroll
    for (int j = 0; j < PF; ++j)
      if (yb - j >= hh) bwd(yb - j, j);
  };
  if (P.rkey) bwd_rows(std::integral_constant<bool, true>());
  else bwd_rows(std::integral_constant<bool, false>());
  if constexpr (AS) cp_async_wait<0>();               // no copy outlives the CTA
}

// ---------------------------------------------------------------------------------
// k_solve: the row solve, core/include/doubleeye/dense_solve.hpp:213-452 (K = 2,
// candidates from the cost stage), plus the --out-conf planes and the confidence
// (:158-171).  One CTA per row; shared-memory working set 49 bytes per pixel.


__device__ __forceinline__ float fmax_ref(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float fmin_ref(float a, float b) { return (b < a) ? b : a; }

__device__ float confidence_dev(float s1, float s2, float lambda, float lrc, float tol) {
  if (!(s1 > -1e29f)) return 0.f;
  const float alt = (s2 > -1e29f) ? fmax_ref(s2, lambda) : lambda;
  const float x = logf(fmax_ref((1.f - alt) / fmax_ref(1.f - s1, 1e-6f), 1e-6f));
  const float logit = 0.692684f + 7.936751f * x;
  const float p = 1.f / (1.f + expf(-fmax_ref(-30.f, fmin_ref(30.f, logit))));
  return (lrc > tol) ? fmin_ref(p, 0.35f) : p;
}

template <int kSolveThreads>
__device__ __forceinline__ void block_excl_scan(int* a, int n, int* warp_sums) {
  // exclusive scan of a[0..n) in place, a[n] = total; contiguous chunks per thread
  const int tid = threadIdx.x;
  const int per = (n + kSolveThreads - 1) / kSolveThreads;
  const int lo = min(n, tid * per), hi = min(n, lo + per);
  int s = 0;
  for (int i = lo; i < hi; ++i) s += a[i];
  // inclusive warp scan of s
  const int lane = tid & 31, w = tid >> 5;
  int v = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  if (lane == 31) warp_sums[w] = v;
  __syncthreads();
  if (w == 0) {
    int ws = lane < (kSolveThreads / 32) ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, ws, o);
      if (lane >= o) ws += u;
    }
    if (lane < kSolveThreads / 32) warp_sums[lane] = ws;
  }
  __syncthreads();
  int run = v - s + (w > 0 ? warp_sums[w - 1] : 0);
  for (int i = lo; i < hi; ++i) { const int c = a[i]; a[i] = run; run += c; }
  if (tid == kSolveThreads - 1) a[n] = run;
  __syncthreads();
}

// At most 40 registers (six 256-thread CTAs' worth, no spills): the solve still fits
// five rows per SM by shared memory, and the registers it leaves free let the other
// launch set's kernels run beside it (the 16-pair batch 2.381 -> 2.376 ms).
template <bool REF_LAYOUT, int kSolveThreads>
__global__ void __launch_bounds__(kSolveThreads, 1536 / kSolveThreads) k_solve(DevCfg cfg, Batch b) {
  extern __shared__ __align__(128) uint8_t smem[];
  const int item = blockIdx.x;
  const int pi = find_pair(b.solve_prefix, b.n, item);
  const DevPair& P = b.p[pi];
  const int W = P.W, H = P.H;
  const int y = item - b.solve_prefix[pi];
  const int dmin = cfg.dmin, hw = cfg.hw, hh = cfg.hh;
  const float lambda = cfg.lambda, gamma = cfg.gamma, damping = cfg.damping, keep = cfg.keep;
  // Candidate state lives in bucket-sorted POSITION order: the members of a right
  // pixel's bucket are contiguous, candidates that claim no right pixel follow them.
  // Shared bytes per pixel: cs 8, beta 8, rho 8, lohi 8, start 4, item 4, pos 4,
  // cd 2, rev 2, cn 1 = 49 (five rows per SM at W = 848).  Arrays that are never
  // live together share storage: the sort cursors live in beta until beta is
  // cleared, pixel-order cs in rho until the sort, and the claim stage's best,
  // bestj and win in lohi, which only the BP sweeps read.
  float* __restrict__ s_cs = reinterpret_cast<float*>(smem);          // [2W] by position
  float* __restrict__ s_beta = s_cs + 2 * W;                           // [2W] by position
  float* __restrict__ s_rho = s_beta + 2 * W;                          // [2W] by position (pixel-order cs first)
  int* __restrict__ s_lohi = reinterpret_cast<int*>(s_rho + 2 * W);    // [2W] bucket bounds lo | hi << 16, -1 none
  int* s_start = s_lohi + 2 * W;                          // [W+1]
  int16_t* s_item = reinterpret_cast<int16_t*>(s_start + W + 1);   // [2W] position -> 2x + j
  int16_t* s_pos = s_item + 2 * W;                        // [2W] 2x + j -> position
  uint8_t* s_cd = reinterpret_cast<uint8_t*>(s_pos + 2 * W);  // [2W] k (valid for j < cn)
  int16_t* s_rev = reinterpret_cast<int16_t*>(s_cd + 2 * W);  // [W]
  int8_t* s_cn = reinterpret_cast<int8_t*>(s_rev + W);    // [W]
  float* s_cspx = s_rho;                                  // pixel-order cs until the sort
  int* s_cur = reinterpret_cast<int*>(s_beta);            // [W] sort cursors until beta is cleared
  float* s_best = reinterpret_cast<float*>(s_lohi);       // [W] after the BP sweeps
  int8_t* s_bestj = reinterpret_cast<int8_t*>(s_lohi + W);     // [W] after the BP sweeps
  uint8_t* s_win = reinterpret_cast<uint8_t*>(s_bestj + W);    // [W] after the BP sweeps
  __shared__ int warp_sums[kSolveThreads / 32];
  __shared__ int s_nitems, s_extra;
  const int tid = threadIdx.x;
  const bool row_ok = y >= hh && y < H - hh;
  const size_t row = size_t(y) * W;
  const float q = 1.f / 16384.f;

  // 1. candidates + margin (dense_solve.hpp:263-268).  The packed keys of a thread's
  //    pixels are fetched four pixels at a time before any is used, so their global
  //    loads overlap instead of waiting one after another.
  auto candidates = [&](int x, uint32_t a, uint32_t bb) {
    int n = 0;
    float c0 = kNegBig, c1 = kNegBig;
    int k0 = 0, k1 = 0;
    if (REF_LAYOUT) {
      n = P.ref_cn[row + x];
      if (n > 0) { c0 = P.ref_cs[2 * (row + x)]; k0 = P.ref_cd[2 * (row + x)]; }
      if (n > 1) { c1 = P.ref_cs[2 * (row + x) + 1]; k1 = P.ref_cd[2 * (row + x) + 1]; }
    } else {
      if (a) { c0 = float(int32_t(a >> 8) - 32768) * q; k0 = 255 - int(a & 255u); n = 1; }
      if (bb) { c1 = float(int32_t(bb >> 8) - 32768) * q; k1 = 255 - int(bb & 255u); n = 2; }
    }
    reinterpret_cast<float2*>(s_cspx)[x] = make_float2(c0, c1);
    s_cd[2 * x] = uint8_t(k0);
    s_cd[2 * x + 1] = uint8_t(k1);
    s_cn[x] = int8_t(n);
    const float alt = (n < 2) ? lambda : fmax_ref(c1, lambda);
    const float m = (n == 0) ? 0.f : c0 - alt;
    if (P.margin) P.margin[row + x] = m;
    s_start[x] = 0;
  };
  for (int xb = tid; xb < W; xb += 4 * kSolveThreads) {
    uint32_t a[4], bb[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int x = xb + u * kSolveThreads;
      const bool ok = !REF_LAYOUT && row_ok && x >= hw + dmin && x < W - hw;
      a[u] = ok ? P.key0[row + x] : 0u;
      bb[u] = ok ? P.key1[row + x] : 0u;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (xb + u * kSolveThreads < W) candidates(xb + u * kSolveThreads, a[u], bb[u]);
  }
  if (tid == 0) { s_start[W] = 0; s_extra = 0; }
  __syncthreads();
  // 2. claimant buckets by right pixel, counting sort (:270-284); the order inside a
  //    bucket is free: only its maxima are ever read
  for (int x = tid; x < W; x += kSolveThreads)
    for (int j = 0; j < s_cn[x]; ++j) {
      const int xr = x - (dmin + s_cd[2 * x + j]);
      if (xr >= 0) atomicAdd(&s_start[xr], 1);
    }
  __syncthreads();
  block_excl_scan<kSolveThreads>(s_start, W, warp_sums);
  for (int xr = tid; xr < W; xr += kSolveThreads) s_cur[xr] = s_start[xr];
  if (tid == 0) s_nitems = s_start[W];
  __syncthreads();
  const int nitems = s_nitems;
  for (int x = tid; x < W; x += kSolveThreads) {
    const int n = s_cn[x];
    for (int j = 0; j < n; ++j) {
      const int xr = x - (dmin + s_cd[2 * x + j]);
      int p, lohi = -1;
      if (xr >= 0) {
        p = atomicAdd(&s_cur[xr], 1);
        lohi = s_start[xr] | (s_start[xr + 1] << 16);
      } else {
        p = nitems + atomicAdd(&s_extra, 1);
      }
      s_item[p] = int16_t(2 * x + j);
      s_pos[2 * x + j] = int16_t(p);
      s_cs[p] = s_cspx[2 * x + j];
      s_lohi[p] = lohi;
    }
  }
  __syncthreads();
  const int nall = nitems + s_extra;
  for (int p = tid; p < nall; p += kSolveThreads) { s_beta[p] = 0.f; s_rho[p] = 0.f; }
  // 3. reverse match over the surviving candidates (:303-313): first maximum in x order
  //    (value desc, index asc) is a total order, so members may be folded four at a
  //    time with their loads issued together
  for (int xr = tid; xr < W; xr += kSolveThreads) {
    int bi = 1 << 30;
    float bv = kNegBig;
    const int lo = s_start[xr], hi = s_start[xr + 1];
    for (int p0 = lo; p0 < hi; p0 += 4) {
      int idx[4];
      float v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int p = min(p0 + u, hi - 1);
        idx[u] = s_item[p];
        v[u] = s_cs[p];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (p0 + u < hi && (v[u] > bv || (v[u] == bv && idx[u] < bi))) { bv = v[u]; bi = idx[u]; }
    }
    s_rev[xr] = int16_t(bi < (1 << 30) ? int(s_cd[bi]) : -1);
  }
  // 4. damped max-sum iterations (:318-341): rho per pixel (its partner's beta through
  //    the position table), beta per bucket position ("max over my bucket excluding me"
  //    over a contiguous run of rho)
  for (int it = 0; it < cfg.iters; ++it) {
    __syncthreads();
    for (int x = tid; x < W; x += kSolveThreads) {
      const int n = s_cn[x];
      if (n == 0) continue;
      const int p0 = s_pos[2 * x];
      if (n == 1) {
        s_rho[p0] = keep * (s_cs[p0] - lambda) + damping * s_rho[p0];
      } else {
        const int p1 = s_pos[2 * x + 1];
        const float b0 = s_beta[p0], b1 = s_beta[p1];
        const float r0 = keep * (s_cs[p0] - fmax_ref(lambda, b1)) + damping * s_rho[p0];
        const float r1 = keep * (s_cs[p1] - fmax_ref(lambda, b0)) + damping * s_rho[p1];
        s_rho[p0] = r0;
        s_rho[p1] = r1;
      }
    }
    __syncthreads();
    for (int p = tid; p < nitems; p += kSolveThreads) {
      const int lohi = s_lohi[p];
      const int lo = lohi & 0xFFFF, hi = lohi >> 16;     // p's bucket, hi > lo
      // The first four members are read at once and reduced as a tree; fmax_ref
      // keeps its left operand on ties, so the tree returns the scan's first
      // maximum, and members past the fourth continue the scan from it.
      float v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int r = lo + u;
        const float t = s_rho[min(r, hi - 1)];
        v[u] = (r < hi && r != p) ? t : kNegBig;
      }
      float ex = fmax_ref(fmax_ref(v[0], v[1]), fmax_ref(v[2], v[3]));
      for (int r = lo + 4; r < hi; ++r)
        if (r != p) ex = fmax_ref(ex, s_rho[r]);
      s_beta[p] = keep * (s_cs[p] - fmax_ref(gamma, ex)) + damping * s_beta[p];
    }
  }
  __syncthreads();
  // 5. belief (:343-358) and the gates (:364-374) folded into eligibility
  for (int x = tid; x < W; x += kSolveThreads) {
    float best = kNegBig;
    int bj = -1;
    const int n = s_cn[x];
    s_win[x] = 0;
    for (int j = 0; j < n; ++j) {
      const int p = s_pos[2 * x + j];
      const float c = s_cs[p];
      if (c <= lambda) continue;
      const float bel = (cfg.iters > 0) ? (s_beta[p] + s_rho[p] - c) : c;
      if (bel > best) { best = bel; bj = j; }
    }
    if (bj >= 0 && cfg.min_margin > 0.f) {
      // the margin of stage 1, from the same two scores
      const float c0 = s_cs[s_pos[2 * x]];
      const float alt = (n < 2) ? lambda : fmax_ref(s_cs[s_pos[2 * x + 1]], lambda);
      if (c0 - alt < cfg.min_margin) bj = -1;
    }
    if (bj >= 0 && cfg.min_ratio > 0.f) {
      const float s2 = (n > 1) ? fmax_ref(s_cs[s_pos[2 * x + 1]], lambda) : lambda;
      const float c1 = fmax_ref(1.f - s_cs[s_pos[2 * x]], 1e-6f);
      if ((1.f - s2) / c1 < cfg.min_ratio) bj = -1;
    }
    s_best[x] = best;
    s_bestj[x] = int8_t(bj);
  }
  __syncthreads();
  // 6. one-to-one claim (:359-378): each eligible pixel claims exactly one right
  //    pixel, so the sequential greedy pass equals, per right pixel, the claimant
  //    first in (belief desc, x asc) order.
  //    (belief desc, x asc) is a total order (a bucket holds at most one candidate
  //    per pixel), so members are folded four at a time, loads first.
  for (int xr = tid; xr < W; xr += kSolveThreads) {
    int wx = -1;
    float wb = 0.f;
    const int lo = s_start[xr], hi = s_start[xr + 1];
    for (int p0 = lo; p0 < hi; p0 += 4) {
      int xs[4];
      bool el[4];
      float bvs[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int idx = s_item[min(p0 + u, hi - 1)];
        xs[u] = idx >> 1;
        el[u] = p0 + u < hi && s_bestj[xs[u]] == (idx & 1);
        bvs[u] = s_best[xs[u]];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (el[u] && (wx < 0 || bvs[u] > wb || (bvs[u] == wb && xs[u] < wx))) { wx = xs[u]; wb = bvs[u]; }
    }
    if (wx >= 0) s_win[wx] = 1;
  }
  __syncthreads();
  // 7. outputs: disparity with sub-pixel fit (:380-434), reverse-match residuals
  //    (:442-451, core/tools/de_dense.cpp:1581-1597), candidate planes, confidence
  const size_t WH = size_t(W) * H;
  auto outputs = [&](int x, uint32_t nb) {
    float dl = __int_as_float(0x7fc00000);
    const int n = s_cn[x];
    const float2 cs2 = make_float2(n > 0 ? s_cs[s_pos[2 * x]] : kNegBig,
                                   n > 1 ? s_cs[s_pos[2 * x + 1]] : kNegBig);
    if (s_win[x]) {
      const int j = s_bestj[x];
      const int d = dmin + s_cd[2 * x + j];
      float off = 0.f;
      if (cfg.subpixel && j == 0) {
        int32_t m16 = -32768, p16 = -32768;
        if (REF_LAYOUT) {
          if (P.ref_cnb) { m16 = P.ref_cnb[2 * (row + x)]; p16 = P.ref_cnb[2 * (row + x) + 1]; }
        } else {
          m16 = lo16(nb); p16 = hi16(nb);
        }
        const float c0 = cs2.x;
        const float cm = (m16 == -32768) ? kNegBig : float(m16) * q;
        const float cp = (p16 == -32768) ? kNegBig : float(p16) * q;
        if (cm > -1e29f && cp > -1e29f) {
          if (cfg.fit_eq) {
            const float lower = cm < cp ? cm : cp;
            const float den = c0 - lower;
            if (den > 1e-6f) { off = 0.5f * (cp - cm) / den; off = off > 0.5f ? 0.5f : (off < -0.5f ? -0.5f : off); }
          } else {
            const float den = 2.f * c0 - cm - cp;
            if (den > 1e-6f) { off = 0.5f * (cp - cm) / den; off = off > 0.5f ? 0.5f : (off < -0.5f ? -0.5f : off); }
          }
        }
      }
      dl = float(d) + off;
    }
    if (P.disp) P.disp[row + x] = dl;
    float lrc2 = __int_as_float(0x7fc00000);
    float lrc = cfg.lrc ? __int_as_float(0x7fc00000) : kNegBig;
    if (dl == dl) {
      const int xr = x - int(lroundf(dl));
      if (xr >= 0 && xr < W) {
        if (s_rev[xr] >= 0) lrc2 = fabsf(dl - float(dmin + s_rev[xr]));
        if (cfg.lrc && P.rkey) {
          const uint32_t rk = P.rkey[row + xr];
          if (rk) lrc = fabsf(dl - float(dmin + 255 - int(rk & 255u)));
        }
      }
    }
    if (P.lrc2) P.lrc2[row + x] = lrc2;
    const float s1 = n > 0 ? cs2.x : kNegBig;
    const float s2 = n > 1 ? cs2.y : kNegBig;
    if (P.cand) {
      P.cand[row + x] = s1;
      P.cand[WH + row + x] = s2;
      P.cand[2 * WH + row + x] = n > 0 ? float(dmin + s_cd[2 * x]) : kNegBig;
      P.cand[3 * WH + row + x] = n > 1 ? float(dmin + s_cd[2 * x + 1]) : kNegBig;
      P.cand[4 * WH + row + x] = lrc;
      P.cand[5 * WH + row + x] = lrc2;
    }
    if (P.conf) {
      uint8_t cv = 0;
      if (dl == dl)
        cv = uint8_t(lroundf(confidence_dev(s1, s2, lambda, (lrc2 == lrc2) ? lrc2 : 0.f, 1.f) * 255.f));
      P.conf[row + x] = cv;
    }
  };
  // the neighbour words of a thread's pixels, four at a time, loads first
  const bool want_nb = !REF_LAYOUT && cfg.subpixel;
  for (int xb = tid; xb < W; xb += 4 * kSolveThreads) {
    uint32_t nb[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int x = xb + u * kSolveThreads;
      nb[u] = (want_nb && x < W && s_win[x]) ? P.nb[row + x] : 0x80008000u;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (xb + u * kSolveThreads < W) outputs(xb + u * kSolveThreads, nb[u]);
  }
}

// Reference-layout candidates (core/tools/de_dense_cuda.cu:384-390) from packed keys.
__global__ void k_export(DevCfg cfg, Batch b) {
  const int item = blockIdx.x;
  const int pi = find_pair(b.solve_prefix, b.n, item);
  const DevPair& P = b.p[pi];
  const int W = P.W, H = P.H, y = item - b.solve_prefix[pi];
  const bool row_ok = y >= cfg.hh && y < H - cfg.hh;
  const float q = 1.f / 16384.f;
  for (int x = threadIdx.x; x < W; x += blockDim.x) {
    const size_t i = size_t(y) * W + x;
    uint32_t a = 0, bb = 0, nb = 0x80008000u;
    if (row_ok && x >= cfg.hw + cfg.dmin && x < W - cfg.hw) { a = P.key0[i]; bb = P.key1[i]; nb = P.nb[i]; }
    int n = 0;
    P.ref_cs[2 * i] = kNegBig; P.ref_cs[2 * i + 1] = kNegBig;
    P.ref_cd[2 * i] = -1; P.ref_cd[2 * i + 1] = -1;
    if (a) { P.ref_cs[2 * i] = float(int32_t(a >> 8) - 32768) * q; P.ref_cd[2 * i] = 255 - int(a & 255u); n = 1; }
    if (bb) { P.ref_cs[2 * i + 1] = float(int32_t(bb >> 8) - 32768) * q; P.ref_cd[2 * i + 1] = 255 - int(bb & 255u); n = 2; }
    P.ref_cn[i] = n;
    if (P.ref_cnb) {
      P.ref_cnb[2 * i] = int16_t(n && cfg.subpixel ? lo16(nb) : -32768);
      P.ref_cnb[2 * i + 1] = int16_t(n && cfg.subpixel ? hi16(nb) : -32768);
    }
  }
}

size_t rows_smem(const Batch& b, int TS, int G, bool packed, int ring) {
  int cpm = 0, apm = 0, maxW = 0;
  for (int i = 0; i < b.n; ++i) {
    cpm = std::max(cpm, b.p[i].cpitch);
    apm = std::max(apm, b.p[i].apitch);
    maxW = std::max(maxW, b.p[i].W);
  }
  size_t s = size_t(TS) * 64 * 2;
  s += size_t(cpm) * 16;
  s += 2 * ((size_t(apm) * 2 + 127) & ~size_t(127));
  s += size_t(ring) * (kRowsChunk / (64 * G)) * (64 * G) * 2;
  if (!packed) s += size_t(maxW) * 2;
  return (s + 15) & ~size_t(15);
}

size_t solve_smem(int W) { return size_t(W) * 49 + 64; }

template <typename K>
cudaError_t set_smem(K kernel, size_t bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}

}  // namespace

cudaError_t launch_census(const DevCfg& cfg, const Batch& b, cudaStream_t s) {
  const int tiles = b.pix_prefix[b.n];
  if (tiles == 0) return cudaSuccess;
  if ((cfg.hw == 3 || cfg.hw == 4) && cfg.hh == 3) {  // 32 x (8 NR) tiles of its own
    thread_local Batch b2;
    b2 = b;
    b2.pix_prefix[0] = 0;
    for (int i = 0; i < b.n; ++i)
      b2.pix_prefix[i + 1] = b2.pix_prefix[i] + ((b.p[i].W + kCTX - 1) / kCTX) *
                                                    ((b.p[i].H + kC2Y - 1) / kC2Y);
    if (cfg.hw == 3) k_census_rows<3><<<b2.pix_prefix[b.n], dim3(kCTX, kCTY), 0, s>>>(cfg, b2);
    else k_census_rows<4><<<b2.pix_prefix[b.n], dim3(kCTX, kCTY), 0, s>>>(cfg, b2);
  } else {
    k_census_generic<<<tiles, dim3(kCTX, kCTY), 0, s>>>(cfg, b);
  }
  return cudaGetLastError();
}

struct de_cfg_hw { int hw, dmin; };
int g_rows_ctas_per_sm = 32;      // upper bound on row CTAs per SM (rows in flight)
int g_solve_threads = 0;          // threads per row in the solve: 128, 256, 512, 0 = by width
int g_cols_pf = 0;                // rows the column kernel prefetches: 4, 8, 16, 0 = by shape
int g_cols_async = 1;             // 8-row prefetch through shared memory (cp.async)

template <bool PACKED, int TS, int G>
cudaError_t launch_rows_t(const DevCfg& cfg, const Batch& b, cudaStream_t s) {
  auto kern2 = k_rows<PACKED, TS, G, 2>;
  auto kern3 = k_rows<PACKED, TS, G, 3>;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  // rows in flight with two and with three backward stages.  Two only where they put
  // more rows in flight (a batch with fewer rows than the SMs hold either way keeps
  // three), and only at Dpad 64: measured per shape, the extra rows per SM gain 3% at
  // 320x240 D=64 (13 rows per SM instead of 10); at Dpad 128 they gained as one launch
  // set but lose 1.4% on the 848x480 batch once the column kernel leaves room for the
  // other launch set's rows (seven rows per SM are better there), and at Dpad 256
  // they lose 1-2%.  The occupancy of each footprint is looked up once per kernel and
  // size.
  struct Occ { const void* k; size_t sm; int fit; };
  thread_local std::vector<Occ> occ_cache;
  auto fit_of = [&](auto kern, size_t sm) -> int {
    for (const Occ& o : occ_cache)
      if (o.k == reinterpret_cast<const void*>(kern) && o.sm == sm) return o.fit;
    int fit = 0;
    if (set_smem(kern, sm) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, kern, 32 * G, sm) != cudaSuccess) {
      cudaGetLastError();
      fit = 1;
    }
    if (occ_cache.size() > 64) occ_cache.clear();
    occ_cache.push_back({reinterpret_cast<const void*>(kern), sm, fit});
    return fit;
  };
  const size_t sm2 = rows_smem(b, TS, G, PACKED, 2), sm3 = rows_smem(b, TS, G, PACKED, 3);
  const int per2 = std::max(1, std::min(fit_of(kern2, sm2), g_rows_ctas_per_sm));
  const int per3 = std::max(1, std::min(fit_of(kern3, sm3), g_rows_ctas_per_sm));
  const int items = b.rows_prefix[b.n];
  cudaError_t e;
  if (G == 1 && std::min(items, per2 * nsm) > std::min(items, per3 * nsm)) {
    if ((e = set_smem(kern2, sm2)) != cudaSuccess) return e;
    kern2<<<std::min(items, per2 * nsm), 32 * G, sm2, s>>>(cfg, b);
  } else {
    if ((e = set_smem(kern3, sm3)) != cudaSuccess) return e;
    kern3<<<std::min(items, per3 * nsm), 32 * G, sm3, s>>>(cfg, b);
  }
  return cudaGetLastError();
}

template <int G>
cudaError_t launch_rows_g(const DevCfg& cfg, const Batch& b, cudaStream_t s) {
  const int TS = cfg.trunc < 16 ? 16 : 256;
  if (cfg.packed)
    return TS == 16 ? launch_rows_t<true, 16, G>(cfg, b, s) : launch_rows_t<true, 256, G>(cfg, b, s);
  return TS == 16 ? launch_rows_t<false, 16, G>(cfg, b, s) : launch_rows_t<false, 256, G>(cfg, b, s);
}

// One launch per disparity group present in the batch (Dpad = 64 G).
cudaError_t launch_rows(const DevCfg& cfg, const Batch& b, cudaStream_t s) {
  if (b.rows_prefix[b.n] == 0) return cudaSuccess;
  thread_local Batch sub;
  for (int G = 1; G <= 4; ++G) {
    sub = b;
    sub.n = 0;
    sub.rows_prefix[0] = 0;
    sub.maxDpad = 64 * G;
    for (int i = 0; i < b.n; ++i) {
      if (b.p[i].Dpad != 64 * G) continue;
      sub.p[sub.n] = b.p[i];
      sub.rows_prefix[sub.n + 1] = sub.rows_prefix[sub.n] + (b.rows_prefix[i + 1] - b.rows_prefix[i]);
      ++sub.n;
    }
    if (sub.n == 0 || sub.rows_prefix[sub.n] == 0) continue;
    cudaError_t e;
    switch (G) {
      case 1: e = launch_rows_g<1>(cfg, sub, s); break;
      case 2: e = launch_rows_g<2>(cfg, sub, s); break;
      case 3: e = launch_rows_g<3>(cfg, sub, s); break;
      default: e = launch_rows_g<4>(cfg, sub, s); break;
    }
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

void set_solve_threads(int v) { g_solve_threads = (v == 128 || v == 256 || v == 512) ? v : 0; }
int get_solve_threads() { return g_solve_threads; }
void set_rows_ctas_per_sm(int v) { g_rows_ctas_per_sm = v < 1 ? 1 : v; }
int get_rows_ctas_per_sm() { return g_rows_ctas_per_sm; }

template <int KT, int TPCP, int NT>
cudaError_t launch_cols_nt(const DevCfg& cfg, const Batch& b0, const de_cfg_hw& hwc,
                           cudaStream_t s) {
  constexpr int NCOL = NT / TPCP;
  thread_local Batch b;                               // tiles instead of columns
  b = b0;
  b.cols_prefix[0] = 0;
  for (int i = 0; i < b.n; ++i) {
    const int ncols = std::max(0, b.p[i].W - 2 * hwc.hw - hwc.dmin);
    b.cols_prefix[i + 1] = b.cols_prefix[i] + (ncols + NCOL - 1) / NCOL;
  }
  const int tiles = b.cols_prefix[b.n];
  if (tiles == 0) return cudaSuccess;
  // PF = 16 at 4 disparities per lane; 8 where the ring still fits the register
  // budget; else 4
  const int pf = g_cols_pf ? g_cols_pf : (KT == 4 ? 16 : 8);
  if constexpr (KT == 4) {
    if (pf == 16) {
      k_cols<KT, TPCP, 16, NT><<<tiles, NT, 0, s>>>(cfg, b);
      return cudaGetLastError();
    }
  }
  if constexpr (KT == 8) {
    if (pf >= 8 && cfg.cols_async) {                  // the ring in shared memory
      constexpr size_t ring_bytes = size_t(NT) * 8 * (KT / 2) * 4;
      const cudaError_t e = set_smem(k_cols<KT, TPCP, 8, NT, true>, ring_bytes);
      if (e != cudaSuccess) return e;
      k_cols<KT, TPCP, 8, NT, true><<<tiles, NT, ring_bytes, s>>>(cfg, b);
      return cudaGetLastError();
    }
  }
  if constexpr (KT == 4 || (KT == 8 && TPCP <= 16)) {
    if (pf >= 8) {
      k_cols<KT, TPCP, 8, NT><<<tiles, NT, 0, s>>>(cfg, b);
      return cudaGetLastError();
    }
  }
  k_cols<KT, TPCP, 4, NT><<<tiles, NT, 0, s>>>(cfg, b);
  return cudaGetLastError();
}

int g_cols_cta = 0;               // column-kernel CTA threads: 128, 256, or 0 = by shape
void set_cols_cta(int v) { g_cols_cta = (v == 128 || v == 256) ? v : 0; }
int get_cols_cta() { return g_cols_cta; }

// CTA size: 128 threads while the batch is too small to give every SM several
// 256-thread tiles (finer tiles spread the column groups over more SMs), else 256.
template <int KT, int TPCP>
cudaError_t launch_cols_t(const DevCfg& cfg, const Batch& b, const de_cfg_hw& hwc,
                          cudaStream_t s, long work) {
  const int nt = g_cols_cta ? g_cols_cta : (work < 148L * 32 * 16 * 8 ? 128 : 256);
  if (nt == 128) return launch_cols_nt<KT, TPCP, 128>(cfg, b, hwc, s);
  return launch_cols_nt<KT, TPCP, 256>(cfg, b, hwc, s);
}

int g_expire_polls = 0;
void set_expire_polls(int v) { g_expire_polls = v < 0 ? 0 : (v > (1 << 20) ? (1 << 20) : v); }
int get_expire_polls() { return g_expire_polls; }

void set_cols_pf(int v) { g_cols_pf = (v == 4 || v == 8 || v == 16) ? v : 0; }
void set_cols_async(int v) { g_cols_async = v ? 1 : 0; }
int get_cols_async() { return g_cols_async; }
int get_cols_pf() { return g_cols_pf; }

int g_cols_kt = 0;                // 0 = by batch size, else 4, 8 or 16 disparities per lane
void set_cols_kt(int v) { g_cols_kt = (v == 4 || v == 8 || v == 16) ? v : 0; }
int get_cols_kt() { return g_cols_kt; }

// Disparities per lane KT; lanes per column Dpad/KT rounded up to a power of two.
// By default KT = 4 for batches too small to fill the GPU with columns (one column
// per warp, the most columns in flight), else KT = 8.  KT = 4 needs Dpad <= 128 (32
// lanes), KT = 16 needs Dpad >= 128.  `b` holds pairs of one disparity group.
cudaError_t launch_cols_g(const DevCfg& cfg, const Batch& b, cudaStream_t s) {
  if (b.cols_prefix[b.n] == 0) return cudaSuccess;
  const de_cfg_hw hwc{cfg.hw, cfg.dmin};
  const long work = long(b.cols_prefix[b.n]) * b.maxDpad;
  const int maxDpad = b.maxDpad;
  int kt = g_cols_kt ? g_cols_kt : (work < 148L * 32 * 16 * 4 ? 4 : 8);
  if (kt == 4 && maxDpad > 128) kt = 8;
  if (kt == 16 && maxDpad <= 64) kt = 8;
  if (kt == 4) {
    if (maxDpad <= 64) return launch_cols_t<4, 16>(cfg, b, hwc, s, work);
    return launch_cols_t<4, 32>(cfg, b, hwc, s, work);
  }
  if (kt == 8) {
    switch (maxDpad) {
      case 64: return launch_cols_t<8, 8>(cfg, b, hwc, s, work);
      case 128: return launch_cols_t<8, 16>(cfg, b, hwc, s, work);
      default: return launch_cols_t<8, 32>(cfg, b, hwc, s, work);
    }
  }
  switch (maxDpad) {
    case 128: return launch_cols_t<16, 8>(cfg, b, hwc, s, work);
    default: return launch_cols_t<16, 16>(cfg, b, hwc, s, work);
  }
}

// One launch per disparity group present in the batch (Dpad = 64 G), so a pair's
// column groups are sized for its own Dpad rather than the batch's largest, and each
// group picks its tile shape from its own work.
cudaError_t launch_cols(const DevCfg& cfg, const Batch& b, cudaStream_t s) {
  if (b.cols_prefix[b.n] == 0) return cudaSuccess;
  thread_local Batch sub;
  for (int G = 1; G <= 4; ++G) {
    sub = b;
    sub.n = 0;
    sub.cols_prefix[0] = 0;
    sub.maxDpad = 64 * G;
    for (int i = 0; i < b.n; ++i) {
      if (b.p[i].Dpad != 64 * G) continue;
      sub.p[sub.n] = b.p[i];
      sub.cols_prefix[sub.n + 1] = sub.cols_prefix[sub.n] + (b.cols_prefix[i + 1] - b.cols_prefix[i]);
      ++sub.n;
    }
    if (sub.n == 0) continue;
    const cudaError_t e = launch_cols_g(cfg, sub, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// `b` holds pairs of one width class.  Shared memory is sized for the class's widest
// row; threads per row come from the knob, or by width (512 above 1024 pixels, else
// 256).
cudaError_t launch_solve_w(const DevCfg& cfg, const Batch& b, bool from_ref, cudaStream_t s) {
  const int items = b.solve_prefix[b.n];
  if (items == 0) return cudaSuccess;
  int maxW = 0;
  for (int i = 0; i < b.n; ++i) maxW = maxW > b.p[i].W ? maxW : b.p[i].W;
  const size_t sm = solve_smem(maxW);
  cudaError_t e;
  auto go = [&](auto kern, int nt) -> cudaError_t {
    cudaError_t e2 = set_smem(kern, sm);
    if (e2 != cudaSuccess) return e2;
    kern<<<items, nt, sm, s>>>(cfg, b);
    return cudaSuccess;
  };
  const int nt = g_solve_threads ? g_solve_threads : (maxW > 1024 ? 512 : 256);
  switch (nt) {
    case 128: e = from_ref ? go(k_solve<true, 128>, 128) : go(k_solve<false, 128>, 128); break;
    case 512: e = from_ref ? go(k_solve<true, 512>, 512) : go(k_solve<false, 512>, 512); break;
    default: e = from_ref ? go(k_solve<true, 256>, 256) : go(k_solve<false, 256>, 256); break;
  }
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

// One launch per width class (up to 512, up to 1024, wider): the shared-memory
// working set grows with the row, so a narrow pair launched beside a wide one would
// run at the wide pair's occupancy.
cudaError_t launch_solve(const DevCfg& cfg, const Batch& b, bool from_ref, cudaStream_t s) {
  if (b.solve_prefix[b.n] == 0) return cudaSuccess;
  thread_local Batch sub;
  constexpr int kLimit[3] = {512, 1024, 1 << 30};
  for (int c = 0; c < 3; ++c) {
    const int lo = c ? kLimit[c - 1] : 0;
    sub = b;
    sub.n = 0;
    sub.solve_prefix[0] = 0;
    for (int i = 0; i < b.n; ++i) {
      if (b.p[i].W <= lo || b.p[i].W > kLimit[c]) continue;
      sub.p[sub.n] = b.p[i];
      sub.solve_prefix[sub.n + 1] = sub.solve_prefix[sub.n] + (b.solve_prefix[i + 1] - b.solve_prefix[i]);
      ++sub.n;
    }
    if (sub.n == 0) continue;
    const cudaError_t e = launch_solve_w(cfg, sub, from_ref, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_export_candidates(const DevCfg& cfg, const Batch& b, cudaStream_t s) {
  const int items = b.solve_prefix[b.n];
  if (items == 0) return cudaSuccess;
  k_export<<<items, 256, 0, s>>>(cfg, b);
  return cudaGetLastError();
}

}  // namespace de
