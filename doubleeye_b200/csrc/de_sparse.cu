// Sparse (keypoint) path: census at keypoints, the FAST + Shi-Tomasi detector,
// and keypoint MASDA (candidate graph, max-sum message passing, decision).
//
//   census_at              core/src/preproc.cpp:142-162
//   detect_keypoints_fast  core/src/preproc.cpp:442-545 (is_fast_corner :373-400,
//                          shi_tomasi_at :402-432, local_std_at :164-182)
//   match_masda            core/src/match.cpp:334-417 (build_candidates :46-102,
//                          pair_score :298-332, row_margins :112-132, emit :134-231)
//
// The reference is sequential C++.  Here:
//   * the detector is one pass over pixels (corner test + response), then the
//     greedy strongest-first suppression resolved per candidate (a point is kept
//     iff none of its stronger neighbours is kept, settled depth first by any thread
//     that needs it), which yields exactly the sequential result; then one CTA per
//     grid cell refines its survivors and keeps the strongest per_cell.
//   * one CTA solves one matching problem end to end: y-sort of the right points
//     (bitonic, shared memory), candidate rows (one thread per left point), CSR/CSC
//     edge lists, the damped rho/beta sweeps, margins, the mutual-best pass and the
//     greedy completion (rounds of edges that are the strongest remaining option of
//     both their row and their column, which is again exactly the sequential greedy).
// Float arithmetic follows the reference's operation order without contraction
// (the library is built with --fmad=false), so results are bit-identical to the
// reference wherever its sort order is defined; exact ties between equal keys are
// broken by input position (the reference's std::sort leaves them unspecified).

#include <algorithm>
#include <cstdint>
#include <cstring>

#include <cuda_runtime.h>

#include "de_internal.h"

namespace de {
namespace {

constexpr float kNegBig = -1e30f;
constexpr int kSortMax = 16384;          // right keypoints per problem (shared-memory sort)
constexpr int kMaxCell = 128;            // detector grid cell edge

__device__ __forceinline__ float fmax_ref(float a, float b) { return (a < b) ? b : a; }

// ---------------------------------------------------------------------------------
// census_at for a list of keypoints at int(x + 0.5), int(y + 0.5) (the rounding of
// core/tools/de_match.cpp:230 and core/src/match.cpp:604-611).
__global__ void k_census_at(const uint8_t* __restrict__ img, int W, int H,
                            const de_keypoint* __restrict__ kp, int n, const int* n_dev,
                            int hw, int hh, uint64_t* desc, uint8_t* ok) {
  const int cnt = n_dev ? min(n, *n_dev) : n;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cnt) return;
  const int x = int(kp[t].x + 0.5f), y = int(kp[t].y + 0.5f);
  const bool inside = x >= hw && y >= hh && x < W - hw && y < H - hh;
  uint64_t v = 0;
  if (inside) {
    const int c = __ldg(img + size_t(y) * W + x);
    int b = 0;
    for (int dy = -hh; dy <= hh; ++dy) {
      const uint8_t* row = img + size_t(y + dy) * W + x;
      for (int dx = -hw; dx <= hw; ++dx) {
        if (dx == 0 && dy == 0) continue;
        if (int(__ldg(row + dx)) < c) v |= 1ull << b;
        ++b;
      }
    }
  }
  desc[t] = v;
  if (ok) ok[t] = inside ? 1 : 0;
}

// ---------------------------------------------------------------------------------
// Detector.

__device__ __forceinline__ bool run9(unsigned m) {
  const unsigned t = m | (m << 16);
  unsigned r = t & (t >> 1);         // runs of 2
  r &= r >> 2;                       // runs of 4
  r &= r >> 4;                       // runs of 8
  r &= t >> 8;                       // runs of 9
  return (r & 0xFFFFu) != 0;
}

// is_fast_corner for an interior pixel (3 <= x < W-3, 3 <= y < H-3).
__device__ bool fast_corner(const uint8_t* __restrict__ img, int W, int x, int y, int thr) {
  // radius-3 Bresenham ring from the top, clockwise (core/src/preproc.cpp:356-357)
  constexpr int kRingX[16] = {0, 1, 2, 3, 3, 3, 2, 1, 0, -1, -2, -3, -3, -3, -2, -1};
  constexpr int kRingY[16] = {-3, -3, -2, -1, 0, 1, 2, 3, 3, 3, 2, 1, 0, -1, -2, -3};
  const uint8_t* p = img + size_t(y) * W + x;
  const int c = __ldg(p);
  const int hi = c + thr, lo = c - thr;
  int v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __ldg(p + kRingY[k] * W + kRingX[k]);
  int bright = 0, dark = 0;
#pragma unroll
  for (int k = 0; k < 16; k += 4) {
    bright += v[k] > hi;
    dark += (v[k] <= hi) & (v[k] < lo);
  }
  if (bright < 2 && dark < 2) return false;
  unsigned bm = 0, dm = 0;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    bm |= unsigned(v[k] > hi) << k;
    dm |= unsigned(v[k] <= hi && v[k] < lo) << k;
  }
  return run9(bm) || run9(dm);
}

// shi_tomasi_at, same operation order (every partial sum is exact in float).
__device__ float shi_tomasi(const uint8_t* __restrict__ img, int W, int H, int x, int y,
                            int gw) {
  const int r = max(1, gw / 2);
  if (x - r - 1 < 0 || y - r - 1 < 0 || x + r + 1 >= W || y + r + 1 >= H) return 0.f;
  float sxx = 0.f, syy = 0.f, sxy = 0.f;
  for (int dy = -r; dy <= r; ++dy)
    for (int dx = -r; dx <= r; ++dx) {
      const int px = x + dx, py = y + dy;
      const uint8_t* rm = img + size_t(py - 1) * W;
      const uint8_t* r0 = img + size_t(py) * W;
      const uint8_t* rp = img + size_t(py + 1) * W;
      const float gx = (float(__ldg(rm + px + 1)) - float(__ldg(rm + px - 1)) +
                        2.f * (float(__ldg(r0 + px + 1)) - float(__ldg(r0 + px - 1))) +
                        float(__ldg(rp + px + 1)) - float(__ldg(rp + px - 1))) * 0.125f;
      const float gy = (float(__ldg(rp + px - 1)) - float(__ldg(rm + px - 1)) +
                        2.f * (float(__ldg(rp + px)) - float(__ldg(rm + px))) +
                        float(__ldg(rp + px + 1)) - float(__ldg(rm + px + 1))) * 0.125f;
      sxx += gx * gx;
      syy += gy * gy;
      sxy += gx * gy;
    }
  const float n = 1.f / float((2 * r + 1) * (2 * r + 1));
  const float a = sxx * n, b = syy * n, c = sxy * n;
  const float half_tr = 0.5f * (a + b);
  const float disc = sqrtf(fmax_ref(0.f, 0.25f * (a - b) * (a - b) + c * c));
  return half_tr - disc;
}

// local_std_at over a 7x7 window clamped to the image: integer sums (exact, as the
// reference's double sums are), then the reference's double-precision moments.
__device__ float local_std7(const uint8_t* __restrict__ img, int W, int H, int x, int y) {
  const int x0 = max(0, x - 3), x1 = min(W - 1, x + 3);
  const int y0 = max(0, y - 3), y1 = min(H - 1, y + 3);
  int s1 = 0, s2 = 0;
  for (int yy = y0; yy <= y1; ++yy)
    for (int xx = x0; xx <= x1; ++xx) {
      const int v = __ldg(img + size_t(yy) * W + xx);
      s1 += v;
      s2 += v * v;
    }
  const double n = double((y1 - y0 + 1) * (x1 - x0 + 1));
  const double mean = double(s1) / n;
  const double var = double(s2) / n - mean * mean;
  return var > 0.0 ? float(sqrt(var)) : 0.f;
}

// Detector workspace, carved from one caller allocation.
struct DetWs {
  float* resp;        // [H*W] response at candidates
  uint8_t* state;     // [H*W + 32] 0 none, 1 undecided, 2 kept, 3 suppressed
  int* listA;         // [H*W] candidate pixel indices
  int* listB;         // [H*W]
  int* counters;      // [0] candidates, [1] error
  de_keypoint* slot;  // [cells * keep]
  int* cellcnt;       // [cells]
};

size_t det_ws_bytes(int W, int H, int cells, int keep) {
  const size_t px = size_t(W) * H;
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  return up(px * 4) + up(px + 32) + 2 * up(px * 4) + up(64) + up(size_t(cells) * keep * 16) +
         up(size_t(cells) * 4);
}

DetWs carve_det(void* ws, int W, int H, int cells, int keep) {
  const size_t px = size_t(W) * H;
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  uint8_t* p = static_cast<uint8_t*>(ws);
  DetWs d;
  d.resp = reinterpret_cast<float*>(p);           p += up(px * 4);
  d.state = p;                                    p += up(px + 32);   // word reads past the end
  d.listA = reinterpret_cast<int*>(p);            p += up(px * 4);
  d.listB = reinterpret_cast<int*>(p);            p += up(px * 4);
  d.counters = reinterpret_cast<int*>(p);         p += up(64);
  d.slot = reinterpret_cast<de_keypoint*>(p);     p += up(size_t(cells) * keep * 16);
  d.cellcnt = reinterpret_cast<int*>(p);
  return d;
}

// Stage 1: FAST + response at every pixel of the search window; writes the state
// of every pixel and appends candidates (order irrelevant: later stages use the
// total order response desc, then pixel index).
__global__ void k_fast(const uint8_t* __restrict__ img, int W, int H, int border, int thr,
                       int gw, float min_response, DetWs d) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  bool is_cand = false;
  float r = 0.f;
  if (x < W && y < H) {
    if (x >= border && x < W - border && y >= border && y < H - border &&
        fast_corner(img, W, x, y, thr)) {
      r = shi_tomasi(img, W, H, x, y, gw);
      is_cand = !(r < min_response);
    }
    const size_t i = size_t(y) * W + x;
    d.state[i] = is_cand ? 1 : 0;
    if (is_cand) d.resp[i] = r;
  }
  const unsigned ballot = __ballot_sync(0xffffffffu, is_cand);
  if (!ballot) return;
  const int lane = threadIdx.x + threadIdx.y * blockDim.x & 31;
  int base = 0;
  if (lane == __ffs(ballot) - 1) base = atomicAdd(&d.counters[0], __popc(ballot));
  base = __shfl_sync(0xffffffffu, base, __ffs(ballot) - 1);
  if (is_cand) d.listA[base + __popc(ballot & ((1u << lane) - 1u))] = y * W + x;
}

// Stage 2: greedy suppression, strongest first.  The sequential rule (keep a point
// unless an already kept, stronger point lies in its square) makes a point's fate a
// function of the fates of its stronger neighbours only: kept iff none of them is
// kept.  Each thread settles one candidate by resolving undecided stronger
// neighbours depth first and records every settled fate in the state map.  Threads
// never wait for one another: one that reads a stale "undecided" recomputes that
// fate itself and necessarily reaches the same value, so concurrent writes agree.
constexpr int kNmsStack = 32;
constexpr int kNmsGuard = 1 << 22;       // visits per thread before it gives up

__device__ __forceinline__ bool stronger(float rj, int j, float r, int i) {
  return rj > r || (rj == r && j < i);    // response desc, then scan order
}

__global__ void __launch_bounds__(256) k_nms(int W, int H, int rad, DetWs d) {
  const int n = d.counters[0];
  volatile uint8_t* st = d.state;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int root = d.listA[q];
    int stack[kNmsStack];
    int guard = 0;
    while (st[root] == 1) {
      int sp = 0;
      stack[sp++] = root;
      while (sp > 0) {
        if (++guard > kNmsGuard) {
          d.counters[1] = 1;
          return;
        }
        const int t = stack[sp - 1];
        if (st[t] != 1) { --sp; continue; }
        const int x = t % W, y = t / W;
        const float r = d.resp[t];
        bool supp = false;
        int pend = -1;
        for (int dy = -rad; dy <= rad && !supp; ++dy) {
          const int py = y + dy;
          if (py < 0 || py >= H) continue;
          for (int dx = -rad; dx <= rad; ++dx) {
            const int px = x + dx;
            if (px < 0 || px >= W) continue;
            const int j = py * W + px;
            const int s = st[j];
            if (s == 0 || s == 3 || j == t) continue;
            if (!stronger(d.resp[j], j, r, t)) continue;
            if (s == 2) { supp = true; break; }
            pend = j;
          }
        }
        if (supp) { st[t] = 3; --sp; continue; }
        if (pend < 0) { st[t] = 2; --sp; continue; }
        if (sp == kNmsStack) {              // keep the deeper half; the rest is redone
#pragma unroll
          for (int k = 0; k < kNmsStack / 2; ++k) stack[k] = stack[k + kNmsStack / 2];
          sp = kNmsStack / 2;
        }
        stack[sp++] = pend;
      }
    }
  }
}

// The same suppression for radii up to RM with the window's states fetched first:
// each window row's bytes arrive as aligned 32-bit words, all rows' loads issued
// before any is used, so a visit costs one round trip for the states plus one per
// candidate neighbour's response, instead of one per window pixel.  The visit's
// logic (scan order, the pending neighbour chosen, the guard) is k_nms's.
template <int RM>
__global__ void __launch_bounds__(256) k_nms_w(int W, int H, int rad, DetWs d) {
  constexpr int NR = 2 * RM + 1;                      // window rows
  constexpr int NW = (2 * RM + 1 + 3) / 4;            // aligned words of a row segment
  const int n = d.counters[0];
  volatile uint8_t* st = d.state;
  const volatile uint32_t* stw = reinterpret_cast<const volatile uint32_t*>(d.state);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int root = d.listA[q];
    int stack[kNmsStack];
    int guard = 0;
    while (st[root] == 1) {
      int sp = 0;
      stack[sp++] = root;
      while (sp > 0) {
        if (++guard > kNmsGuard) {
          d.counters[1] = 1;
          return;
        }
        const int t = stack[sp - 1];
        if (st[t] != 1) { --sp; continue; }
        const int x = t % W, y = t / W;
        const int x0 = max(x - rad, 0), x1 = min(x + rad, W - 1);
        const float r = d.resp[t];
        uint32_t seg[NR][NW];                         // byte i of row a: pixel x0 + i
#pragma unroll
        for (int a = 0; a < NR; ++a) {
          const int py = y - RM + a;
          const bool ok = a >= RM - rad && a <= RM + rad && py >= 0 && py < H;
          const size_t b0 = size_t(ok ? py : y) * W + x0;
          const size_t w0 = b0 >> 2;
          uint32_t w[NW + 1];
#pragma unroll
          for (int k = 0; k <= NW; ++k) w[k] = stw[w0 + k];
          const uint32_t sel = 0x3210u + 0x1111u * uint32_t(b0 & 3);
#pragma unroll
          for (int k = 0; k < NW; ++k) seg[a][k] = ok ? __byte_perm(w[k], w[k + 1], sel) : 0u;
        }
        bool supp = false;
        int pend = -1;
#pragma unroll
        for (int a = 0; a < NR; ++a) {
          const int py = y - RM + a;
#pragma unroll
          for (int i = 0; i < 2 * RM + 1; ++i) {
            if (supp || x0 + i > x1) continue;
            const int s = int((seg[a][i >> 2] >> (8 * (i & 3))) & 0xFFu);
            const int j = py * W + x0 + i;
            if (s == 0 || s == 3 || j == t) continue;
            if (!stronger(d.resp[j], j, r, t)) continue;
            if (s == 2) supp = true;
            else pend = j;
          }
        }
        if (supp) { st[t] = 3; --sp; continue; }
        if (pend < 0) { st[t] = 2; --sp; continue; }
        if (sp == kNmsStack) {              // keep the deeper half; the rest is redone
#pragma unroll
          for (int k = 0; k < kNmsStack / 2; ++k) stack[k] = stack[k + kNmsStack / 2];
          sp = kNmsStack / 2;
        }
        stack[sp++] = pend;
      }
    }
  }
}

// Stage 3: one CTA per grid cell.  Texture floor, sub-pixel, strongest per_cell.
__global__ void __launch_bounds__(256) k_cells(const uint8_t* __restrict__ img, int W, int H,
                                               int cell, int cols, int keep, int gw,
                                               float min_std, int subpixel, DetWs d) {
  extern __shared__ __align__(16) uint8_t smem[];
  de_keypoint* kp = reinterpret_cast<de_keypoint*>(smem);
  const int cap = ((cell + 1) / 2) * ((cell + 1) / 2);
  int* idx = reinterpret_cast<int*>(kp + cap);
  __shared__ int s_n;
  const int c = blockIdx.x;
  const int x0 = (c % cols) * cell, y0 = (c / cols) * cell;
  const int x1 = min(W, x0 + cell), y1 = min(H, y0 + cell);
  const int cw = x1 - x0;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  for (int t = threadIdx.x; t < cw * (y1 - y0); t += blockDim.x) {
    const int xi = x0 + t % cw, yi = y0 + t / cw;
    const size_t i = size_t(yi) * W + xi;
    if (d.state[i] != 2) continue;
    de_keypoint k;
    k.x = float(xi);
    k.y = float(yi);
    k.response = d.resp[i];
    k.local_std = local_std7(img, W, H, xi, yi);
    if (k.local_std < min_std) continue;
    if (subpixel) {
      const float cc = k.response;
      const float l = shi_tomasi(img, W, H, xi - 1, yi, gw);
      const float r = shi_tomasi(img, W, H, xi + 1, yi, gw);
      const float dxx = l - 2.f * cc + r;
      if (fabsf(dxx) > 1e-12f) {
        const float dd = 0.5f * (l - r) / dxx;
        if (fabsf(dd) <= 0.5f) k.x += dd;
      }
      const float u = shi_tomasi(img, W, H, xi, yi - 1, gw);
      const float dn = shi_tomasi(img, W, H, xi, yi + 1, gw);
      const float dyy = u - 2.f * cc + dn;
      if (fabsf(dyy) > 1e-12f) {
        const float dd = 0.5f * (u - dn) / dyy;
        if (fabsf(dd) <= 0.5f) k.y += dd;
      }
    }
    const int q = atomicAdd(&s_n, 1);
    if (q < cap) {            // kept points are >= 2 apart, so q < cap always
      kp[q] = k;
      idx[q] = int(i);
    }
  }
  __syncthreads();
  const int n = min(s_n, cap);
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    const float r = kp[q].response;
    const int iq = idx[q];
    int rank = 0;
    for (int o = 0; o < n; ++o) {
      const float ro = kp[o].response;
      rank += (ro > r || (ro == r && idx[o] < iq)) ? 1 : 0;
    }
    if (rank < keep) d.slot[size_t(c) * keep + rank] = kp[q];
  }
  if (threadIdx.x == 0) d.cellcnt[c] = min(n, keep);
}

// Exclusive scan of a[0..n) (global memory) by one CTA of NT threads; returns total.
template <int NT>
__device__ int cta_excl_scan(int* a, int n, int* warp_sums) {
  const int tid = threadIdx.x;
  const int per = (n + NT - 1) / NT;
  const int lo = min(n, tid * per), hi = min(n, lo + per);
  int s = 0;
  for (int i = lo; i < hi; ++i) s += a[i];
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
    int ws = lane < NT / 32 ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, ws, o);
      if (lane >= o) ws += u;
    }
    if (lane < NT / 32) warp_sums[lane] = ws;
  }
  __syncthreads();
  int run = v - s + (w > 0 ? warp_sums[w - 1] : 0);
  for (int i = lo; i < hi; ++i) {
    const int c = a[i];
    a[i] = run;
    run += c;
  }
  const int total = warp_sums[NT / 32 - 1];
  __syncthreads();
  return total;
}

// Stage 4: cells in row-major order, each cell's kept points in strength order.
__global__ void __launch_bounds__(1024) k_det_emit(int cells, int keep, DetWs d,
                                                  de_keypoint* out, int cap, int* n_out) {
  __shared__ int warp_sums[32];
  const int total = cta_excl_scan<1024>(d.cellcnt, cells, warp_sums);
  __syncthreads();
  for (int c = threadIdx.x; c < cells; c += blockDim.x) {
    const int base = d.cellcnt[c];
    const int cnt = (c + 1 < cells ? d.cellcnt[c + 1] : total) - base;
    for (int k = 0; k < cnt; ++k)
      if (base + k < cap) out[base + k] = d.slot[size_t(c) * keep + k];
  }
  if (threadIdx.x == 0) {
    *n_out = total;
    if (d.counters[1]) *n_out = -1;
  }
}

// ---------------------------------------------------------------------------------
// Keypoint MASDA: one CTA of 1024 threads per problem.

struct MatchWs {
  int* cnt;          // [nl + 1] candidates per left point, then row offsets
  int* slot_j;       // [nl * maxc]
  float* slot_s;     // [nl * maxc]
  int* order;        // [nr] right points in (y, index) order
  int* ei;           // [E] edge lists in the reference's edge order
  int* ej;
  float* es;
  float* beta;
  float* rho;
  float* belief;
  int* cstart;       // [nr + 1] column offsets
  int* cfill;        // [nr]
  int* citems;       // [E]
  int* best_row;     // [nl]
  int* best_col;     // [nr]
  float* margin;     // [nl]
  uint8_t* rt;       // [nl]
  uint8_t* ct;       // [nr]
  int* rbest;        // [nl]
  int* cbest;        // [nr]
  int* acc;          // [nl] pass-2 accepted edges
  int* flag;         // [nl + 1] pass-1 accepts, then output offsets
};

__host__ __device__ inline size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

size_t match_ws_bytes(int nl, int nr, int maxc) {
  const size_t E = size_t(nl) * maxc;
  const size_t L = size_t(nl) + 1, R = size_t(nr) + 1;
  return up256(L * 4) + up256(E * 4) * 2 + up256(R * 4) + up256(E * 4) * 6 + up256(R * 4) * 2 +
         up256(E * 4) + up256(L * 4) + up256(R * 4) + up256(L * 4) + up256(L) + up256(R) +
         up256(L * 4) + up256(R * 4) + up256(L * 4) + up256(L * 4);
}

MatchWs carve_match(void* ws, int nl, int nr, int maxc) {
  const size_t E = size_t(nl) * maxc;
  const size_t L = size_t(nl) + 1, R = size_t(nr) + 1;
  uint8_t* p = static_cast<uint8_t*>(ws);
  auto take = [&](size_t b) { uint8_t* q = p; p += up256(b); return q; };
  MatchWs m;
  m.cnt = reinterpret_cast<int*>(take(L * 4));
  m.slot_j = reinterpret_cast<int*>(take(E * 4));
  m.slot_s = reinterpret_cast<float*>(take(E * 4));
  m.order = reinterpret_cast<int*>(take(R * 4));
  m.ei = reinterpret_cast<int*>(take(E * 4));
  m.ej = reinterpret_cast<int*>(take(E * 4));
  m.es = reinterpret_cast<float*>(take(E * 4));
  m.beta = reinterpret_cast<float*>(take(E * 4));
  m.rho = reinterpret_cast<float*>(take(E * 4));
  m.belief = reinterpret_cast<float*>(take(E * 4));
  m.cstart = reinterpret_cast<int*>(take(R * 4));
  m.cfill = reinterpret_cast<int*>(take(R * 4));
  m.citems = reinterpret_cast<int*>(take(E * 4));
  m.best_row = reinterpret_cast<int*>(take(L * 4));
  m.best_col = reinterpret_cast<int*>(take(R * 4));
  m.margin = reinterpret_cast<float*>(take(L * 4));
  m.rt = take(L);
  m.ct = take(R);
  m.rbest = reinterpret_cast<int*>(take(L * 4));
  m.cbest = reinterpret_cast<int*>(take(R * 4));
  m.acc = reinterpret_cast<int*>(take(L * 4));
  m.flag = reinterpret_cast<int*>(take(L * 4));
  return m;
}

struct MatchArgs {
  const de_keypoint* kl;
  const uint64_t* dl;
  const de_keypoint* kr;
  const uint64_t* dr;
  int nl_cap, nr_cap;     // host-side sizes
  const int* nl_dev;      // optional device counts (<= caps; negative = 0)
  const int* nr_dev;
  de_match* out;
  int cap;
  int* n_out;
  de_match_stats* stats;
  float max_dy, min_disp, max_disp, sigma_y, w_y, damping, lambda, gamma, eps;
  int maxc, iters, census_bits;
  int smem_bytes;         // dynamic shared memory of the launch
  de_match_prior prior;   // soft disparity priors per left keypoint (arrays may be null)
};

__device__ __forceinline__ uint32_t ord_f32(float v) {   // order-preserving bits
  const uint32_t b = __float_as_uint(v);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// pair_score, core/src/match.cpp:298-332: descriptor agreement minus the y-residual
// penalty, minus each soft disparity prior's penalty where left keypoint i has one
// (sigma > 0), in the reference's order of operations.
__device__ __forceinline__ float pair_score(const de_keypoint& l, const de_keypoint& r,
                                            uint64_t dl, uint64_t dr, const MatchArgs& a,
                                            int i) {
  const float half = 0.5f * float(a.census_bits);
  const float desc = (half - float(__popcll(dl ^ dr))) / half;
  const float dy = (l.y - r.y) / (a.sigma_y > 0 ? a.sigma_y : 1.f);
  float score = desc - a.w_y * dy * dy;
  const de_match_prior& p = a.prior;
  if (p.coarse_sd) {
    const float sd = p.coarse_sd[i];
    if (sd > 0.f) {
      const float e = ((l.x - r.x) - p.coarse_d[i]) / sd;
      score -= p.w_coarse * e * e;
    }
  }
  if (p.smooth_sd) {
    const float sd = p.smooth_sd[i];
    if (sd > 0.f) {
      const float e = ((l.x - r.x) - p.smooth_d[i]) / sd;
      score -= p.w_smooth * e * e;
    }
  }
  return score;
}

// Priority of the greedy completion: belief desc, score desc, edge index asc.
__device__ __forceinline__ bool prio_before(const MatchWs& m, int a, int b) {
  const float ba = m.belief[a], bb = m.belief[b];
  if (ba != bb) return ba > bb;
  const float sa = m.es[a], sb = m.es[b];
  if (sa != sb) return sa > sb;
  return a < b;
}

template <typename Less, typename T>
__device__ void cta_bitonic(T* s, int N, Less less) {   // N a power of two
  for (int k = 2; k <= N; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const T a = s[i], b = s[ixj];
          const bool up = (i & k) == 0;
          if (up ? less(b, a) : less(a, b)) {
            s[i] = b;
            s[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
}

__device__ float cta_max(float v, float* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax_ref(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float r = red[0];
  for (int w = 1; w < int(blockDim.x >> 5); ++w) r = fmax_ref(r, red[w]);
  __syncthreads();
  return r;
}

__device__ int cta_or(int v, int* red) {
  v = __any_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  int r = 0;
  for (int w = 0; w < int(blockDim.x >> 5); ++w) r |= red[w];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(1024, 1) k_match(MatchArgs a, MatchWs m) {
  extern __shared__ __align__(16) uint8_t smem[];
  uint64_t* keys = reinterpret_cast<uint64_t*>(smem);
  __shared__ int warp_sums[32];
  __shared__ float redf[32];
  __shared__ int redi[32];
  __shared__ int s_nacc;
  const int tid = threadIdx.x, NT = blockDim.x;
  const int nl = a.nl_dev ? max(0, min(a.nl_cap, *a.nl_dev)) : a.nl_cap;
  const int nr = a.nr_dev ? max(0, min(a.nr_cap, *a.nr_dev)) : a.nr_cap;
  const int maxc = a.maxc;

  // --- right points in y order (ties by index) -------------------------------------
  int N = 1;
  while (N < nr) N <<= 1;
  for (int i = tid; i < N; i += NT)
    keys[i] = (i < nr) ? (uint64_t(ord_f32(a.kr[i].y)) << 32) | uint32_t(i) : ~0ull;
  __syncthreads();
  cta_bitonic(keys, N, [](uint64_t x, uint64_t y) { return x < y; });
  for (int i = tid; i < nr; i += NT) m.order[i] = int(keys[i] & 0xffffffffu);
  __syncthreads();

  // --- candidate rows (build_candidates) --------------------------------------------
  for (int i = tid; i < nl; i += NT) {
    const de_keypoint l = a.kl[i];
    const uint32_t klo = ord_f32(l.y - a.max_dy), khi = ord_f32(l.y + a.max_dy);
    int lo = 0, hi = nr;
    {
      int p = 0, q = nr;
      while (p < q) {
        const int md = (p + q) >> 1;
        if (uint32_t(keys[md] >> 32) < klo) p = md + 1; else q = md;
      }
      lo = p;
      q = nr;
      while (p < q) {
        const int md = (p + q) >> 1;
        if (!(khi < uint32_t(keys[md] >> 32))) p = md + 1; else q = md;
      }
      hi = p;
    }
    int ns = 0;
    for (int p = lo; p < hi; ++p) {
      const float d = l.x - a.kr[int(keys[p] & 0xffffffffu)].x;
      ns += (d < a.min_disp || d > a.max_disp) ? 0 : 1;
    }
    const uint64_t dli = a.dl[i];
    int* sj = m.slot_j + size_t(i) * maxc;
    float* ss = m.slot_s + size_t(i) * maxc;
    if (ns <= maxc) {
      int k = 0;
      for (int p = lo; p < hi; ++p) {
        const int j = int(keys[p] & 0xffffffffu);
        const de_keypoint r = a.kr[j];
        const float d = l.x - r.x;
        if (d < a.min_disp || d > a.max_disp) continue;
        sj[k] = j;
        ss[k] = pair_score(l, r, dli, a.dr[j], a, i);
        ++k;
      }
    } else {                  // best maxc by score, in score order (ties: band order)
      for (int p = lo; p < hi; ++p) {
        const int j = int(keys[p] & 0xffffffffu);
        const de_keypoint r = a.kr[j];
        const float d = l.x - r.x;
        if (d < a.min_disp || d > a.max_disp) continue;
        const float s = pair_score(l, r, dli, a.dr[j], a, i);
        int rank = 0;
        for (int q = lo; q < hi && rank < maxc; ++q) {
          const int jq = int(keys[q] & 0xffffffffu);
          const de_keypoint rq = a.kr[jq];
          const float dq = l.x - rq.x;
          if (dq < a.min_disp || dq > a.max_disp) continue;
          const float sq = pair_score(l, rq, dli, a.dr[jq], a, i);
          rank += (sq > s || (sq == s && q < p)) ? 1 : 0;
        }
        if (rank < maxc) {
          sj[rank] = j;
          ss[rank] = s;
        }
      }
    }
    m.cnt[i] = min(ns, maxc);
  }
  __syncthreads();
  const int E = cta_excl_scan<1024>(m.cnt, nl, warp_sums);
  if (tid == 0) m.cnt[nl] = E;
  for (int j = tid; j < nr; j += NT) {
    m.cstart[j] = 0;
    m.cfill[j] = 0;
  }
  __syncthreads();
  for (int i = tid; i < nl; i += NT) {
    const int b = m.cnt[i], c = m.cnt[i + 1] - b;
    for (int k = 0; k < c; ++k) {
      const int e = b + k;
      const int j = m.slot_j[size_t(i) * maxc + k];
      m.ei[e] = i;
      m.ej[e] = j;
      m.es[e] = m.slot_s[size_t(i) * maxc + k];
      m.beta[e] = 0.f;
      m.rho[e] = 0.f;
      atomicAdd(&m.cstart[j], 1);
    }
  }
  __syncthreads();
  cta_excl_scan<1024>(m.cstart, nr, warp_sums);
  if (tid == 0) m.cstart[nr] = E;
  __syncthreads();
  for (int e = tid; e < E; e += NT) {
    const int j = m.ej[e];
    m.citems[m.cstart[j] + atomicAdd(&m.cfill[j], 1)] = e;
  }
  __syncthreads();

  // --- damped max-sum sweeps ---------------------------------------------------------
  // The sweeps walk each point's edges with dependent loads, so their state (row and
  // column offsets, column items, scores, beta, rho) moves to shared memory when it
  // fits (a few thousand edges take well under the 227 KB); the sort keys there are
  // dead by now.  Same operations in the same order either way.
  const int* bcnt = m.cnt;
  const int* bcst = m.cstart;
  const int* bcit = m.citems;
  const float* bes = m.es;
  float* bbeta = m.beta;
  float* brho = m.rho;
  const size_t bp_bytes = size_t(nl + 1 + nr + 1) * 4 + size_t(E) * 16;
  const bool bp_smem = bp_bytes <= size_t(a.smem_bytes);
  if (bp_smem) {
    int* s_cnt = reinterpret_cast<int*>(smem);
    int* s_cst = s_cnt + (nl + 1);
    int* s_cit = s_cst + (nr + 1);
    float* s_es = reinterpret_cast<float*>(s_cit + E);
    float* s_beta = s_es + E;
    float* s_rho = s_beta + E;
    for (int i = tid; i <= nl; i += NT) s_cnt[i] = m.cnt[i];
    for (int j = tid; j <= nr; j += NT) s_cst[j] = m.cstart[j];
    for (int e = tid; e < E; e += NT) {
      s_cit[e] = m.citems[e];
      s_es[e] = m.es[e];
      s_beta[e] = 0.f;
      s_rho[e] = 0.f;
    }
    __syncthreads();
    bcnt = s_cnt; bcst = s_cst; bcit = s_cit; bes = s_es; bbeta = s_beta; brho = s_rho;
  }
  const float d0 = (a.damping < 0.f) ? 0.f : a.damping;
  const float dmp = (0.99f < d0) ? 0.99f : d0;
  float prev = 1e30f, md = 0.f;
  int it = 0, osc = 0, conv = 0;
  for (; it < a.iters && E > 0; ++it) {
    float loc = 0.f;
    for (int i = tid; i < nl; i += NT) {
      const int b = bcnt[i], c = bcnt[i + 1];
      float best = kNegBig, second = kNegBig;
      int bi = -1;
      for (int e = b; e < c; ++e) {
        const float v = bbeta[e];
        if (v > best) { second = best; best = v; bi = e; } else if (v > second) second = v;
      }
      for (int e = b; e < c; ++e) {
        const float comp = fmax_ref(a.lambda, (e == bi) ? second : best);
        const float tgt = bes[e] - comp;
        const float old = brho[e];
        const float upd = (1.f - dmp) * tgt + dmp * old;
        loc = fmax_ref(loc, fabsf(upd - old));
        brho[e] = upd;
      }
    }
    __syncthreads();
    for (int j = tid; j < nr; j += NT) {
      const int b = bcst[j], c = bcst[j + 1];
      float best = kNegBig, second = kNegBig;
      int bi = -1;
      for (int q = b; q < c; ++q) {
        const int e = bcit[q];
        const float v = brho[e];
        if (v > best) { second = best; best = v; bi = e; } else if (v > second) second = v;
      }
      for (int q = b; q < c; ++q) {
        const int e = bcit[q];
        const float comp = fmax_ref(a.gamma, (e == bi) ? second : best);
        const float tgt = bes[e] - comp;
        const float old = bbeta[e];
        const float upd = (1.f - dmp) * tgt + dmp * old;
        loc = fmax_ref(loc, fabsf(upd - old));
        bbeta[e] = upd;
      }
    }
    md = cta_max(loc, redf);            // includes the barrier the next sweep needs
    if (md > prev) ++osc;
    prev = md;
    if (md < a.eps) {
      conv = 1;
      ++it;
      break;
    }
  }

  if (bp_smem) {                      // the later stages read beta and rho globally
    for (int e = tid; e < E; e += NT) {
      m.beta[e] = bbeta[e];
      m.rho[e] = brho[e];
    }
    __syncthreads();
  }

  // --- belief, margins, mutual best ----------------------------------------------------
  for (int e = tid; e < E; e += NT) m.belief[e] = m.beta[e] + m.rho[e] - m.es[e];
  __syncthreads();
  for (int i = tid; i < nl; i += NT) {
    const int b = m.cnt[i], c = m.cnt[i + 1];
    float b1 = kNegBig, b2 = kNegBig, bl = kNegBig;
    int br = -1;
    for (int e = b; e < c; ++e) {
      const float s = m.es[e];
      if (s > b1) { b2 = b1; b1 = s; } else if (s > b2) b2 = s;
      if (s <= a.lambda) continue;
      if (br < 0 || m.belief[e] > bl) { br = e; bl = m.belief[e]; }
    }
    m.margin[i] = (b1 == kNegBig) ? 0.f
                                  : b1 - ((b2 == kNegBig) ? a.lambda : fmax_ref(b2, a.lambda));
    m.best_row[i] = br;
    m.rt[i] = 0;
  }
  for (int j = tid; j < nr; j += NT) {
    float bl = kNegBig;
    int bc = -1;
    for (int q = m.cstart[j]; q < m.cstart[j + 1]; ++q) {
      const int e = m.citems[q];
      if (m.es[e] <= a.lambda) continue;
      const float v = m.belief[e];
      if (bc < 0 || v > bl || (v == bl && e < bc)) { bc = e; bl = v; }
    }
    m.best_col[j] = bc;
    m.ct[j] = 0;
  }
  __syncthreads();
  for (int i = tid; i < nl; i += NT) {
    const int e = m.best_row[i];
    m.flag[i] = (e >= 0 && m.best_col[m.ej[e]] == e) ? 1 : 0;
  }
  __syncthreads();
  const int n1 = cta_excl_scan<1024>(m.flag, nl, warp_sums);
  auto emit = [&](int e, int pos) {
    if (pos >= a.cap) return;
    const int i = m.ei[e], j = m.ej[e];
    de_match r;
    r.left = i;
    r.right = j;
    r.score = m.es[e];
    r.belief = m.belief[e];
    r.disparity = a.kl[i].x - a.kr[j].x;
    r.dy = a.kl[i].y - a.kr[j].y;
    r.margin = m.margin[i];
    a.out[pos] = r;
  };
  for (int i = tid; i < nl; i += NT) {
    const int e = m.best_row[i];
    const int pos = m.flag[i];
    const int nxt = (i + 1 < nl) ? m.flag[i + 1] : n1;
    if (nxt != pos) {                 // accepted in the mutual pass
      emit(e, pos);
      m.rt[i] = 1;
      m.ct[m.ej[e]] = 1;
    }
  }
  if (tid == 0) s_nacc = 0;
  __syncthreads();

  // --- greedy completion as rounds of locally strongest edges -------------------------
  for (int round = 0; round <= nl; ++round) {
    int any = 0;
    for (int i = tid; i < nl; i += NT) {
      int bst = -1;
      if (!m.rt[i])
        for (int e = m.cnt[i]; e < m.cnt[i + 1]; ++e) {
          if (m.es[e] <= a.lambda || m.ct[m.ej[e]]) continue;
          if (bst < 0 || prio_before(m, e, bst)) bst = e;
        }
      m.rbest[i] = bst;
      any |= bst >= 0;
    }
    for (int j = tid; j < nr; j += NT) {
      int bst = -1;
      if (!m.ct[j])
        for (int q = m.cstart[j]; q < m.cstart[j + 1]; ++q) {
          const int e = m.citems[q];
          if (m.es[e] <= a.lambda || m.rt[m.ei[e]]) continue;
          if (bst < 0 || prio_before(m, e, bst)) bst = e;
        }
      m.cbest[j] = bst;
    }
    if (!cta_or(any, redi)) break;    // barrier inside
    for (int i = tid; i < nl; i += NT) {
      const int e = m.rbest[i];
      if (e >= 0 && m.cbest[m.ej[e]] == e) {
        m.rt[i] = 1;
        m.ct[m.ej[e]] = 1;
        m.acc[atomicAdd(&s_nacc, 1)] = e;
      }
    }
    __syncthreads();
  }
  const int n2 = s_nacc;
  int* sidx = reinterpret_cast<int*>(smem);
  int N2 = 1;
  while (N2 < n2) N2 <<= 1;
  for (int k = tid; k < N2; k += NT) sidx[k] = (k < n2) ? m.acc[k] : -1;
  __syncthreads();
  cta_bitonic(sidx, N2, [&](int x, int y) {
    if (x < 0) return false;
    if (y < 0) return true;
    return prio_before(m, x, y);
  });
  for (int k = tid; k < n2; k += NT) emit(sidx[k], n1 + k);
  if (tid == 0) {
    *a.n_out = n1 + n2;
    if (a.stats) {
      de_match_stats s;
      s.left = nl;
      s.right = nr;
      s.candidates = E;
      s.iterations_run = it;
      s.converged = conv;
      s.final_max_delta = (it > 0) ? md : 0.f;
      s.oscillating = osc;
      *a.stats = s;
    }
  }
}


// ---------------------------------------------------------------------------------
// Keypoint read-out from a dense map (core/tools/de_dense_cuda.cu:866-899): each
// keypoint looks up the disparity and margin at its rounded, clamped pixel; keypoints
// where the map has no positive disparity are dropped; order is kept.  One CTA, an
// ordered compaction in chunks of 1024.
__global__ void __launch_bounds__(1024) k_kp_readout(const de_keypoint* kp, int n,
                                                     const int* n_dev, const float* disp,
                                                     const float* margin, int W, int H,
                                                     de_kp_disparity* out, int cap,
                                                     int* n_out) {
  __shared__ int warp_cnt[32];
  __shared__ int s_total;
  const int cnt = n_dev ? max(0, min(n, *n_dev)) : n;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_total = 0;
  __syncthreads();
  for (int base = 0; base < cnt; base += 1024) {
    const int i = base + threadIdx.x;
    de_kp_disparity r{};
    bool ok = false;
    if (i < cnt) {
      const de_keypoint k = kp[i];
      const int x = min(max(int(k.x + 0.5f), 0), W - 1);
      const int y = min(max(int(k.y + 0.5f), 0), H - 1);
      const float d = disp[size_t(y) * W + x];
      ok = d > 0.f;
      r.x = k.x;
      r.y = k.y;
      r.disparity = d;
      r.margin = margin ? margin[size_t(y) * W + x] : 0.f;
    }
    const unsigned b = __ballot_sync(0xffffffffu, ok);
    if (lane == 0) warp_cnt[w] = __popc(b);
    __syncthreads();
    if (w == 0) {
      int v = warp_cnt[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
      }
      warp_cnt[lane] = v - warp_cnt[lane];        // exclusive
    }
    __syncthreads();
    const int pos = s_total + warp_cnt[w] + __popc(b & ((1u << lane) - 1u));
    if (ok && pos < cap) out[pos] = r;
    __syncthreads();
    if (threadIdx.x == 1023) s_total = pos + (ok ? 1 : 0);
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_out = s_total;
}

int check_det(const de_det_cfg* c, int W, int H) {
  if (!c) return set_error(DE_ERR_ARG, "detector config is NULL");
  if (W < 16 || H < 16 || W > kMaxW || H > kMaxH)
    return set_error(DE_ERR_ARG, "image %dx%d outside 16..%d x 16..%d", W, H, kMaxW, kMaxH);
  if (c->grad_window < 1 || c->grad_window > 15)
    return set_error(DE_ERR_ARG, "grad_window %d outside 1..15", c->grad_window);
  if (std::max(4, c->cell) > kMaxCell)
    return set_error(DE_ERR_ARG, "cell %d above %d", c->cell, kMaxCell);
  if (c->per_cell > 4096 || c->nms_radius > 16 || c->fast_threshold < 0 ||
      c->fast_threshold > 255)
    return set_error(DE_ERR_ARG, "per_cell/nms_radius/fast_threshold out of range");
  return DE_OK;
}

void det_geometry(const de_det_cfg* c, int W, int H, int* cell, int* cols, int* cells,
                  int* keep) {
  *cell = std::max(4, c->cell);
  *cols = (W + *cell - 1) / *cell;
  *cells = *cols * ((H + *cell - 1) / *cell);
  *keep = std::max(1, c->per_cell);
}

}  // namespace

size_t detect_ws_bytes(int W, int H, const de_det_cfg* c) {
  int cell, cols, cells, keep;
  det_geometry(c, W, H, &cell, &cols, &cells, &keep);
  return det_ws_bytes(W, H, cells, keep);
}

int detect_fast_dev(const uint8_t* img, int W, int H, const de_det_cfg* c, de_keypoint* out,
                    int cap, int* n_out, void* ws, size_t bytes, cudaStream_t s) {
  if (int rc = check_det(c, W, H)) return rc;
  if (!img || !n_out || (!out && cap > 0) || !ws || cap < 0)
    return set_error(DE_ERR_ARG, "NULL image, output or workspace");
  int cell, cols, cells, keep;
  det_geometry(c, W, H, &cell, &cols, &cells, &keep);
  const size_t need = det_ws_bytes(W, H, cells, keep);
  if (bytes < need)
    return set_error(DE_ERR_ARG, "detector workspace %zu bytes < %zu", bytes, need);
  DetWs d = carve_det(ws, W, H, cells, keep);
  cudaError_t e = cudaMemsetAsync(d.counters, 0, 64, s);
  if (e != cudaSuccess) return set_error(DE_ERR_CUDA, "cudaMemsetAsync: %s", cudaGetErrorString(e));
  const int border = std::max(c->border, 5);
  const dim3 blk(32, 8), grd((W + 31) / 32, (H + 7) / 8);
  k_fast<<<grd, blk, 0, s>>>(img, W, H, border, c->fast_threshold, c->grad_window,
                             c->min_response, d);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int rad = std::max(1, c->nms_radius);
  if (rad <= 3) k_nms_w<3><<<sms * 8, 256, 0, s>>>(W, H, rad, d);
  else if (rad <= 7) k_nms_w<7><<<sms * 8, 256, 0, s>>>(W, H, rad, d);
  else k_nms<<<sms * 8, 256, 0, s>>>(W, H, rad, d);
  const int capk = ((cell + 1) / 2) * ((cell + 1) / 2);
  const size_t sm = size_t(capk) * (sizeof(de_keypoint) + sizeof(int));
  e = cudaFuncSetAttribute(k_cells, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
  if (e != cudaSuccess) return set_error(DE_ERR_CUDA, "k_cells smem: %s", cudaGetErrorString(e));
  k_cells<<<cells, 256, sm, s>>>(img, W, H, cell, cols, keep, c->grad_window,
                                  c->min_local_std, c->subpixel, d);
  k_det_emit<<<1, 1024, 0, s>>>(cells, keep, d, out, cap, n_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(DE_ERR_CUDA, "detector launch: %s", cudaGetErrorString(e));
  return DE_OK;
}

int census_at_dev(const uint8_t* img, int W, int H, const de_keypoint* kp, int n,
                  const int* n_dev, int hw, int hh, uint64_t* desc, uint8_t* ok,
                  cudaStream_t s) {
  if (!img || (!kp && n > 0) || (!desc && n > 0) || n < 0)
    return set_error(DE_ERR_ARG, "NULL image, keypoints or output");
  if (hw < 1 || hh < 1 || hw > 7 || hh > 7 || (2 * hw + 1) * (2 * hh + 1) - 1 > 64)
    return set_error(DE_ERR_ARG, "census window %dx%d does not fit 64 bits",
                     2 * hw + 1, 2 * hh + 1);
  if (n == 0) return DE_OK;
  k_census_at<<<(n + 255) / 256, 256, 0, s>>>(img, W, H, kp, n, n_dev, hw, hh, desc, ok);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(DE_ERR_CUDA, "census_at launch: %s", cudaGetErrorString(e));
  return DE_OK;
}

int kp_readout_dev(const de_keypoint* kp, int n, const int* n_dev, const float* disp,
                   const float* margin, int W, int H, de_kp_disparity* out, int cap,
                   int* n_out, cudaStream_t s) {
  if (n < 0 || cap < 0 || (n > 0 && (!kp || !disp)) || (cap > 0 && !out) || !n_out ||
      W < 1 || H < 1)
    return set_error(DE_ERR_ARG, "NULL keypoints, map or output, or bad size");
  k_kp_readout<<<1, 1024, 0, s>>>(kp, n, n_dev, disp, margin, W, H, out, cap, n_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(DE_ERR_CUDA, "readout: %s", cudaGetErrorString(e));
  return DE_OK;
}

int check_match_cfg(const de_match_cfg* c) {
  if (!c) return set_error(DE_ERR_ARG, "match config is NULL");
  if (c->max_candidates > 1024)
    return set_error(DE_ERR_ARG, "max_candidates %d above 1024", c->max_candidates);
  if (c->census_bits < 1 || c->census_bits > 64)
    return set_error(DE_ERR_ARG, "census_bits %d outside 1..64", c->census_bits);
  if (c->iterations < 0 || c->iterations > 100000)
    return set_error(DE_ERR_ARG, "iterations %d outside 0..100000", c->iterations);
  return DE_OK;
}

size_t match_ws_bytes_for(int nl, int nr, const de_match_cfg* c) {
  return match_ws_bytes(nl, nr, std::max(1, c->max_candidates));
}

int match_masda_dev(const de_keypoint* kl, const uint64_t* dl, int nl, const int* nl_dev,
                    const de_keypoint* kr, const uint64_t* dr, int nr, const int* nr_dev,
                    const de_match_cfg* c, const de_match_prior* prior, de_match* out,
                    int cap, int* n_out, de_match_stats* stats, void* ws, size_t bytes,
                    cudaStream_t s) {
  if (int rc = check_match_cfg(c)) return rc;
  if (nl < 0 || nr < 0 || nl > (1 << 20) || nr > kSortMax)
    return set_error(DE_ERR_ARG, "keypoint counts %d/%d outside 0..%d / 0..%d", nl, nr,
                     1 << 20, kSortMax);
  if (!n_out || (cap > 0 && !out) || cap < 0 || (nl > 0 && (!kl || !dl)) ||
      (nr > 0 && (!kr || !dr)) || !ws)
    return set_error(DE_ERR_ARG, "NULL keypoints, descriptors, output or workspace");
  const int maxc = std::max(1, c->max_candidates);
  const size_t need = match_ws_bytes(std::max(nl, 1), std::max(nr, 1), maxc);
  if (bytes < need)
    return set_error(DE_ERR_ARG, "match workspace %zu bytes < %zu", bytes, need);
  MatchArgs a;
  a.kl = kl; a.dl = dl; a.kr = kr; a.dr = dr;
  a.nl_cap = nl; a.nr_cap = nr; a.nl_dev = nl_dev; a.nr_dev = nr_dev;
  a.out = out; a.cap = cap; a.n_out = n_out; a.stats = stats;
  a.max_dy = c->max_dy; a.min_disp = c->min_disparity; a.max_disp = c->max_disparity;
  a.sigma_y = c->sigma_y; a.w_y = c->w_y; a.damping = c->damping;
  a.lambda = c->lambda; a.gamma = c->gamma; a.eps = c->converge_eps;
  a.maxc = maxc; a.iters = c->iterations; a.census_bits = c->census_bits;
  a.prior = de_match_prior{};
  if (prior) {
    if ((prior->coarse_sd && !prior->coarse_d) || (prior->smooth_sd && !prior->smooth_d))
      return set_error(DE_ERR_ARG, "a prior's sigma array is given without its disparities");
    a.prior = *prior;
  }
  MatchWs m = carve_match(ws, std::max(nl, 1), std::max(nr, 1), maxc);
  int N = 1;
  while (N < std::max(nr, 1)) N <<= 1;
  // the sort keys need N * 8 bytes; the BP sweeps use whatever the SM offers beyond
  // (one CTA per problem, so the whole of it)
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, k_match);
  if (e != cudaSuccess) return set_error(DE_ERR_CUDA, "k_match attributes: %s", cudaGetErrorString(e));
  const size_t avail = size_t(std::max(0, optin - int(fa.sharedSizeBytes))) & ~size_t(15);
  const size_t sm = std::max(std::max(size_t(N) * 8, size_t(1024)), avail);
  a.smem_bytes = int(sm);
  e = cudaFuncSetAttribute(k_match, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
  if (e != cudaSuccess) return set_error(DE_ERR_CUDA, "k_match smem: %s", cudaGetErrorString(e));
  k_match<<<1, 1024, sm, s>>>(a, m);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(DE_ERR_CUDA, "match launch: %s", cudaGetErrorString(e));
  return DE_OK;
}

}  // namespace de

// ---- C ABI --------------------------------------------------------------------------

extern "C" {

int de_census_at_dev(const uint8_t* img, int W, int H, const de_keypoint* kp, int n,
                     const int* n_dev, int hw, int hh, uint64_t* desc, uint8_t* ok,
                     void* stream) {
  return de::census_at_dev(img, W, H, kp, n, n_dev, hw, hh, desc, ok,
                           static_cast<cudaStream_t>(stream));
}

int de_keypoint_readout_dev(const de_keypoint* kp, int n, const int* n_dev,
                            const float* disp, const float* margin, int W, int H,
                            de_kp_disparity* out, int cap, int* n_out, void* stream) {
  return de::kp_readout_dev(kp, n, n_dev, disp, margin, W, H, out, cap, n_out,
                            static_cast<cudaStream_t>(stream));
}

int de_detect_workspace_bytes(int W, int H, const de_det_cfg* cfg, size_t* bytes) {
  if (!bytes) return de::set_error(DE_ERR_ARG, "bytes is NULL");
  if (int rc = de::check_det(cfg, W, H)) return rc;
  *bytes = de::detect_ws_bytes(W, H, cfg);
  return DE_OK;
}

int de_detect_fast_dev(const uint8_t* img, int W, int H, const de_det_cfg* cfg,
                       de_keypoint* out, int cap, int* n_out, void* workspace, size_t bytes,
                       void* stream) {
  return de::detect_fast_dev(img, W, H, cfg, out, cap, n_out, workspace, bytes,
                             static_cast<cudaStream_t>(stream));
}

int de_match_workspace_bytes(int nl, int nr, const de_match_cfg* cfg, size_t* bytes) {
  if (!bytes) return de::set_error(DE_ERR_ARG, "bytes is NULL");
  if (int rc = de::check_match_cfg(cfg)) return rc;
  if (nl < 0 || nr < 0) return de::set_error(DE_ERR_ARG, "negative keypoint count");
  *bytes = de::match_ws_bytes_for(std::max(nl, 1), std::max(nr, 1), cfg);
  return DE_OK;
}

int de_match_masda_dev(const de_keypoint* kl, const uint64_t* dl, int nl, const int* nl_dev,
                       const de_keypoint* kr, const uint64_t* dr, int nr, const int* nr_dev,
                       const de_match_cfg* cfg, de_match* out, int cap, int* n_out,
                       de_match_stats* stats, void* workspace, size_t bytes, void* stream) {
  return de::match_masda_dev(kl, dl, nl, nl_dev, kr, dr, nr, nr_dev, cfg, nullptr, out, cap,
                             n_out, stats, workspace, bytes, static_cast<cudaStream_t>(stream));
}

int de_match_masda_prior_dev(const de_keypoint* kl, const uint64_t* dl, int nl,
                             const int* nl_dev, const de_keypoint* kr, const uint64_t* dr,
                             int nr, const int* nr_dev, const de_match_cfg* cfg,
                             const de_match_prior* prior, de_match* out, int cap, int* n_out,
                             de_match_stats* stats, void* workspace, size_t bytes,
                             void* stream) {
  return de::match_masda_dev(kl, dl, nl, nl_dev, kr, dr, nr, nr_dev, cfg, prior, out, cap,
                             n_out, stats, workspace, bytes, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
