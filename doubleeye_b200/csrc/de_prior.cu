// The disparity prior as a per-plane mask: core/tools/de_dense.cpp:797-853 (mask),
// :438-483 (filter over a rectangle), :1166-1297 (score, filter and insert under the
// mask), driven by --prior (:1756-1813).
//
// A prior (a previous frame's disparity, a coarse pass) says where each disparity
// plane is worth computing: plane d is needed at the pixels whose band
// [round(prior) - band, round(prior) + band] contains d.  Per image row and plane this
// is an interval of x; per plane a bounding box.  The reference then scores and
// filters each needed plane only over its bounding box padded by 8 pixels (the
// recursive filter's chains start at the rectangle's edges, so values differ from the
// full-plane filter there) and inserts the plane into a pixel's top-2 only inside the
// row intervals.  Sub-pixel refinement is off under a prior (the tool turns it off).
//
// Layout here: the plane-minor volume [y][x][Dpad] of the dense path, so threads of a
// warp take 32 consecutive planes of one row (or column) and every step of their
// sequential chains touches 64 contiguous bytes.  Planes are independent until the
// top-2, which is merged per pixel with a 64-bit compare-and-swap on two packed keys
// ((v + 32768) << 8 | (255 - k), unique per plane), so the insertion order does not
// matter.

#include <algorithm>

#include <cuda_runtime.h>

#include "de_internal.h"

namespace de {
namespace {

constexpr int kMaskPad = 8;          // core/tools/de_dense.cpp:857 (MPAD)
constexpr int kCasLimit = 1 << 20;   // retries of one top-2 merge before giving up

struct Rect { int ylo, yhi, xlo, xhi, pylo, pyhi; };

__device__ __forceinline__ bool plane_rect(const int* box, int D, int k, int W, int H, int hw,
                                           int hh, int d, Rect* r) {
  const int pylo = box[k], pyhi = box[D + k], pxlo = box[2 * D + k], pxhi = box[3 * D + k];
  if (pyhi < pylo) return false;                       // no pixel wants this plane
  r->ylo = max(hh, pylo - kMaskPad);
  r->yhi = min(H - hh, pyhi + 1 + kMaskPad);
  r->xlo = max(hw + d, pxlo - kMaskPad);
  r->xhi = min(W - hw, pxhi + 1 + kMaskPad);
  r->pylo = pylo;
  r->pyhi = pyhi;
  return r->yhi - r->ylo >= 1 && r->xhi - r->xlo >= 2;
}

__global__ void k_prior_init(int* box, int D, int W, int H, unsigned long long* top2,
                             long long WH) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < WH;
       i += (long long)gridDim.x * blockDim.x)
    top2[i] = 0ull;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < D; k += gridDim.x * blockDim.x) {
    box[k] = H;
    box[D + k] = -1;
    box[2 * D + k] = W;
    box[3 * D + k] = -1;
  }
}

// One CTA per image row: the row's intervals in shared memory, then the planes'
// bounding boxes.  Pixels with a non-finite prior want no plane.
__global__ void k_prior_mask(const float* __restrict__ prior, int W, int H, int D, int dmin,
                             int dmax, int band, int16_t* mx0, int16_t* mx1, int* box) {
  extern __shared__ int sm[];
  int* r0 = sm;
  int* r1 = sm + D;
  const int y = blockIdx.x;
  for (int k = threadIdx.x; k < D; k += blockDim.x) {
    r0[k] = W;
    r1[k] = -1;
  }
  __syncthreads();
  for (int x = threadIdx.x; x < W; x += blockDim.x) {
    const float p = prior[size_t(y) * W + x];
    if (!isfinite(p)) continue;
    const int dc = int(lroundf(fminf(fmaxf(p, -1e6f), 1e6f)));
    const int klo = max(dmin, dc - band) - dmin;
    const int khi = min(dmax, dc + band) - dmin;
    for (int k = klo; k <= khi; ++k) {
      atomicMin(&r0[k], x);
      atomicMax(&r1[k], x);
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < D; k += blockDim.x) {
    const int a = r0[k], b = r1[k];
    mx0[size_t(y) * D + k] = int16_t(a);
    mx1[size_t(y) * D + k] = int16_t(b);
    if (b < a) continue;
    atomicMin(&box[k], y);
    atomicMax(&box[D + k], y);
    atomicMin(&box[2 * D + k], a);
    atomicMax(&box[3 * D + k], b);
  }
}

__device__ __forceinline__ int32_t score_at(const DevCfg& c, const DevPair& P, int y, int x,
                                            int d) {
  const uint64_t wl = P.cwL[size_t(y) * P.cpitch + P.lpad + x];
  const uint64_t wr = P.cwR[size_t(y) * P.cpitch + x - d];
  int h;
  if (c.packed) {
    const uint32_t lo = uint32_t(wl) ^ uint32_t(wr);
    const uint32_t hi = uint32_t(wl >> 32) ^ uint32_t(wr >> 32);
    h = __popc(lo) + __popc(hi & 0xFFFFu);
  } else {
    h = __popcll(wl ^ wr);
  }
  const int a = abs(int(P.L[size_t(y) * P.W + x]) - int(P.R[size_t(y) * P.W + x - d]));
  return (int32_t(c.tbl[h]) * (1024 - c.wq) + int32_t(c.adt[a]) * c.wq) >> 10;
}

__device__ __forceinline__ int32_t rf(int32_t c, int32_t f, int32_t a) {
  return c + ((a * (f - c) + (1 << 14)) >> 15);
}

// Horizontal passes over each needed plane's rectangle: thread = (row, plane).
__global__ void k_prior_rows(DevCfg cfg, DevPair P, const int* __restrict__ box) {
  const int D = P.D, W = P.W, H = P.H, Dpad = P.Dpad;
  const int y = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= D) return;
  const int d = cfg.dmin + k;
  Rect r;
  if (!plane_rect(box, D, k, W, H, cfg.hw, cfg.hh, d, &r) || y < r.ylo || y >= r.yhi) return;
  int16_t* v = P.vol + size_t(y) * W * Dpad + k;
  const uint16_t* ax = P.ax + size_t(y) * P.apitch + P.lpad;
  int32_t f = score_at(cfg, P, y, r.xlo, d);
  v[size_t(r.xlo) * Dpad] = int16_t(f);
  for (int x = r.xlo + 1; x < r.xhi; ++x) {
    f = rf(score_at(cfg, P, y, x, d), f, ax[x]);
    v[size_t(x) * Dpad] = int16_t(f);
  }
  for (int x = r.xhi - 2; x >= r.xlo; --x) {
    f = rf(v[size_t(x) * Dpad], f, ax[x + 1]);
    v[size_t(x) * Dpad] = int16_t(f);
  }
}

__device__ __forceinline__ void top2_insert(unsigned long long* p, uint32_t key, int* err) {
  unsigned long long old = *reinterpret_cast<volatile unsigned long long*>(p);
  for (int i = 0; i < kCasLimit; ++i) {
    const uint32_t k0 = uint32_t(old >> 32), k1 = uint32_t(old);
    if (key <= k1) return;                               // keys are unique per plane
    const unsigned long long nv =
        key > k0 ? (static_cast<unsigned long long>(key) << 32) | k0
                 : (static_cast<unsigned long long>(k0) << 32) | key;
    const unsigned long long seen = atomicCAS(p, old, nv);
    if (seen == old) return;
    old = seen;
  }
  if (err) atomicExch(err, 2);
}

// Vertical passes and the masked insert: thread = (column, plane).
__global__ void k_prior_cols(DevCfg cfg, DevPair P, const int* __restrict__ box,
                             const int16_t* __restrict__ mx0, const int16_t* __restrict__ mx1,
                             unsigned long long* top2, int* err) {
  const int D = P.D, W = P.W, H = P.H, Dpad = P.Dpad;
  const int x = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= D) return;
  const int d = cfg.dmin + k;
  Rect r;
  if (!plane_rect(box, D, k, W, H, cfg.hw, cfg.hh, d, &r) || x < r.xlo || x >= r.xhi) return;
  int16_t* col = P.vol + size_t(x) * Dpad + k;
  const size_t st = size_t(W) * Dpad;
  int32_t f = col[size_t(r.ylo) * st];
  for (int y = r.ylo + 1; y < r.yhi; ++y) {
    f = rf(col[size_t(y) * st], f, P.ay[size_t(y) * W + x]);
    col[size_t(y) * st] = int16_t(f);
  }
  const int iy0 = max(r.ylo, r.pylo), iy1 = min(r.yhi, r.pyhi + 1);
  const uint32_t kk = uint32_t(255 - k);
  auto insert = [&](int y, int32_t v) {
    if (y < iy0 || y >= iy1) return;
    const int xa = max(r.xlo, int(mx0[size_t(y) * D + k]));
    const int xb = min(r.xhi, int(mx1[size_t(y) * D + k]) + 1);
    if (x < xa || x >= xb) return;
    const uint32_t key = (uint32_t(v + 32768) << 8) | kk;
    top2_insert(top2 + size_t(y) * W + x, key, err);
    if (P.rkey) atomicMax(P.rkey + size_t(y) * W + x - d, key);
  };
  insert(r.yhi - 1, f);                                  // the last row: forward value
  for (int y = r.yhi - 2; y >= r.ylo; --y) {
    f = rf(col[size_t(y) * st], f, P.ay[size_t(y + 1) * W + x]);
    insert(y, f);
  }
}

__global__ void k_prior_keys(DevPair P, const unsigned long long* top2) {
  const long long WH = (long long)P.W * P.H;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < WH;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long t = top2[i];
    P.key0[i] = uint32_t(t >> 32);
    P.key1[i] = uint32_t(t);
    P.nb[i] = 0x80008000u;                               // no sub-pixel neighbours
  }
}

}  // namespace

size_t prior_ws_bytes(int W, int H, int D) {
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  return 2 * up(size_t(H) * D * 2) + up(size_t(D) * 16) + up(size_t(W) * H * 8);
}

cudaError_t launch_prior(const DevCfg& cfg, const Batch& b, const float* prior, int band,
                         void* ws, cudaStream_t s) {
  const DevPair& P = b.p[0];
  const int W = P.W, H = P.H, D = P.D;
  auto up = [](size_t v) { return (v + 255) & ~size_t(255); };
  uint8_t* p = static_cast<uint8_t*>(ws);
  int16_t* mx0 = reinterpret_cast<int16_t*>(p);                 p += up(size_t(H) * D * 2);
  int16_t* mx1 = reinterpret_cast<int16_t*>(p);                 p += up(size_t(H) * D * 2);
  int* box = reinterpret_cast<int*>(p);                         p += up(size_t(D) * 16);
  unsigned long long* top2 = reinterpret_cast<unsigned long long*>(p);
  const long long WH = (long long)W * H;
  k_prior_init<<<int(std::min<long long>((WH + 255) / 256, 1184)), 256, 0, s>>>(box, D, W, H,
                                                                               top2, WH);
  k_prior_mask<<<H, 256, size_t(2) * D * sizeof(int), s>>>(prior, W, H, D, cfg.dmin,
                                                           cfg.dmin + D - 1, band, mx0, mx1,
                                                           box);
  const int kb = (D + 127) / 128;
  k_prior_rows<<<dim3(kb, H), 128, 0, s>>>(cfg, P, box);
  k_prior_cols<<<dim3(kb, W), 128, 0, s>>>(cfg, P, box, mx0, mx1, top2, b.err);
  k_prior_keys<<<int(std::min<long long>((WH + 255) / 256, 1184)), 256, 0, s>>>(P, top2);
  return cudaGetLastError();
}

}  // namespace de
