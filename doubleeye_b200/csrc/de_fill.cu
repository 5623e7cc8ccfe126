// Hole filling of a disparity map, so it can serve as a prior: the reference's
// `fill` (article/coarse_to_fine.py:58-76), "nearest-valid inpainting by iterated
// 4-neighbour averaging".  Up to 128 Jacobi sweeps; in each, every non-finite pixel
// with at least one finite 4-neighbour (neighbours wrap around the image edges, as
// np.roll does) becomes the float32 mean of those neighbours, summed in the order
// left, right, up, down.  The sweeps stop when one changes nothing; what is still
// non-finite then becomes 0.  A prior with holes is refused by the prior path (the
// reference's tool refuses one too), so a previous frame's map goes through this
// first.
//
// Temporal blocking: a CTA loads a 32x32 tile with an 8-pixel halo into shared
// memory and runs 8 sweeps there (sweep i is exact on the tile shrunk by i), so one
// launch advances the whole map by 8 sweeps with one read and one write of it.  Up to
// 16 launches give the 128 sweeps.  A pixel only ever goes from non-finite to
// finite, so a launch that changes nothing means every later sweep would change
// nothing too: launch j records whether it changed anything, and launch j+1 returns
// at once when launch j did not.  The last kernel zeroes what is left.

#include <algorithm>

#include <cuda_runtime.h>

#include "de_internal.h"

namespace de {
namespace {

constexpr int kFT = 32;                 // tile edge
constexpr int kFR = 8;                  // halo = sweeps per launch
constexpr int kFS = kFT + 2 * kFR;      // shared edge
constexpr int kFLaunches = 16;          // 16 x 8 = 128 sweeps, the reference's cap

__device__ __forceinline__ int wrap(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}

// One launch of kFR sweeps.  flags[j] != 0: launch j changed some pixel.
__global__ void __launch_bounds__(256) k_fill_sweeps(const float* __restrict__ in,
                                                     float* __restrict__ out, int W, int H,
                                                     int* flags, int j) {
  if (j > 0 && flags[j - 1] == 0) return;            // converged: nothing moves any more
  __shared__ float s[2][kFS][kFS + 1];
  __shared__ int changed;
  const int x0 = blockIdx.x * kFT - kFR, y0 = blockIdx.y * kFT - kFR;
  const int tid = threadIdx.x;
  if (tid == 0) changed = 0;
  for (int i = tid; i < kFS * kFS; i += blockDim.x) {
    const int ty = i / kFS, tx = i % kFS;
    s[0][ty][tx] = in[size_t(wrap(y0 + ty, H)) * W + wrap(x0 + tx, W)];
  }
  __syncthreads();
  int cur = 0;
  for (int it = 1; it <= kFR; ++it) {
    // sweep `it` is exact on [it, kFS - it) in both directions
    const int lo = it, n = kFS - 2 * it;
    for (int i = tid; i < n * n; i += blockDim.x) {
      const int ty = lo + i / n, tx = lo + i % n;
      const float v = s[cur][ty][tx];
      float r = v;
      if (!isfinite(v)) {
        const float nb[4] = {s[cur][ty][tx - 1], s[cur][ty][tx + 1], s[cur][ty - 1][tx],
                             s[cur][ty + 1][tx]};
        float acc = 0.f, cnt = 0.f;
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (isfinite(nb[q])) { acc = __fadd_rn(acc, nb[q]); cnt = __fadd_rn(cnt, 1.f); }
        if (cnt > 0.f) r = __fdiv_rn(acc, cnt);
      }
      s[cur ^ 1][ty][tx] = r;
    }
    cur ^= 1;
    __syncthreads();
  }
  for (int i = tid; i < kFT * kFT; i += blockDim.x) {
    const int ty = i / kFT, tx = i % kFT;
    const int x = blockIdx.x * kFT + tx, y = blockIdx.y * kFT + ty;
    if (x >= W || y >= H) continue;
    const size_t g = size_t(y) * W + x;
    const float v = s[cur][ty + kFR][tx + kFR];
    if (isfinite(v) != isfinite(in[g])) changed = 1;     // any writer sets the same 1
    out[g] = v;
  }
  __syncthreads();
  if (tid == 0 && changed) atomicExch(&flags[j], 1);
}

__global__ void k_fill_finish(float* dst, const float* tmp, long long n, const int* flags) {
  // launch j wrote buffer (j + 1) & 1 of {dst, tmp}.  The first launch that changed
  // nothing ran (its predecessor changed something) and copied its input, which is the
  // result; if every launch changed something, the 16th wrote it.
  int last = kFLaunches - 1;
  for (int j = 0; j < kFLaunches - 1; ++j)
    if (flags[j] == 0) { last = j; break; }
  const float* src = ((last + 1) & 1) ? tmp : dst;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float v = src[i];
    dst[i] = isfinite(v) ? v : 0.f;
  }
}

}  // namespace

size_t fill_ws_bytes(int W, int H) { return ((size_t(W) * H * 4 + 255) & ~size_t(255)) + 256; }

// src is read only; dst (W x H) receives the filled map; ws holds one map-sized
// ping-pong buffer and the per-launch flags.
int fill_holes_dev(const float* src, float* dst, int W, int H, void* ws, size_t ws_bytes,
                   cudaStream_t s) {
  if (!src || !dst || W < 1 || H < 1 || W > DE_MAX_DIM || H > DE_MAX_DIM)
    return set_error(DE_ERR_ARG, "fill: NULL map or size %dx%d out of range", W, H);
  if (!ws || ws_bytes < fill_ws_bytes(W, H))
    return set_error(DE_ERR_ARG, "fill: workspace %zu bytes, need %zu", ws_bytes,
                     fill_ws_bytes(W, H));
  float* tmp = static_cast<float*>(ws);
  int* flags = reinterpret_cast<int*>(static_cast<uint8_t*>(ws) + fill_ws_bytes(W, H) - 256);
  cudaError_t e = cudaMemsetAsync(flags, 0, kFLaunches * sizeof(int), s);
  // ping-pong: launch j reads (j == 0 ? src : buf[j & 1]) and writes buf[(j + 1) & 1],
  // with buf = {dst, tmp}
  float* buf[2] = {dst, tmp};
  const dim3 grid((W + kFT - 1) / kFT, (H + kFT - 1) / kFT);
  for (int j = 0; j < kFLaunches && e == cudaSuccess; ++j) {
    k_fill_sweeps<<<grid, 256, 0, s>>>(j == 0 ? src : buf[j & 1], buf[(j + 1) & 1], W, H,
                                       flags, j);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    const long long n = (long long)W * H;
    k_fill_finish<<<int(std::min<long long>((n + 255) / 256, 148 * 8)), 256, 0, s>>>(
        dst, tmp, n, flags);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return set_error(DE_ERR_CUDA, "fill: %s", cudaGetErrorString(e));
  return DE_OK;
}

}  // namespace de

extern "C" int de_prior_fill_dev(const float* src, float* dst, int W, int H, void* workspace,
                                 size_t bytes, void* stream) {
  return de::fill_holes_dev(src, dst, W, H, workspace, bytes, static_cast<cudaStream_t>(stream));
}

extern "C" size_t de_prior_fill_workspace_bytes(int W, int H) {
  return (W < 1 || H < 1) ? 0 : de::fill_ws_bytes(W, H);
}
