// Edge-list MASDA in double precision: the reference's Python entry points.
//
//   masda_sparse / _seg_max_excluding / decide   article/masda_stereo.py:392-492
//   build_problem / hamming / census / to_edges  article/masda_stereo.py:264-326,445-450
//   dense_problem                                article/dense_masda.py:39-79
//
// The Python reference runs in NumPy float64; so does this path (operation for
// operation, no contraction), so message histories are bit-identical.  The work is
// proportional to the number of candidate edges, which for dense_problem is W*H*D
// (52 M at 848x480, D=128), so every pass is a grid-wide kernel:
//   * "max over my row excluding me" = segment max, how many attain it, and the
//     largest value below it, accumulated with 64-bit atomics on order-preserving
//     keys (so any accumulation order gives NumPy's value);
//   * the greedy decision (argsort by belief, accept an edge whose row and column are
//     still free) runs as rounds: an edge that is the strongest remaining option of
//     both its row and its column is exactly the one the sequential greedy accepts,
//     so each round accepts all of those and drops the edges they block.
// NumPy's argsort leaves the order of exactly equal beliefs unspecified; here ties go
// to the lower edge index (a stable argsort).

#include <algorithm>
#include <climits>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "de_internal.h"

namespace de {
namespace {

using u64 = unsigned long long;

__device__ __forceinline__ u64 okey(double v) {   // order-preserving; -0 and +0 equal
  const u64 b = static_cast<u64>(__double_as_longlong(v + 0.0));
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dkey(u64 k) {
  const u64 b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double(static_cast<long long>(b));
}
__device__ __forceinline__ double fmax_np(double a, double b) { return (a < b) ? b : a; }

constexpr u64 kKeyNegInf = 0x000fffffffffffffull;   // okey(-inf)

int grid_for(long long n, int per_block = 256) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  const long long need = (n + per_block - 1) / per_block;
  return int(std::max(1LL, std::min(need, (long long)sms * 8)));
}

#define GRID_STRIDE(i, n) \
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); \
       i += (long long)gridDim.x * blockDim.x)

// ---- segment statistics ------------------------------------------------------------

__global__ void k_seg_reset(u64* m1, u64* m2, int* cnt, long long n) {
  GRID_STRIDE(k, n) {
    m1[k] = kKeyNegInf;
    m2[k] = kKeyNegInf;
    cnt[k] = 0;
  }
}

__global__ void k_seg_max(const double* v, const int64_t* idx, long long E, u64* m1,
                          const int* done) {
  if (done && *done) return;
  GRID_STRIDE(e, E) atomicMax(m1 + idx[e], okey(v[e]));
}

__global__ void k_seg_second(const double* v, const int64_t* idx, long long E, const u64* m1,
                             u64* m2, int* cnt, const int* done) {
  if (done && *done) return;
  GRID_STRIDE(e, E) {
    const long long k = idx[e];
    const u64 x = okey(v[e]);
    if (x >= m1[k]) atomicAdd(cnt + k, 1);
    else atomicMax(m2 + k, x);
  }
}

__device__ __forceinline__ double excluding(u64 x, u64 m1, u64 m2, int cnt) {
  return dkey((x >= m1) ? (cnt > 1 ? m1 : m2) : m1);
}

__global__ void k_seg_out(const double* v, const int64_t* idx, long long E, const u64* m1,
                          const u64* m2, const int* cnt, double* out) {
  GRID_STRIDE(e, E) {
    const long long k = idx[e];
    out[e] = excluding(okey(v[e]), m1[k], m2[k], cnt[k]);
  }
}

// ---- message passing (masda_stereo.py:469-480) -------------------------------------

struct BpArgs {
  const int64_t* ei;
  const int64_t* ej;
  const double* se;
  double* beta;
  double* rho;
  u64 *m1r, *m2r, *m1c, *m2c;
  int *cntr, *cntc;
  u64* delta;        // [0] rho pass, [1] beta pass
  int* done;
  double* hist;
  int* n_hist;
  long long E, m, n;
  double lam, gam, damping, eps;
};

__device__ void block_max_to(u64* dst, u64 v) {
  __shared__ u64 red[32];
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    u64 r = red[0];
    for (int w = 1; w < int(blockDim.x >> 5); ++w) r = max(r, red[w]);
    atomicMax(dst, r);
  }
}

__global__ void k_bp_init(BpArgs a) {
  GRID_STRIDE(e, a.E) {
    a.beta[e] = 0.0;
    a.rho[e] = 0.0;
  }
  GRID_STRIDE(k, a.m) { a.m1r[k] = kKeyNegInf; a.m2r[k] = kKeyNegInf; a.cntr[k] = 0; }
  GRID_STRIDE(k, a.n) { a.m1c[k] = kKeyNegInf; a.m2c[k] = kKeyNegInf; a.cntc[k] = 0; }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.delta[0] = a.delta[1] = okey(0.0);
    *a.done = 0;
    *a.n_hist = 0;
  }
}

// rho = (1-d) * (s - max(lam, max_{row, excl}(beta))) + d * rho; feeds the column max.
__global__ void k_bp_rho(BpArgs a) {
  if (*a.done) return;
  u64 dmax = okey(0.0);
  GRID_STRIDE(e, a.E) {
    const long long i = a.ei[e];
    const double comp = fmax_np(a.lam, excluding(okey(a.beta[e]), a.m1r[i], a.m2r[i],
                                                 a.cntr[i]));
    const double old = a.rho[e];
    const double nr = (1.0 - a.damping) * (a.se[e] - comp) + a.damping * old;
    a.rho[e] = nr;
    dmax = max(dmax, okey(fabs(nr - old)));
    atomicMax(a.m1c + a.ej[e], okey(nr));
  }
  block_max_to(a.delta + 0, dmax);
}

// Column second-best over the new rho; clears the row statistics for the beta pass.
__global__ void k_bp_col_second(BpArgs a) {
  if (*a.done) return;
  GRID_STRIDE(e, a.E) {
    const long long j = a.ej[e];
    const u64 x = okey(a.rho[e]);
    if (x >= a.m1c[j]) atomicAdd(a.cntc + j, 1);
    else atomicMax(a.m2c + j, x);
  }
  GRID_STRIDE(k, a.m) { a.m1r[k] = kKeyNegInf; a.m2r[k] = kKeyNegInf; a.cntr[k] = 0; }
}

__global__ void k_bp_beta(BpArgs a) {
  if (*a.done) return;
  u64 dmax = okey(0.0);
  GRID_STRIDE(e, a.E) {
    const long long j = a.ej[e];
    const double comp = fmax_np(a.gam, excluding(okey(a.rho[e]), a.m1c[j], a.m2c[j],
                                                 a.cntc[j]));
    const double old = a.beta[e];
    const double nb = (1.0 - a.damping) * (a.se[e] - comp) + a.damping * old;
    a.beta[e] = nb;
    dmax = max(dmax, okey(fabs(nb - old)));
    atomicMax(a.m1r + a.ei[e], okey(nb));
  }
  block_max_to(a.delta + 1, dmax);
}

// Row second-best for the next rho pass; clears the column statistics.
__global__ void k_bp_row_second(BpArgs a) {
  if (*a.done) return;
  GRID_STRIDE(e, a.E) {
    const long long i = a.ei[e];
    const u64 x = okey(a.beta[e]);
    if (x >= a.m1r[i]) atomicAdd(a.cntr + i, 1);
    else atomicMax(a.m2r + i, x);
  }
  GRID_STRIDE(k, a.n) { a.m1c[k] = kKeyNegInf; a.m2c[k] = kKeyNegInf; a.cntc[k] = 0; }
}

__global__ void k_bp_finish(BpArgs a, int it) {
  if (*a.done) return;
  const double d = fmax_np(dkey(a.delta[0]), dkey(a.delta[1]));
  a.hist[it] = d;
  *a.n_hist = it + 1;
  a.delta[0] = a.delta[1] = okey(0.0);
  if (d < a.eps) *a.done = 1;
}

__global__ void k_belief(const double* beta, const double* rho, const double* se, long long E,
                         double* belief) {
  GRID_STRIDE(e, E) belief[e] = beta[e] + rho[e] - se[e];
}

// ---- greedy decision in belief order (masda_stereo.py:392-414, 482-491) -----------

struct DecArgs {
  const int64_t* ei;
  const int64_t* ej;
  const double* se;
  const double* belief;
  int64_t* assign;   // [m]
  u64 *rbk, *cbk;    // best key per row / column
  int *rbi, *cbi;    // lowest edge index with that key
  uint8_t *rt, *ct;
  int* list[2];
  int* count;        // [0], [1] list sizes, [2] accepted this round
  long long E, m, n;
  double lam;
};

__global__ void k_dec_init(DecArgs a) {
  GRID_STRIDE(k, a.m) { a.assign[k] = -1; a.rbk[k] = 0; a.rbi[k] = INT_MAX; a.rt[k] = 0; }
  GRID_STRIDE(k, a.n) { a.cbk[k] = 0; a.cbi[k] = INT_MAX; a.ct[k] = 0; }
  GRID_STRIDE(e, a.E) {
    if (a.se[e] <= a.lam || !isfinite(a.belief[e])) continue;
    a.list[0][atomicAdd(a.count + 0, 1)] = int(e);
  }
}

__global__ void k_dec_best(DecArgs a, int cur) {
  const int nact = a.count[cur];
  GRID_STRIDE(q, nact) {
    const int e = a.list[cur][q];
    const u64 k = okey(a.belief[e]);
    atomicMax(a.rbk + a.ei[e], k);
    atomicMax(a.cbk + a.ej[e], k);
  }
}

__global__ void k_dec_index(DecArgs a, int cur) {
  const int nact = a.count[cur];
  GRID_STRIDE(q, nact) {
    const int e = a.list[cur][q];
    const u64 k = okey(a.belief[e]);
    if (k == a.rbk[a.ei[e]]) atomicMin(a.rbi + a.ei[e], e);
    if (k == a.cbk[a.ej[e]]) atomicMin(a.cbi + a.ej[e], e);
  }
}

__global__ void k_dec_accept(DecArgs a, int cur) {
  const int nact = a.count[cur];
  GRID_STRIDE(q, nact) {
    const int e = a.list[cur][q];
    const long long i = a.ei[e], j = a.ej[e];
    if (a.rbi[i] == e && a.cbi[j] == e) {
      a.assign[i] = j;
      a.rt[i] = 1;
      a.ct[j] = 1;
    }
  }
}

__global__ void k_dec_keep(DecArgs a, int cur) {
  const int nact = a.count[cur];
  GRID_STRIDE(q, nact) {
    const int e = a.list[cur][q];
    const long long i = a.ei[e], j = a.ej[e];
    a.rbk[i] = 0;
    a.rbi[i] = INT_MAX;
    a.cbk[j] = 0;
    a.cbi[j] = INT_MAX;
    if (!a.rt[i] && !a.ct[j]) a.list[cur ^ 1][atomicAdd(a.count + (cur ^ 1), 1)] = e;
  }
}

__global__ void k_dec_flip(int* count, int cur) {
  count[cur] = 0;            // the list just consumed becomes the next output
}

// Caller-supplied node indices are checked on the device before any pass uses them.
__global__ void k_check_idx(const int64_t* idx, long long E, long long n, int* bad) {
  GRID_STRIDE(e, E)
    if (idx[e] < 0 || idx[e] >= n) *bad = 1;
}

// ---- problem construction ------------------------------------------------------------

__global__ void k_hamming(const uint64_t* a, const uint64_t* b, long long n, int32_t* out) {
  GRID_STRIDE(k, n) out[k] = __popcll(a[k] ^ b[k]);
}

__global__ void k_census_pts(const uint8_t* __restrict__ img, int W, int H,
                             const int32_t* xy, long long n, int hw, int hh, uint64_t* out,
                             uint8_t* ok) {
  GRID_STRIDE(t, n) {
    const int x = xy[2 * t], y = xy[2 * t + 1];
    const bool in = x >= hw && y >= hh && x < W - hw && y < H - hh;
    uint64_t v = 0;
    if (in) {
      const int c = img[size_t(y) * W + x];
      int bit = 0;
      for (int dy = -hh; dy <= hh; ++dy)
        for (int dx = -hw; dx <= hw; ++dx) {
          if (dx == 0 && dy == 0) continue;
          if (int(img[size_t(y + dy) * W + x + dx]) < c) v |= 1ull << bit;
          ++bit;
        }
    }
    out[t] = v;
    if (ok) ok[t] = in;
  }
}

// build_problem: S[i, j] = (24 - h)/24 - w_y * (dy / sigma_y)^2 where the gates pass,
// -inf elsewhere; NumPy's types: dy, d, the gates and the penalty in float32, the
// descriptor term in float64, the sum rounded to float32.
__global__ void k_build_problem(const float* pl, const uint64_t* dl, long long m,
                                const float* pr, const uint64_t* dr, long long n,
                                float max_dy, float dmin, float dmax, float sigma_y,
                                float w_y, double half, float* S) {
  GRID_STRIDE(t, m * n) {
    const long long i = t / n, j = t % n;
    const float dy = pl[2 * i + 1] - pr[2 * j + 1];
    const float d = pl[2 * i] - pr[2 * j];
    float s = -INFINITY;
    if (fabsf(dy) <= max_dy && d >= dmin && d <= dmax) {
      const double desc = (half - double(__popcll(dl[i] ^ dr[j]))) / half;
      const float q = dy / sigma_y;
      const float pen = w_y * (q * q);
      s = float(desc - double(pen));
    }
    S[t] = s;
  }
}

// to_edges: finite entries of an m x n matrix in row-major order.
__global__ void k_row_count(const float* S, long long m, long long n, int64_t* cnt) {
  const int lane = threadIdx.x & 31;
  for (long long i = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; i < m;
       i += ((long long)gridDim.x * blockDim.x) >> 5) {
    long long c = 0;
    for (long long j = lane; j < n; j += 32) c += isfinite(S[i * n + j]) ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) cnt[i] = c;
  }
}

__global__ void k_excl_scan_i64(int64_t* a, long long n, int64_t* total) {
  // one CTA of 1024 threads, contiguous chunks
  __shared__ int64_t sums[1024];
  const int tid = threadIdx.x;
  const long long per = (n + 1023) / 1024;
  const long long lo = (tid * per < n) ? tid * per : n;
  const long long hi = (lo + per < n) ? lo + per : n;
  int64_t s = 0;
  for (long long i = lo; i < hi; ++i) s += a[i];
  sums[tid] = s;
  __syncthreads();
  if (tid == 0) {
    int64_t run = 0;
    for (int k = 0; k < 1024; ++k) { const int64_t c = sums[k]; sums[k] = run; run += c; }
    *total = run;
  }
  __syncthreads();
  int64_t run = sums[tid];
  for (long long i = lo; i < hi; ++i) { const int64_t c = a[i]; a[i] = run; run += c; }
}

__global__ void k_row_write(const float* S, long long m, long long n, const int64_t* off,
                            int64_t* ei, int64_t* ej, double* se, long long cap) {
  const int lane = threadIdx.x & 31;
  for (long long i = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; i < m;
       i += ((long long)gridDim.x * blockDim.x) >> 5) {
    long long base = off[i];
    for (long long j0 = 0; j0 < n; j0 += 32) {
      const long long j = j0 + lane;
      const float v = (j < n) ? S[i * n + j] : 0.f;
      const bool f = j < n && isfinite(v);
      const unsigned b = __ballot_sync(0xffffffffu, f);
      if (f) {
        const long long e = base + __popc(b & ((1u << lane) - 1u));
        if (e < cap) {
          ei[e] = i;
          ej[e] = j;
          se[e] = double(v);
        }
      }
      base += __popc(b);
    }
  }
}

// dense_problem: census images, then one edge per (d, y, x) in the reference's order
// (d outer, then rows, then columns).
__global__ void k_census_plain(const uint8_t* __restrict__ img, int W, int H, int hw, int hh,
                               uint64_t* out) {
  GRID_STRIDE(t, (long long)W * H) {
    const int x = int(t % W), y = int(t / W);
    uint64_t v = 0;
    if (x >= hw && x < W - hw && y >= hh && y < H - hh) {
      const int c = img[t];
      int bit = 0;
      for (int dy = -hh; dy <= hh; ++dy)
        for (int dx = -hw; dx <= hw; ++dx) {
          if (dx == 0 && dy == 0) continue;
          if (int(img[size_t(y + dy) * W + x + dx]) < c) v |= 1ull << bit;
          ++bit;
        }
    }
    out[t] = v;
  }
}

constexpr int kMaxDpBlocks = 512;
struct DpArgs {
  const uint64_t* cl;
  const uint64_t* cr;
  int64_t* ei;
  int64_t* ej;
  float* se;
  int W, H, hw, hh, dmin, nd;
  long long E;
  float tab[65];
  long long off[kMaxDpBlocks + 1];
};

__global__ void k_dense_problem(DpArgs a) {
  GRID_STRIDE(t, a.E) {
    int lo = 0, hi = a.nd;                      // block k with off[k] <= t < off[k+1]
    while (hi - lo > 1) {
      const int md = (lo + hi) >> 1;
      if (a.off[md] <= t) lo = md; else hi = md;
    }
    const int dd = a.dmin + lo;
    const long long local = t - a.off[lo];
    const int nx = a.W - 2 * a.hw - dd;
    const int y = a.hh + int(local / nx);
    const int x = a.hw + dd + int(local % nx);
    const long long p = (long long)y * a.W + x;
    a.ei[t] = p;
    a.ej[t] = p - dd;
    a.se[t] = a.tab[__popcll(a.cl[p] ^ a.cr[p - dd])];
  }
}

size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

// ---- host side ------------------------------------------------------------------------

size_t masda_edges_ws_bytes(long long E, long long m, long long n) {
  const size_t e = size_t(std::max(E, 1LL)), mm = size_t(std::max(m, 1LL)),
               nn = size_t(std::max(n, 1LL));
  return up256(e * 8) * 3 + up256(mm * 8) * 2 + up256(nn * 8) * 2 + up256(mm * 4) +
         up256(nn * 4) + up256(64) + up256(e * 4) * 2 + up256(mm) + up256(nn) +
         up256(mm * 4) + up256(nn * 4);
}

namespace {

struct EdgeWs {
  double *beta, *rho, *belief;
  u64 *m1r, *m2r, *m1c, *m2c;
  int *cntr, *cntc;
  u64* misc;         // [0..1] delta, [2] done|n_hist, [3..4] counts
  int *listA, *listB;
  uint8_t *rt, *ct;
  int *rbi, *cbi;
};

EdgeWs carve_edges(void* ws, long long E, long long m, long long n) {
  const size_t e = size_t(std::max(E, 1LL)), mm = size_t(std::max(m, 1LL)),
               nn = size_t(std::max(n, 1LL));
  uint8_t* p = static_cast<uint8_t*>(ws);
  auto take = [&](size_t b) { uint8_t* q = p; p += up256(b); return q; };
  EdgeWs w;
  w.beta = reinterpret_cast<double*>(take(e * 8));
  w.rho = reinterpret_cast<double*>(take(e * 8));
  w.belief = reinterpret_cast<double*>(take(e * 8));
  w.m1r = reinterpret_cast<u64*>(take(mm * 8));
  w.m2r = reinterpret_cast<u64*>(take(mm * 8));
  w.m1c = reinterpret_cast<u64*>(take(nn * 8));
  w.m2c = reinterpret_cast<u64*>(take(nn * 8));
  w.cntr = reinterpret_cast<int*>(take(mm * 4));
  w.cntc = reinterpret_cast<int*>(take(nn * 4));
  w.misc = reinterpret_cast<u64*>(take(64));
  w.listA = reinterpret_cast<int*>(take(e * 4));
  w.listB = reinterpret_cast<int*>(take(e * 4));
  w.rt = take(mm);
  w.ct = take(nn);
  w.rbi = reinterpret_cast<int*>(take(mm * 4));
  w.cbi = reinterpret_cast<int*>(take(nn * 4));
  return w;
}

int cuda_err(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(DE_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return DE_OK;
}

int check_edges(const int64_t* ei, const int64_t* ej, long long E, long long m, long long n) {
  if (E < 0 || m < 0 || n < 0) return set_error(DE_ERR_ARG, "negative size");
  if (E > INT_MAX - 1) return set_error(DE_ERR_ARG, "%lld edges above %d", E, INT_MAX - 1);
  if (E > 0 && (!ei || !ej)) return set_error(DE_ERR_ARG, "NULL edge arrays");
  return DE_OK;
}

// Rejects edges whose node index is out of range (blocks for the check).
int validate_idx(const int64_t* a, long long na, const int64_t* b, long long nb, long long E,
                 int* flag, cudaStream_t s) {
  if (E == 0) return DE_OK;
  int host = 0;
  cudaMemsetAsync(flag, 0, sizeof(int), s);
  k_check_idx<<<grid_for(E), 256, 0, s>>>(a, E, na, flag);
  if (b) k_check_idx<<<grid_for(E), 256, 0, s>>>(b, E, nb, flag);
  cudaError_t e = cudaMemcpyAsync(&host, flag, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_error(DE_ERR_CUDA, "index check: %s", cudaGetErrorString(e));
  if (host) return set_error(DE_ERR_ARG, "an edge names a node outside 0..m-1 / 0..n-1");
  return DE_OK;
}

// The greedy decision; blocks until done (checks the remaining count between rounds).
int run_decide(const int64_t* ei, const int64_t* ej, const double* se, const double* belief,
               long long E, long long m, long long n, double lam, int64_t* assign,
               const EdgeWs& w, cudaStream_t s) {
  DecArgs a;
  a.ei = ei; a.ej = ej; a.se = se; a.belief = belief; a.assign = assign;
  a.rbk = w.m1r; a.cbk = w.m1c; a.rbi = w.rbi; a.cbi = w.cbi; a.rt = w.rt; a.ct = w.ct;
  a.list[0] = w.listA; a.list[1] = w.listB;
  a.count = reinterpret_cast<int*>(w.misc + 3);
  a.E = E; a.m = m; a.n = n; a.lam = lam;
  cudaMemsetAsync(a.count, 0, 16, s);
  const int g = grid_for(std::max({E, m, n}));
  k_dec_init<<<g, 256, 0, s>>>(a);
  if (int rc = cuda_err("decision init")) return rc;
  int cur = 0;
  int host_count = 0;
  const long long max_rounds = std::min(m, n) + 2;
  for (long long r = 0; r < max_rounds; r += 4) {
    for (int k = 0; k < 4; ++k) {
      const int ge = grid_for(E);
      k_dec_best<<<ge, 256, 0, s>>>(a, cur);
      k_dec_index<<<ge, 256, 0, s>>>(a, cur);
      k_dec_accept<<<ge, 256, 0, s>>>(a, cur);
      k_dec_keep<<<ge, 256, 0, s>>>(a, cur);
      k_dec_flip<<<1, 1, 0, s>>>(a.count, cur);
      cur ^= 1;
    }
    if (int rc = cuda_err("decision round")) return rc;
    cudaError_t e = cudaMemcpyAsync(&host_count, a.count + cur, sizeof(int),
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
      return set_error(DE_ERR_CUDA, "decision count: %s", cudaGetErrorString(e));
    if (host_count == 0) return DE_OK;
  }
  return set_error(DE_ERR_TIMEOUT, "greedy decision did not finish in %lld rounds", max_rounds);
}

}  // namespace

int masda_edges_dev(const int64_t* ei, const int64_t* ej, const double* se, long long E,
                    long long m, long long n, double lam, double gam, int iters, double damping,
                    double eps, int64_t* assign, double* hist, int* n_hist, double* belief_out,
                    void* ws, size_t bytes, cudaStream_t s) {
  if (int rc = check_edges(ei, ej, E, m, n)) return rc;
  if (iters < 0 || (iters > 0 && (!hist || !n_hist)) || !assign || !ws || (E > 0 && !se))
    return set_error(DE_ERR_ARG, "NULL output, history or workspace");
  const size_t need = masda_edges_ws_bytes(E, m, n);
  if (bytes < need) return set_error(DE_ERR_ARG, "workspace %zu bytes < %zu", bytes, need);
  EdgeWs w = carve_edges(ws, E, m, n);
  if (int rc = validate_idx(ei, m, ej, n, E, reinterpret_cast<int*>(w.misc + 5), s)) return rc;
  BpArgs a;
  a.ei = ei; a.ej = ej; a.se = se; a.beta = w.beta; a.rho = w.rho;
  a.m1r = w.m1r; a.m2r = w.m2r; a.m1c = w.m1c; a.m2c = w.m2c; a.cntr = w.cntr; a.cntc = w.cntc;
  a.delta = w.misc;
  a.done = reinterpret_cast<int*>(w.misc + 2);
  a.hist = hist;
  a.n_hist = n_hist ? n_hist : reinterpret_cast<int*>(w.misc + 2) + 1;
  a.E = E; a.m = m; a.n = n; a.lam = lam; a.gam = gam; a.damping = damping; a.eps = eps;
  const int ge = grid_for(std::max({E, m, n}));
  k_bp_init<<<ge, 256, 0, s>>>(a);
  if (E > 0) {
    k_seg_max<<<grid_for(E), 256, 0, s>>>(w.beta, ei, E, w.m1r, nullptr);
    k_bp_row_second<<<ge, 256, 0, s>>>(a);
    for (int it = 0; it < iters; ++it) {
      k_bp_rho<<<ge, 256, 0, s>>>(a);
      k_bp_col_second<<<ge, 256, 0, s>>>(a);
      k_bp_beta<<<ge, 256, 0, s>>>(a);
      k_bp_row_second<<<ge, 256, 0, s>>>(a);
      k_bp_finish<<<1, 1, 0, s>>>(a, it);
    }
  }
  if (int rc = cuda_err("message passing")) return rc;
  double* belief = belief_out ? belief_out : w.belief;
  k_belief<<<grid_for(E), 256, 0, s>>>(w.beta, w.rho, se, E, belief);
  return run_decide(ei, ej, se, belief, E, m, n, lam, assign, w, s);
}

int masda_decide_dev(const int64_t* ei, const int64_t* ej, const double* se,
                     const double* belief, long long E, long long m, long long n, double lam,
                     int64_t* assign, void* ws, size_t bytes, cudaStream_t s) {
  if (int rc = check_edges(ei, ej, E, m, n)) return rc;
  if (!assign || !ws || (E > 0 && (!se || !belief)))
    return set_error(DE_ERR_ARG, "NULL scores, beliefs, output or workspace");
  const size_t need = masda_edges_ws_bytes(E, m, n);
  if (bytes < need) return set_error(DE_ERR_ARG, "workspace %zu bytes < %zu", bytes, need);
  EdgeWs w = carve_edges(ws, E, m, n);
  if (int rc = validate_idx(ei, m, ej, n, E, reinterpret_cast<int*>(w.misc + 5), s)) return rc;
  return run_decide(ei, ej, se, belief, E, m, n, lam, assign, w, s);
}

int seg_max_excluding_dev(const double* vals, const int64_t* idx, long long E, long long n,
                          double* out, void* ws, size_t bytes, cudaStream_t s) {
  if (E < 0 || n < 0 || (E > 0 && (!vals || !idx || !out)) || !ws)
    return set_error(DE_ERR_ARG, "NULL values, indices, output or workspace");
  const size_t need = up256(size_t(std::max(n, 1LL)) * 8) * 2 +
                      up256(size_t(std::max(n, 1LL)) * 4) + 256;
  if (bytes < need) return set_error(DE_ERR_ARG, "workspace %zu bytes < %zu", bytes, need);
  uint8_t* p = static_cast<uint8_t*>(ws);
  int* flag = reinterpret_cast<int*>(p + need - 256);
  if (int rc = validate_idx(idx, n, nullptr, 0, E, flag, s)) return rc;
  u64* m1 = reinterpret_cast<u64*>(p);
  u64* m2 = reinterpret_cast<u64*>(p + up256(size_t(std::max(n, 1LL)) * 8));
  int* cnt = reinterpret_cast<int*>(p + 2 * up256(size_t(std::max(n, 1LL)) * 8));
  k_seg_reset<<<grid_for(n), 256, 0, s>>>(m1, m2, cnt, n);
  k_seg_max<<<grid_for(E), 256, 0, s>>>(vals, idx, E, m1, nullptr);
  k_seg_second<<<grid_for(E), 256, 0, s>>>(vals, idx, E, m1, m2, cnt, nullptr);
  k_seg_out<<<grid_for(E), 256, 0, s>>>(vals, idx, E, m1, m2, cnt, out);
  return cuda_err("segment max");
}

int hamming_dev(const uint64_t* a, const uint64_t* b, long long n, int32_t* out, cudaStream_t s) {
  if (n < 0 || (n > 0 && (!a || !b || !out))) return set_error(DE_ERR_ARG, "NULL arrays");
  if (n == 0) return DE_OK;
  k_hamming<<<grid_for(n), 256, 0, s>>>(a, b, n, out);
  return cuda_err("hamming");
}

int census_pts_dev(const uint8_t* img, int W, int H, const int32_t* xy, long long n, int hw,
                   int hh, uint64_t* out, uint8_t* ok, cudaStream_t s) {
  if (!img || n < 0 || (n > 0 && (!xy || !out)) || W < 1 || H < 1)
    return set_error(DE_ERR_ARG, "NULL image, points or output");
  if (hw < 0 || hh < 0 || (2 * hw + 1) * (2 * hh + 1) - 1 > 64)
    return set_error(DE_ERR_ARG, "census window %dx%d does not fit 64 bits", 2 * hw + 1,
                     2 * hh + 1);
  if (n == 0) return DE_OK;
  k_census_pts<<<grid_for(n), 256, 0, s>>>(img, W, H, xy, n, hw, hh, out, ok);
  return cuda_err("census at points");
}

int build_problem_dev(const float* pl, const uint64_t* dl, long long m, const float* pr,
                      const uint64_t* dr, long long n, float max_dy, float dmin, float dmax,
                      float sigma_y, float w_y, int bits, float* S, cudaStream_t s) {
  if (m < 0 || n < 0 || (m * n > 0 && (!pl || !dl || !pr || !dr || !S)))
    return set_error(DE_ERR_ARG, "NULL points, descriptors or output");
  if (m * n == 0) return DE_OK;
  k_build_problem<<<grid_for(m * n), 256, 0, s>>>(pl, dl, m, pr, dr, n, max_dy, dmin, dmax,
                                                  sigma_y, w_y, double(bits) / 2.0, S);
  return cuda_err("build problem");
}

int edges_from_matrix_dev(const float* S, long long m, long long n, int64_t* ei, int64_t* ej,
                          double* se, long long cap, int64_t* n_out, void* ws, size_t bytes,
                          cudaStream_t s) {
  if (m < 0 || n < 0 || !n_out || !ws || (m * n > 0 && !S) || (cap > 0 && (!ei || !ej || !se)))
    return set_error(DE_ERR_ARG, "NULL matrix, outputs or workspace");
  if (bytes < up256(size_t(std::max(m, 1LL)) * 8))
    return set_error(DE_ERR_ARG, "workspace too small");
  int64_t* off = static_cast<int64_t*>(ws);
  if (m == 0) return cudaMemsetAsync(n_out, 0, 8, s) == cudaSuccess ? DE_OK
                                                                     : cuda_err("memset");
  k_row_count<<<grid_for(m * 32), 256, 0, s>>>(S, m, n, off);
  k_excl_scan_i64<<<1, 1024, 0, s>>>(off, m, n_out);
  k_row_write<<<grid_for(m * 32), 256, 0, s>>>(S, m, n, off, ei, ej, se, cap);
  return cuda_err("to_edges");
}

long long dense_problem_edges(int W, int H, int dmin, int dmax, int hw, int hh) {
  long long total = 0;
  const long long ny = std::max(0, H - 2 * hh);
  for (int d = dmin; d <= dmax; ++d) total += ny * std::max(0, W - 2 * hw - d);
  return total;
}

int dense_problem_dev(const uint8_t* L, const uint8_t* R, int W, int H, int dmin, int dmax,
                      int hw, int hh, int64_t* ei, int64_t* ej, float* se, long long cap,
                      void* ws, size_t bytes, cudaStream_t s) {
  if (!L || !R || !ws) return set_error(DE_ERR_ARG, "NULL image or workspace");
  if (W < 1 || H < 1 || dmin < 0 || dmax < dmin || dmax - dmin + 1 > kMaxDpBlocks)
    return set_error(DE_ERR_ARG, "disparities %d..%d: need 0 <= dmin <= dmax, at most %d",
                     dmin, dmax, kMaxDpBlocks);
  if (hw < 0 || hh < 0 || (2 * hw + 1) * (2 * hh + 1) - 1 > 64)
    return set_error(DE_ERR_ARG, "census window does not fit 64 bits");
  const long long E = dense_problem_edges(W, H, dmin, dmax, hw, hh);
  if (cap < E || (E > 0 && (!ei || !ej || !se)))
    return set_error(DE_ERR_ARG, "edge capacity %lld < %lld", cap, E);
  const size_t need = 2 * up256(size_t(W) * H * 8);
  if (bytes < need) return set_error(DE_ERR_ARG, "workspace %zu bytes < %zu", bytes, need);
  DpArgs a;
  a.cl = static_cast<const uint64_t*>(ws);
  a.cr = reinterpret_cast<const uint64_t*>(static_cast<uint8_t*>(ws) + up256(size_t(W) * H * 8));
  a.ei = ei; a.ej = ej; a.se = se;
  a.W = W; a.H = H; a.hw = hw; a.hh = hh; a.dmin = dmin; a.nd = dmax - dmin + 1; a.E = E;
  for (int h = 0; h <= 64; ++h) a.tab[h] = float((24.0 - double(h)) / 24.0);
  a.off[0] = 0;
  const long long ny = std::max(0, H - 2 * hh);
  for (int k = 0; k < a.nd; ++k)
    a.off[k + 1] = a.off[k] + ny * std::max(0, W - 2 * hw - (dmin + k));
  const long long px = (long long)W * H;
  k_census_plain<<<grid_for(px), 256, 0, s>>>(L, W, H, hw, hh, const_cast<uint64_t*>(a.cl));
  k_census_plain<<<grid_for(px), 256, 0, s>>>(R, W, H, hw, hh, const_cast<uint64_t*>(a.cr));
  if (E > 0) k_dense_problem<<<grid_for(E), 256, 0, s>>>(a);
  return cuda_err("dense problem");
}

}  // namespace de

// ---- C ABI ----------------------------------------------------------------------------

extern "C" {

int de_masda_edges_workspace_bytes(long long E, long long m, long long n, size_t* bytes) {
  if (!bytes || E < 0 || m < 0 || n < 0) return de::set_error(DE_ERR_ARG, "bad sizes");
  *bytes = de::masda_edges_ws_bytes(E, m, n);
  return DE_OK;
}

int de_masda_edges_dev(const int64_t* ei, const int64_t* ej, const double* se, long long E,
                       long long m, long long n, double lam, double gam, int iters,
                       double damping, double eps, int64_t* assign, double* hist, int* n_hist,
                       double* belief, void* workspace, size_t bytes, void* stream) {
  return de::masda_edges_dev(ei, ej, se, E, m, n, lam, gam, iters, damping, eps, assign, hist,
                             n_hist, belief, workspace, bytes, static_cast<cudaStream_t>(stream));
}

int de_masda_decide_dev(const int64_t* ei, const int64_t* ej, const double* se,
                        const double* belief, long long E, long long m, long long n, double lam,
                        int64_t* assign, void* workspace, size_t bytes, void* stream) {
  return de::masda_decide_dev(ei, ej, se, belief, E, m, n, lam, assign, workspace, bytes,
                              static_cast<cudaStream_t>(stream));
}

int de_seg_max_excluding_dev(const double* vals, const int64_t* idx, long long E, long long n,
                             double* out, void* workspace, size_t bytes, void* stream) {
  return de::seg_max_excluding_dev(vals, idx, E, n, out, workspace, bytes,
                                   static_cast<cudaStream_t>(stream));
}

int de_hamming_dev(const uint64_t* a, const uint64_t* b, long long n, int32_t* out,
                   void* stream) {
  return de::hamming_dev(a, b, n, out, static_cast<cudaStream_t>(stream));
}

int de_census_pts_dev(const uint8_t* img, int W, int H, const int32_t* xy, long long n, int hw,
                      int hh, uint64_t* out, uint8_t* ok, void* stream) {
  return de::census_pts_dev(img, W, H, xy, n, hw, hh, out, ok,
                            static_cast<cudaStream_t>(stream));
}

int de_build_problem_dev(const float* pl, const uint64_t* dl, long long m, const float* pr,
                         const uint64_t* dr, long long n, float max_dy, float dmin, float dmax,
                         float sigma_y, float w_y, int bits, float* S, void* stream) {
  return de::build_problem_dev(pl, dl, m, pr, dr, n, max_dy, dmin, dmax, sigma_y, w_y, bits, S,
                               static_cast<cudaStream_t>(stream));
}

int de_edges_from_matrix_dev(const float* S, long long m, long long n, int64_t* ei,
                             int64_t* ej, double* se, long long cap, int64_t* n_out,
                             void* workspace, size_t bytes, void* stream) {
  return de::edges_from_matrix_dev(S, m, n, ei, ej, se, cap, n_out, workspace, bytes,
                                   static_cast<cudaStream_t>(stream));
}

long long de_dense_problem_edges(int W, int H, int dmin, int dmax, int hw, int hh) {
  if (W < 1 || H < 1 || dmin < 0 || dmax < dmin) return 0;
  return de::dense_problem_edges(W, H, dmin, dmax, hw, hh);
}

int de_dense_problem_dev(const uint8_t* L, const uint8_t* R, int W, int H, int dmin, int dmax,
                         int hw, int hh, int64_t* ei, int64_t* ej, float* se, long long cap,
                         void* workspace, size_t bytes, void* stream) {
  return de::dense_problem_dev(L, R, W, H, dmin, dmax, hw, hh, ei, ej, se, cap, workspace,
                               bytes, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
