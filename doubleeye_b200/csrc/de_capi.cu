// C ABI of the B200 stereo hot path: argument checking, workspace planning, the
// host-built arithmetic tables, the batch descriptor table, and the host-pointer
// context.  See include/doubleeye_b200.h for the contract of every entry point.

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <system_error>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "de_internal.h"

namespace {

thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  const int code = (e == cudaErrorMemoryAllocation) ? DE_ERR_OOM : DE_ERR_CUDA;
  return fail(code, "%s: %s", what, cudaGetErrorString(e));
}

#define DE_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

constexpr size_t kAlign = 256;
inline size_t align_up(size_t v) { return (v + kAlign - 1) & ~(kAlign - 1); }

int census_bits(const de_cfg& c) {
  return (2 * c.census_hw + 1) * (2 * c.census_hh + 1) - 1;
}

int check_cfg(const de_cfg* c) {
  if (!c) return fail(DE_ERR_ARG, "cfg is NULL");
  if (c->dmin < 1) return fail(DE_ERR_ARG, "dmin must be >= 1 (got %d)", c->dmin);
  const int D = c->dmax - c->dmin + 1;
  if (D < 1 || D > DE_MAX_D)
    return fail(DE_ERR_ARG, "disparity count dmax-dmin+1 = %d outside 1..%d", D, DE_MAX_D);
  if (c->census_hw < 1 || c->census_hh < 1 || c->census_hw > 4 || c->census_hh > 4 ||
      census_bits(*c) > 64)
    return fail(DE_ERR_ARG, "census half-window %dx%d unsupported (<= 4, <= 64 bits)",
                c->census_hw, c->census_hh);
  if (!(c->sigma_s > 0.f) || !(c->sigma_r > 0.f))
    return fail(DE_ERR_ARG, "sigma_s and sigma_r must be positive");
  if (c->iters < 0) return fail(DE_ERR_ARG, "iters must be >= 0");
  return DE_OK;
}

int check_dims(int W, int H) {
  if (W < 8 || H < 8 || W > de::kMaxW || H > de::kMaxH)
    return fail(DE_ERR_ARG, "image %dx%d outside 8..%d x 8..%d", W, H, de::kMaxW, de::kMaxH);
  return DE_OK;
}

}  // namespace

namespace de {

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

// Host-built tables, the same expressions as the reference so the values agree bit
// for bit: the filter LUT core/tools/de_dense.cpp:533-546 (float, std::exp), the
// score tables :1201-1223.
void make_dev_cfg(const de_cfg& c, DevCfg* o) {
  std::memset(o, 0, sizeof(*o));
  o->dmin = c.dmin;
  o->iters = c.iters;
  o->hw = c.census_hw;
  o->hh = c.census_hh;
  o->subpixel = c.subpixel != 0;
  o->fit_eq = c.fit_eq != 0;
  o->lrc = c.lrc != 0;
  o->lambda = c.lambda;
  o->gamma = c.gamma;
  o->damping = c.damping;
  o->keep = 1.f - c.damping;
  o->min_margin = c.min_margin;
  o->min_ratio = c.min_ratio;
  o->expire_polls = de::get_expire_polls();
  o->cols_async = de::get_cols_async();
  const int nbits = census_bits(c);
  o->packed = nbits <= 48;
  const int half = nbits / 2;
  for (int h = 0; h <= 2 * half && h < 66; ++h)
    o->tbl[h] = int16_t(((half - h) * 16384) / half);
  const float adc = std::max(0.f, std::min(1.f, c.ad));
  o->wq = int32_t(adc * 1024.f);
  const int T = std::max(1, c.ad_trunc);
  o->trunc = T;
  for (int v = 0; v < 256; ++v)
    o->adt[v] = int16_t(16384 - (2 * 16384 * std::min(v, T)) / T);
  const float kk = -std::sqrt(2.f) / c.sigma_s;
  const float rs = c.sigma_s / c.sigma_r;
  for (int d = 0; d < 256; ++d) {
    const float e = std::exp(kk * (1.f + rs * (float(d) / 255.f)));
    o->rf[d] = uint16_t(std::min(32767.f, e * 32768.f + 0.5f));
  }
}

static int dpad_of(int D) { return (D + 63) & ~63; }

static int cpitch_of(int W) { return (W + 2) & ~1; }
static int apitch_of(int W) { return (W + 8) & ~7; }

size_t pair_workspace_bytes(int W, int H, int D, bool lrc) {
  const size_t WH = size_t(W) * H;
  size_t s = 0;
  s += align_up(size_t(H) * cpitch_of(W) * 8) * 2;    // census words L, R
  s += align_up(size_t(H) * apitch_of(W) * 2);        // ax
  s += align_up(WH * 2);                              // ay
  s += align_up(WH * size_t(dpad_of(D)) * 2);     // filtered volume
  s += align_up(WH * 4) * 3;                      // key0, key1, nb
  if (lrc) s += align_up(WH * 4);                 // reverse-match keys
  return s;
}

void carve_pair(DevPair* p, void* ws, int W, int H, int D, int dmin, bool lrc) {
  const size_t WH = size_t(W) * H;
  uint8_t* c = static_cast<uint8_t*>(ws);
  auto take = [&](size_t bytes) { uint8_t* r = c; c += align_up(bytes); return r; };
  p->cpitch = cpitch_of(W);
  p->apitch = apitch_of(W);
  p->lpad = dmin & 1;
  p->cwL = reinterpret_cast<uint64_t*>(take(size_t(H) * p->cpitch * 8));
  p->cwR = reinterpret_cast<uint64_t*>(take(size_t(H) * p->cpitch * 8));
  p->ax = reinterpret_cast<uint16_t*>(take(size_t(H) * p->apitch * 2));
  p->ay = reinterpret_cast<uint16_t*>(take(WH * 2));
  p->vol = reinterpret_cast<int16_t*>(take(WH * size_t(dpad_of(D)) * 2));
  p->key0 = reinterpret_cast<uint32_t*>(take(WH * 4));
  p->key1 = reinterpret_cast<uint32_t*>(take(WH * 4));
  p->nb = reinterpret_cast<uint32_t*>(take(WH * 4));
  p->rkey = lrc ? reinterpret_cast<uint32_t*>(take(WH * 4)) : nullptr;
  p->W = W;
  p->H = H;
  p->D = D;
  p->Dpad = dpad_of(D);
}

// Copies between pageable and pinned host memory, split over a few threads when
// there is enough to move (one core's memcpy is far below host memory bandwidth).
void parallel_copy(const std::vector<HostCopy>& jobs) {
  size_t total = 0;
  for (const HostCopy& j : jobs) total += j.n;
  const unsigned hc = std::thread::hardware_concurrency();
  const int nt = int(std::min<size_t>({8, hc > 1 ? hc / 2 : 1, total >> 22}));
  if (nt <= 1) {
    for (const HostCopy& j : jobs) std::memcpy(j.dst, j.src, j.n);
    return;
  }
  // cut every copy into pieces of about total / (4 nt) bytes, dealt round-robin
  const size_t piece = std::max<size_t>(size_t(1) << 20, total / (4 * size_t(nt)));
  std::vector<HostCopy> pieces;
  for (const HostCopy& j : jobs)
    for (size_t o = 0; o < j.n; o += piece)
      pieces.push_back({static_cast<uint8_t*>(j.dst) + o, static_cast<const uint8_t*>(j.src) + o,
                        std::min(piece, j.n - o)});
  // Worker t copies pieces t, t + nt, ...; the calling thread does the share of any
  // worker it could not start (no exception leaves this C-ABI path).
  std::vector<std::thread> th;
  th.reserve(nt - 1);
  auto share = [&pieces, nt](int t) {
    for (size_t k = t; k < pieces.size(); k += nt)
      std::memcpy(pieces[k].dst, pieces[k].src, pieces[k].n);
  };
  int started = 1;
  for (int t = 1; t < nt; ++t, ++started) {
    try {
      th.emplace_back(share, t);
    } catch (const std::system_error&) {
      break;
    }
  }
  share(0);
  for (int t = started; t < nt; ++t) share(t);
  for (std::thread& t : th) t.join();
}

}  // namespace de

namespace {

int pair_D(const de_cfg& c, const de_pair& p) {
  const int dmax = p.dmax > 0 ? p.dmax : c.dmax;
  return dmax - c.dmin + 1;
}

int check_pair(const de_cfg& c, const de_pair& p) {
  int rc = check_dims(p.W, p.H);
  if (rc) return rc;
  const int D = pair_D(c, p);
  if (D < 1 || D > DE_MAX_D)
    return fail(DE_ERR_ARG, "pair disparity count %d outside 1..%d", D, DE_MAX_D);
  if (!p.L || !p.R) return fail(DE_ERR_ARG, "pair images are NULL");
  return DE_OK;
}

// Fill one launch set's descriptor table for pairs[first, first+n).
void fill_batch(const de_cfg& c, const de_pair* pairs, int first, int n, uint8_t* ws,
                de::Batch* b, int* err) {
  std::memset(b, 0, sizeof(*b));
  b->n = n;
  b->err = err;
  const int hh = c.census_hh, hw = c.census_hw;
  for (int i = 0; i < n; ++i) {
    const de_pair& p = pairs[first + i];
    const int D = pair_D(c, p);
    de::DevPair& d = b->p[i];
    de::carve_pair(&d, ws, p.W, p.H, D, c.dmin, c.lrc != 0);
    ws += de::pair_workspace_bytes(p.W, p.H, D, c.lrc != 0);
    d.L = p.L;
    d.R = p.R;
    d.disp = p.disp;
    d.margin = p.margin;
    d.conf = p.conf;
    d.cand = p.cand;
    b->maxDpad = std::max(b->maxDpad, d.Dpad);
    const int tiles = ((p.W + 31) / 32) * ((p.H + 7) / 8);
    b->pix_prefix[i + 1] = b->pix_prefix[i] + tiles;
    b->rows_prefix[i + 1] = b->rows_prefix[i] + std::max(0, p.H - 2 * hh);
    b->cols_prefix[i + 1] = b->cols_prefix[i] + std::max(0, p.W - 2 * hw - c.dmin);
    b->solve_prefix[i + 1] = b->solve_prefix[i] + p.H;
  }
}

// Optional stage timing: CUDA events recorded on the launching stream between the
// stages of every de_dense_dev launch set while enabled (the counterpart of the
// reference's event breakdown, core/tools/de_dense_cuda.cu:552-604).
struct StageTimer {
  std::mutex mu;
  bool on = false;
  std::vector<cudaEvent_t> ev;   // groups of 5: before census, rows, cols, solve, after
} g_timer;

void timer_mark(cudaStream_t s, std::vector<cudaEvent_t>* group) {
  cudaEvent_t e;
  if (cudaEventCreate(&e) == cudaSuccess) {
    cudaEventRecord(e, s);
    group->push_back(e);
  }
}

// Streams a batch's parts run on, beside the caller's.  Each thread keeps, per
// device, a few sets of them, each set serving one calling stream at a time (so
// batches issued on different streams, such as a caller's own pipelined streams, do
// not queue behind one another).  A calling stream without a set takes over the set
// used least recently (never one whose streams are part of an open graph capture):
// its streams are reused as they are, so at worst the new caller's parts order
// behind work still queued from the old one.  The table never grows, however many
// streams a caller cycles through; with no set free the batch runs as one launch set.
struct PartStreams {
  cudaStream_t origin = nullptr;
  unsigned long long used = 0;
  cudaStream_t s[4] = {};
  cudaEvent_t fork = nullptr, done[4] = {};
  bool ok = false;
};

PartStreams* part_streams(cudaStream_t origin) {
  constexpr int kSets = 4;
  struct Table { PartStreams set[kSets]; unsigned long long clock = 0; };
  thread_local std::unordered_map<int, Table> tables;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  Table& t = tables[dev];
  PartStreams* g = nullptr;
  for (PartStreams& c : t.set)
    if (c.ok && c.origin == origin) g = &c;
  if (!g) {
    // a set whose streams still belong to an open graph capture is not taken over
    auto capturing = [](const PartStreams& c) {
      for (cudaStream_t x : c.s) {
        cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
        if (x && (cudaStreamIsCapturing(x, &st) != cudaSuccess ||
                  st != cudaStreamCaptureStatusNone)) {
          cudaGetLastError();
          return true;
        }
      }
      return false;
    };
    for (PartStreams& c : t.set) {
      if (!c.ok) { g = &c; break; }
      if ((!g || c.used < g->used) && !capturing(c)) g = &c;
    }
    if (!g) return nullptr;                           // every set busy in a capture
  }
  if (!g->ok) {
    int prio = 0;
    cudaError_t e = cudaStreamGetPriority(origin, &prio);
    if (e == cudaSuccess && !g->fork) e = cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming);
    for (int i = 0; i < 4 && e == cudaSuccess; ++i) {
      if (!g->s[i]) e = cudaStreamCreateWithPriority(&g->s[i], cudaStreamNonBlocking, prio);
      if (e == cudaSuccess && !g->done[i])
        e = cudaEventCreateWithFlags(&g->done[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) { cudaGetLastError(); return nullptr; }   // kept for a retry
    g->ok = true;
  }
  g->origin = origin;
  g->used = ++t.clock;
  return g;
}

// Pairs k, k + parts, k + 2 parts, ... of b, with their work-item prefixes.
void part_batch(const de::Batch& b, int parts, int k, de::Batch* out) {
  de::Batch& g = *out;
  g = b;
  g.n = 0;
  g.maxDpad = 0;
  g.rows_prefix[0] = g.cols_prefix[0] = g.solve_prefix[0] = g.pix_prefix[0] = 0;
  for (int i = k; i < b.n; i += parts) {
    const int j = g.n++;
    g.p[j] = b.p[i];
    g.maxDpad = std::max(g.maxDpad, b.p[i].Dpad);
    g.rows_prefix[j + 1] = g.rows_prefix[j] + (b.rows_prefix[i + 1] - b.rows_prefix[i]);
    g.cols_prefix[j + 1] = g.cols_prefix[j] + (b.cols_prefix[i + 1] - b.cols_prefix[i]);
    g.solve_prefix[j + 1] = g.solve_prefix[j] + (b.solve_prefix[i + 1] - b.solve_prefix[i]);
    g.pix_prefix[j + 1] = g.pix_prefix[j] + (b.pix_prefix[i + 1] - b.pix_prefix[i]);
  }
}

int g_batch_streams = 2;          // parts a batch of several pairs is run as, 1..4

int run_batch(const de_cfg& c, de::Batch& b, cudaStream_t s, int max_parts, bool reg_ring) {
  de::DevCfg dc;
  de::make_dev_cfg(c, &dc);
  if (reg_ring) dc.cols_async = 0;
  if (c.lrc)
    for (int i = 0; i < b.n; ++i)
      DE_CUDA(cudaMemsetAsync(b.p[i].rkey, 0, size_t(b.p[i].W) * b.p[i].H * 4, s));
  std::vector<cudaEvent_t> grp;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cap);
  const bool timed = g_timer.on && cap == cudaStreamCaptureStatusNone;
  // A batch of several pairs runs as up to max_parts parts (pairs taken in turn), each
  // part's census -> rows -> columns -> solve chain on its own stream, so one part's
  // kernel tails overlap another part's work instead of idling SMs between launches.
  // Pairs are independent, so the results are the single chain's.  With stage timing
  // on, the stages run in order on the caller's stream.
  const int parts = std::min(b.n, max_parts);
  PartStreams* ps = (!timed && parts > 1) ? part_streams(s) : nullptr;
  if (ps) {
    thread_local de::Batch sub;
    DE_CUDA(cudaEventRecord(ps->fork, s));
    for (int k = 0; k < parts; ++k) {
      part_batch(b, parts, k, &sub);
      cudaStream_t t = ps->s[k];
      DE_CUDA(cudaStreamWaitEvent(t, ps->fork, 0));
      DE_CUDA(de::launch_census(dc, sub, t));
      DE_CUDA(de::launch_rows(dc, sub, t));
      DE_CUDA(de::launch_cols(dc, sub, t));
      DE_CUDA(de::launch_solve(dc, sub, false, t));
      DE_CUDA(cudaEventRecord(ps->done[k], t));
      DE_CUDA(cudaStreamWaitEvent(s, ps->done[k], 0));
    }
    return DE_OK;
  }
  if (timed) timer_mark(s, &grp);
  DE_CUDA(de::launch_census(dc, b, s));
  if (timed) timer_mark(s, &grp);
  DE_CUDA(de::launch_rows(dc, b, s));
  if (timed) timer_mark(s, &grp);
  DE_CUDA(de::launch_cols(dc, b, s));
  if (timed) timer_mark(s, &grp);
  DE_CUDA(de::launch_solve(dc, b, false, s));
  if (timed) {
    timer_mark(s, &grp);
    std::lock_guard<std::mutex> lk(g_timer.mu);
    if (grp.size() == 5) g_timer.ev.insert(g_timer.ev.end(), grp.begin(), grp.end());
    else for (cudaEvent_t e : grp) cudaEventDestroy(e);
  }
  return DE_OK;
}

}  // namespace

extern "C" {

const char* de_last_error(void) { return g_err; }
const char* de_version(void) { return "doubleeye_b200 0.1 (sm_100a)"; }

void de_cfg_default(de_cfg* c) {
  if (!c) return;
  c->dmin = 1;
  c->dmax = 60;
  c->iters = 0;
  c->sigma_s = 8.f;
  c->sigma_r = 0.20f;
  c->ad = 0.15f;
  c->ad_trunc = 10;
  c->lambda = -0.1f;
  c->gamma = -0.1f;
  c->damping = 0.4f;
  c->min_margin = 0.f;
  c->min_ratio = 0.f;
  c->subpixel = 1;
  c->fit_eq = 1;
  c->lrc = 0;
  c->census_hw = 3;
  c->census_hh = 3;
}

void de_det_cfg_default(de_det_cfg* c) {
  if (!c) return;
  c->grad_window = 3;
  c->cell = 32;
  c->per_cell = 3;
  c->min_response = 1.0f;
  c->min_local_std = 2.0f;
  c->border = 8;
  c->subpixel = 1;
  c->fast_threshold = 8;
  c->nms_radius = 3;
}

void de_match_cfg_default(de_match_cfg* c) {
  if (!c) return;
  c->max_dy = 2.0f;
  c->min_disparity = 1.0f;
  c->max_disparity = 220.0f;
  c->max_candidates = 24;
  c->sigma_y = 1.0f;
  c->w_y = 1.0f;
  c->iterations = 20;
  c->damping = 0.4f;
  c->lambda = 0.0f;
  c->gamma = 0.0f;
  c->converge_eps = 1e-4f;
  c->census_bits = 48;
}

int de_dense_workspace_bytes(const de_cfg* cfg, const de_pair* pairs, int n,
                             size_t* bytes) {
  int rc = check_cfg(cfg);
  if (rc) return rc;
  if (!bytes || n < 0 || (n > 0 && !pairs)) return fail(DE_ERR_ARG, "bad arguments");
  size_t s = de::kStatusBytes;
  for (int i = 0; i < n; ++i) {
    if ((rc = check_pair(*cfg, pairs[i]))) return rc;
    s += de::pair_workspace_bytes(pairs[i].W, pairs[i].H, pair_D(*cfg, pairs[i]),
                                  cfg->lrc != 0);
  }
  *bytes = s;
  return DE_OK;
}

int de_dense_dev(const de_cfg* cfg, const de_pair* pairs, int n, void* workspace,
                 size_t ws_bytes, void* stream) {
  return de::dense_dev(cfg, pairs, n, workspace, ws_bytes, static_cast<cudaStream_t>(stream),
                       g_batch_streams);
}

}  // extern "C"

int de::dense_dev(const de_cfg* cfg, const de_pair* pairs, int n, void* workspace,
                  size_t ws_bytes, cudaStream_t stream, int max_parts, bool reg_ring) {
  size_t need = 0;
  int rc = de_dense_workspace_bytes(cfg, pairs, n, &need);
  if (rc) return rc;
  if (need > ws_bytes || (need && !workspace))
    return fail(DE_ERR_ARG, "workspace %zu bytes, need %zu", ws_bytes, need);
  cudaStream_t s = stream;
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  int* err = reinterpret_cast<int*>(ws);
  ws += de::kStatusBytes;
  DE_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  static de::Batch b;          // large; filled and consumed under the lock
  static std::mutex mu;
  for (int first = 0; first < n; first += de::kMaxBatch) {
    const int m = std::min(de::kMaxBatch, n - first);
    std::lock_guard<std::mutex> lk(mu);
    fill_batch(*cfg, pairs, first, m, ws, &b, err);
    for (int i = 0; i < m; ++i)
      ws += de::pair_workspace_bytes(pairs[first + i].W, pairs[first + i].H,
                                     pair_D(*cfg, pairs[first + i]), cfg->lrc != 0);
    if ((rc = run_batch(*cfg, b, s, max_parts, reg_ring))) return rc;
  }
  return DE_OK;
}

extern "C" {

int de_dense_prior_workspace_bytes(const de_cfg* cfg, const de_pair* pair, size_t* bytes) {
  if (!bytes || !pair) return fail(DE_ERR_ARG, "NULL argument");
  size_t ws = 0;
  int rc = de_dense_workspace_bytes(cfg, pair, 1, &ws);
  if (rc) return rc;
  *bytes = ws + de::prior_ws_bytes(pair->W, pair->H, pair_D(*cfg, *pair));
  return DE_OK;
}

int de_dense_prior_dev(const de_cfg* cfg, const de_pair* pair, const float* prior, int band,
                       void* workspace, size_t ws_bytes, void* stream) {
  size_t need = 0;
  int rc = de_dense_prior_workspace_bytes(cfg, pair, &need);
  if (rc) return rc;
  if (!prior) return fail(DE_ERR_ARG, "prior is NULL");
  if (band < 0 || band > DE_MAX_D) return fail(DE_ERR_ARG, "band %d outside 0..%d", band, DE_MAX_D);
  if (cfg->census_hw != 3 || cfg->census_hh != 3)
    return fail(DE_ERR_ARG, "the prior mask is the reference's 7x7-census path");
  if (need > ws_bytes || !workspace)
    return fail(DE_ERR_ARG, "workspace %zu bytes, need %zu", ws_bytes, need);
  de_cfg c2 = *cfg;
  c2.subpixel = 0;                    // as the reference tool does under a prior
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  int* err = reinterpret_cast<int*>(ws);
  DE_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  static de::Batch b;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  fill_batch(c2, pair, 0, 1, ws + de::kStatusBytes, &b, err);
  uint8_t* pws = ws + de::kStatusBytes +
                 de::pair_workspace_bytes(pair->W, pair->H, pair_D(c2, *pair), c2.lrc != 0);
  de::DevCfg dc;
  de::make_dev_cfg(c2, &dc);
  if (c2.lrc)
    DE_CUDA(cudaMemsetAsync(b.p[0].rkey, 0, size_t(pair->W) * pair->H * 4, s));
  DE_CUDA(de::launch_census(dc, b, s));
  DE_CUDA(de::launch_prior(dc, b, prior, band, pws, s));
  DE_CUDA(de::launch_solve(dc, b, false, s));
  return DE_OK;
}

int de_census_dev(const de_cfg* cfg, const uint8_t* L, const uint8_t* R, int W, int H,
                  uint64_t* cl, uint64_t* cr, uint16_t* ax, uint16_t* ay, void* stream) {
  int rc = check_cfg(cfg);
  if (rc || (rc = check_dims(W, H))) return rc;
  if (!L || !R || !cl || !cr || !ax || !ay) return fail(DE_ERR_ARG, "NULL buffer");
  de::DevCfg dc;
  de::make_dev_cfg(*cfg, &dc);
  dc.packed = 0;                               // plain census words for callers
  static de::Batch b;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  std::memset(&b, 0, sizeof(b));
  b.n = 1;
  b.p[0].L = L; b.p[0].R = R; b.p[0].cwL = cl; b.p[0].cwR = cr; b.p[0].ax = ax;
  b.p[0].ay = ay; b.p[0].W = W; b.p[0].H = H;
  b.p[0].cpitch = W; b.p[0].apitch = W; b.p[0].lpad = 0;
  b.pix_prefix[1] = ((W + 31) / 32) * ((H + 7) / 8);
  DE_CUDA(de::launch_census(dc, b, static_cast<cudaStream_t>(stream)));
  return DE_OK;
}

size_t de_cost_workspace_bytes(int W, int H, int D) {
  return de::kStatusBytes + de::pair_workspace_bytes(W, H, D, false);
}

int de_cost_top2_dev(const de_cfg* cfg, const uint8_t* L, const uint8_t* R, int W, int H,
                     float* cs, int* cd, int* cn, int16_t* cnb, void* workspace,
                     size_t ws_bytes, void* stream) {
  int rc = check_cfg(cfg);
  if (rc || (rc = check_dims(W, H))) return rc;
  if (!L || !R || !cs || !cd || !cn) return fail(DE_ERR_ARG, "NULL buffer");
  const int D = cfg->dmax - cfg->dmin + 1;
  const size_t need = de_cost_workspace_bytes(W, H, D);
  if (ws_bytes < need || !workspace)
    return fail(DE_ERR_ARG, "workspace %zu bytes, need %zu", ws_bytes, need);
  de_cfg c2 = *cfg;
  c2.lrc = 0;
  de::DevCfg dc;
  de::make_dev_cfg(c2, &dc);
  static de::Batch b;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  de_pair p{};
  p.L = L; p.R = R; p.W = W; p.H = H;
  int* err = static_cast<int*>(workspace);
  fill_batch(c2, &p, 0, 1, static_cast<uint8_t*>(workspace) + de::kStatusBytes, &b, err);
  b.p[0].ref_cs = cs; b.p[0].ref_cd = cd; b.p[0].ref_cn = cn; b.p[0].ref_cnb = cnb;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DE_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  DE_CUDA(de::launch_census(dc, b, s));
  DE_CUDA(de::launch_rows(dc, b, s));
  DE_CUDA(de::launch_cols(dc, b, s));
  DE_CUDA(de::launch_export_candidates(dc, b, s));
  return DE_OK;
}

int de_solve_dev(const de_cfg* cfg, int W, int H, const float* cs, const int* cd,
                 const int* cn, const int16_t* cnb, float* disp, float* margin,
                 float* lrc2, void* stream) {
  int rc = check_cfg(cfg);
  if (rc) return rc;
  if (W < 1 || H < 1 || W > de::kMaxW || H > de::kMaxH)   // any row count, one row too
    return fail(DE_ERR_ARG, "candidates %dx%d outside 1..%d x 1..%d", W, H, de::kMaxW, de::kMaxH);
  if (!cs || !cd || !cn || !disp) return fail(DE_ERR_ARG, "NULL buffer");
  de_cfg c2 = *cfg;
  c2.lrc = 0;
  de::DevCfg dc;
  de::make_dev_cfg(c2, &dc);
  static de::Batch b;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  std::memset(&b, 0, sizeof(b));
  b.n = 1;
  de::DevPair& P = b.p[0];
  P.W = W; P.H = H;
  P.ref_cs = const_cast<float*>(cs);
  P.ref_cd = const_cast<int*>(cd);
  P.ref_cn = const_cast<int*>(cn);
  P.ref_cnb = const_cast<int16_t*>(cnb);
  P.disp = disp; P.margin = margin; P.lrc2 = lrc2;
  b.solve_prefix[1] = H;
  DE_CUDA(de::launch_solve(dc, b, true, static_cast<cudaStream_t>(stream)));
  return DE_OK;
}

int de_stage_timing(int enable) {
  std::lock_guard<std::mutex> lk(g_timer.mu);
  g_timer.on = enable != 0;
  return DE_OK;
}

int de_stage_times(float* ms, int n, int* launches) {
  std::lock_guard<std::mutex> lk(g_timer.mu);
  for (int i = 0; i < n; ++i) ms[i] = 0.f;
  int groups = 0;
  cudaError_t err = cudaSuccess;
  for (size_t g = 0; g + 5 <= g_timer.ev.size(); g += 5, ++groups)
    for (int k = 0; k < 4 && k < n; ++k) {
      float t = 0.f;
      cudaError_t e = cudaEventSynchronize(g_timer.ev[g + k + 1]);
      if (e == cudaSuccess) e = cudaEventElapsedTime(&t, g_timer.ev[g + k], g_timer.ev[g + k + 1]);
      if (e != cudaSuccess) err = e;
      ms[k] += t;
    }
  for (cudaEvent_t e : g_timer.ev) cudaEventDestroy(e);
  g_timer.ev.clear();
  if (launches) *launches = groups;
  if (err != cudaSuccess) return cuda_fail(err, "stage timing events");
  return DE_OK;
}

int de_set_param(const char* name, int value) {
  if (!name) return fail(DE_ERR_ARG, "name is NULL");
  if (!std::strcmp(name, "rows_ctas_per_sm")) { de::set_rows_ctas_per_sm(value); return DE_OK; }
  if (!std::strcmp(name, "cols_kt")) { de::set_cols_kt(value); return DE_OK; }
  if (!std::strcmp(name, "cols_pf")) { de::set_cols_pf(value); return DE_OK; }
  if (!std::strcmp(name, "cols_cta")) { de::set_cols_cta(value); return DE_OK; }
  if (!std::strcmp(name, "solve_threads")) { de::set_solve_threads(value); return DE_OK; }
  if (!std::strcmp(name, "expire_wait_polls")) { de::set_expire_polls(value); return DE_OK; }
  if (!std::strcmp(name, "batch_streams")) {
    g_batch_streams = std::min(4, std::max(1, value));
    return DE_OK;
  }
  if (!std::strcmp(name, "cols_async")) { de::set_cols_async(value); return DE_OK; }
  return fail(DE_ERR_ARG, "unknown parameter %s", name);
}

int de_get_param(const char* name, int* value) {
  if (!name || !value) return fail(DE_ERR_ARG, "NULL argument");
  if (!std::strcmp(name, "rows_ctas_per_sm")) { *value = de::get_rows_ctas_per_sm(); return DE_OK; }
  if (!std::strcmp(name, "cols_kt")) { *value = de::get_cols_kt(); return DE_OK; }
  if (!std::strcmp(name, "cols_pf")) { *value = de::get_cols_pf(); return DE_OK; }
  if (!std::strcmp(name, "cols_cta")) { *value = de::get_cols_cta(); return DE_OK; }
  if (!std::strcmp(name, "solve_threads")) { *value = de::get_solve_threads(); return DE_OK; }
  if (!std::strcmp(name, "expire_wait_polls")) { *value = de::get_expire_polls(); return DE_OK; }
  if (!std::strcmp(name, "batch_streams")) { *value = g_batch_streams; return DE_OK; }
  if (!std::strcmp(name, "cols_async")) { *value = de::get_cols_async(); return DE_OK; }
  return fail(DE_ERR_ARG, "unknown parameter %s", name);
}

int de_workspace_status(const void* workspace, void* stream, int* status) {
  if (!status) return fail(DE_ERR_ARG, "NULL argument");
  if (!workspace) {                    // the no-allocation entry point's scratch
    void* head = nullptr;
    if (const int rc = de::noalloc_status_word(&head)) return rc;
    workspace = head;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DE_CUDA(cudaMemcpyAsync(status, workspace, sizeof(int), cudaMemcpyDeviceToHost, s));
  DE_CUDA(cudaStreamSynchronize(s));
  return DE_OK;
}

// confidence(), core/include/doubleeye/dense_solve.hpp:158-166.
float de_confidence(float s1, float s2, float lambda, float lrc, float lrc_tol) {
  if (!(s1 > -1e29f)) return 0.f;
  const float alt = (s2 > -1e29f) ? std::max(s2, lambda) : lambda;
  const float x = std::log(std::max((1.f - alt) / std::max(1.f - s1, 1e-6f), 1e-6f));
  const float logit = 0.692684f + 7.936751f * x;
  const float p = 1.f / (1.f + std::exp(-std::max(-30.f, std::min(30.f, logit))));
  return (lrc > lrc_tol) ? std::min(p, 0.35f) : p;
}

}  // extern "C"

// ---------------------------------------------------------------------------------
// Host-pointer context: pinned staging, device buffers and workspace grown on
// demand, one stream.
struct de_ctx {
  de_cfg cfg;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy = nullptr;                       // downloads beside compute
  cudaStream_t upload = nullptr;                     // uploads beside compute
  static constexpr int kChunks = 5;                  // most chunks a batch is cut into
  // compute streams of a chunked batch, priority falling with the chunk's order
  cudaStream_t cs[kChunks] = {};
  cudaEvent_t ev_in[kChunks] = {}, ev_done[kChunks] = {};
  void* dws = nullptr;        size_t dws_cap = 0;
  void* dio = nullptr;        size_t dio_cap = 0;    // device images + outputs
  void* hio = nullptr;        size_t hio_cap = 0;    // pinned mirror of dio
  // Whether a host pointer was page-locked when last asked.  A stale answer only
  // costs speed: a pageable buffer taken for pinned is copied by the driver's own
  // staging, a pinned one taken for pageable through the mirror.
  std::unordered_map<const void*, bool> pinned;
};

namespace {

int grow_dev(void** p, size_t* cap, size_t need) {
  if (need <= *cap) return DE_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  DE_CUDA(cudaMalloc(p, need));
  *cap = need;
  return DE_OK;
}

int grow_host(void** p, size_t* cap, size_t need) {
  if (need <= *cap) return DE_OK;
  if (*p) cudaFreeHost(*p);
  *p = nullptr;
  *cap = 0;
  DE_CUDA(cudaHostAlloc(p, need, cudaHostAllocDefault));
  *cap = need;
  return DE_OK;
}

// Per-pair offsets inside the I/O block: all inputs first, then all outputs, so one
// copy moves the inputs up and one moves the outputs back.
struct IoLayout { size_t L, R, disp, margin, conf, cand; };
struct IoPlan { std::vector<IoLayout> p; size_t in_end = 0, out_begin = 0, end = 0; };
IoPlan io_plan(const de_pair* hp, int n) {
  IoPlan plan;
  plan.p.resize(n);
  size_t o = 0;
  for (int i = 0; i < n; ++i) {
    const size_t WH = size_t(hp[i].W) * hp[i].H;
    plan.p[i].L = o;  o = align_up(o + WH);
    plan.p[i].R = o;  o = align_up(o + WH);
  }
  plan.in_end = o;
  plan.out_begin = o;
  for (int i = 0; i < n; ++i) {
    const size_t WH = size_t(hp[i].W) * hp[i].H;
    plan.p[i].disp = o;    o = align_up(o + (hp[i].disp ? WH * 4 : 0));
    plan.p[i].margin = o;  o = align_up(o + (hp[i].margin ? WH * 4 : 0));
    plan.p[i].conf = o;    o = align_up(o + (hp[i].conf ? WH : 0));
    plan.p[i].cand = o;    o = align_up(o + (hp[i].cand ? WH * 24 : 0));
  }
  plan.end = o;
  return plan;
}

// Host memory the GPU can reach directly: pinned by cudaHostAlloc or registered.
bool host_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();                                // clear the sticky-free error
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

}  // namespace

extern "C" {

int de_ctx_create(const de_cfg* cfg, int device, de_ctx** out) {
  int rc = check_cfg(cfg);
  if (rc) return rc;
  if (!out) return fail(DE_ERR_ARG, "out is NULL");
  int ndev = 0;
  DE_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(DE_ERR_ARG, "no CUDA device %d", device);
  DE_CUDA(cudaSetDevice(device));
  de_ctx* c = new de_ctx;
  c->cfg = *cfg;
  c->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->upload, cudaStreamNonBlocking);
  int least = 0, greatest = 0;
  if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  for (int i = 0; i < de_ctx::kChunks && e == cudaSuccess; ++i)   // greatest is the lowest number
    e = cudaStreamCreateWithPriority(&c->cs[i], cudaStreamNonBlocking, std::min(greatest + i, least));
  for (int i = 0; i < de_ctx::kChunks && e == cudaSuccess; ++i) {
    e = cudaEventCreateWithFlags(&c->ev_in[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_done[i], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    de_ctx_destroy(c);
    return cuda_fail(e, "creating the context's streams and events");
  }
  *out = c;
  return DE_OK;
}

int de_ctx_destroy(de_ctx* c) {
  if (!c) return DE_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->copy) cudaStreamSynchronize(c->copy);
  if (c->upload) cudaStreamSynchronize(c->upload);
  for (int i = 0; i < de_ctx::kChunks; ++i)
    if (c->cs[i]) cudaStreamSynchronize(c->cs[i]);
  if (c->dws) cudaFree(c->dws);
  if (c->dio) cudaFree(c->dio);
  if (c->hio) cudaFreeHost(c->hio);
  for (int i = 0; i < de_ctx::kChunks; ++i) {
    if (c->ev_in[i]) cudaEventDestroy(c->ev_in[i]);
    if (c->ev_done[i]) cudaEventDestroy(c->ev_done[i]);
  }
  for (int i = 0; i < de_ctx::kChunks; ++i)
    if (c->cs[i]) cudaStreamDestroy(c->cs[i]);
  if (c->upload) cudaStreamDestroy(c->upload);
  if (c->copy) cudaStreamDestroy(c->copy);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return DE_OK;
}

int de_ctx_set_cfg(de_ctx* c, const de_cfg* cfg) {
  if (!c) return fail(DE_ERR_ARG, "ctx is NULL");
  int rc = check_cfg(cfg);
  if (rc) return rc;
  c->cfg = *cfg;
  return DE_OK;
}

int de_ctx_dense_batch(de_ctx* c, const de_pair* hp, int n) {
  if (!c || n < 0 || (n > 0 && !hp)) return fail(DE_ERR_ARG, "bad arguments");
  if (n == 0) return DE_OK;
  DE_CUDA(cudaSetDevice(c->device));
  int rc;
  size_t ws = 0;
  if ((rc = de_dense_workspace_bytes(&c->cfg, hp, n, &ws))) return rc;
  const IoPlan plan = io_plan(hp, n);
  if ((rc = grow_dev(&c->dio, &c->dio_cap, plan.end))) return rc;
  if ((rc = grow_host(&c->hio, &c->hio_cap, plan.end + kAlign))) return rc;
  uint8_t* Hb = static_cast<uint8_t*>(c->hio);
  uint8_t* Db = static_cast<uint8_t*>(c->dio);
  int* hstat = reinterpret_cast<int*>(Hb + plan.end);   // pinned: one status word a chunk
  for (int k = 0; k < de_ctx::kChunks; ++k) hstat[k] = 0;
  auto is_pinned = [&](const void* p) {
    auto it = c->pinned.find(p);
    if (it != c->pinned.end()) return it->second;
    if (c->pinned.size() >= 4096) c->pinned.clear();
    return c->pinned[p] = host_pinned(p);
  };
  // Each host buffer moves by DMA straight from or to the caller's memory when that
  // memory is pinned, else through the context's pinned mirror at the same offset.
  struct Io { void* host; size_t off, bytes; bool pinned; int pair; };
  std::vector<de_pair> dp(n);
  size_t out_bytes = 0;
  for (int i = 0; i < n; ++i) {
    const IoLayout& l = plan.p[i];
    const size_t WH = size_t(hp[i].W) * hp[i].H;
    out_bytes += (hp[i].disp ? WH * 4 : 0) + (hp[i].margin ? WH * 4 : 0) +
                 (hp[i].conf ? WH : 0) + (hp[i].cand ? WH * 24 : 0);
    dp[i] = hp[i];
    dp[i].L = Db + l.L;
    dp[i].R = Db + l.R;
    dp[i].disp = hp[i].disp ? reinterpret_cast<float*>(Db + l.disp) : nullptr;
    dp[i].margin = hp[i].margin ? reinterpret_cast<float*>(Db + l.margin) : nullptr;
    dp[i].conf = hp[i].conf ? Db + l.conf : nullptr;
    dp[i].cand = hp[i].cand ? reinterpret_cast<float*>(Db + l.cand) : nullptr;
  }
  auto inputs = [&](int first, int last) {
    std::vector<Io> v;
    for (int i = first; i < last; ++i) {
      const IoLayout& l = plan.p[i];
      const size_t WH = size_t(hp[i].W) * hp[i].H;
      v.push_back({const_cast<uint8_t*>(hp[i].L), l.L, WH, is_pinned(hp[i].L), i});
      v.push_back({const_cast<uint8_t*>(hp[i].R), l.R, WH, is_pinned(hp[i].R), i});
    }
    return v;
  };
  auto outputs = [&]() {
    std::vector<Io> v;
    for (int i = 0; i < n; ++i) {
      const IoLayout& l = plan.p[i];
      const size_t WH = size_t(hp[i].W) * hp[i].H;
      auto out = [&](void* h, size_t off, size_t bytes) {
        if (h) v.push_back({h, off, bytes, is_pinned(h), i});
      };
      out(hp[i].disp, l.disp, WH * 4);
      out(hp[i].margin, l.margin, WH * 4);
      out(hp[i].conf, l.conf, WH);
      out(hp[i].cand, l.cand, WH * 24);
    }
    return v;
  };
  auto stage = [&](const std::vector<Io>& v) {          // pageable inputs into the mirror
    std::vector<de::HostCopy> jobs;
    for (const Io& io : v)
      if (!io.pinned) jobs.push_back({Hb + io.off, io.host, io.bytes});
    de::parallel_copy(jobs);
  };
  auto move = [&](const Io& io, bool up, cudaStream_t st) -> cudaError_t {
    void* h = io.pinned ? io.host : Hb + io.off;
    return up ? cudaMemcpyAsync(Db + io.off, h, io.bytes, cudaMemcpyHostToDevice, st)
              : cudaMemcpyAsync(h, Db + io.off, io.bytes, cudaMemcpyDeviceToHost, st);
  };
  // Chunks when there is enough to move: chunk k+1's upload (upload stream) and
  // chunk k's download (download stream) run while another chunk computes, so only
  // the first upload and the last download are exposed.  Each chunk computes on its
  // own stream in its own workspace slice, at a priority below the chunk before it:
  // the first chunk runs as if alone and the later ones take the SMs it leaves idle
  // (its tails, its lightly occupied kernels), so chunking costs little device
  // efficiency.  Five chunks from 8 pairs up: small ends (n/8 pairs each) keep the
  // exposed first upload and last download short, and three equal middle chunks
  // finish one after another so their downloads overlap the compute behind them
  // (16 pairs of 848x480: 2, 4, 4, 4, 2).  The first chunk is uploaded and launched
  // before anything else is prepared.
  int bound[de_ctx::kChunks + 1] = {0};
  int nch = 1;
  if (out_bytes >= (size_t(8) << 20) && n >= 8) {
    const int e = std::max(1, n / 8), mid = n - 2 * e;
    const int sizes[5] = {e, (mid + 2) / 3, (mid + 1) / 3, mid / 3, e};
    nch = 5;
    for (int k = 0; k < nch; ++k) bound[k + 1] = bound[k] + sizes[k];
  } else if (out_bytes >= (size_t(8) << 20) && n >= 4) {
    nch = 2;
    bound[1] = (2 * n + 2) / 3;
  }
  bound[nch] = n;
  size_t woff[de_ctx::kChunks + 1] = {0};
  for (int k = 0; k < nch; ++k) {
    size_t wk = 0;
    if ((rc = de_dense_workspace_bytes(&c->cfg, hp + bound[k], bound[k + 1] - bound[k], &wk)))
      return rc;
    woff[k + 1] = woff[k] + wk;
  }
  if ((rc = grow_dev(&c->dws, &c->dws_cap, std::max(ws, woff[nch])))) return rc;
  uint8_t* dws = static_cast<uint8_t*>(c->dws);
  std::vector<Io> outs;
  auto enqueue = [&]() -> int {
    int r;
    const std::vector<Io> in0 = inputs(0, bound[1]);
    stage(in0);
    for (const Io& io : in0) DE_CUDA(move(io, true, c->cs[0]));
    for (int k = 0; k < nch; ++k) {
      cudaStream_t sk = c->cs[k];
      if (k > 0) DE_CUDA(cudaStreamWaitEvent(sk, c->ev_in[k], 0));
      // chunks already overlap one another: each runs as one launch set, with the
      // column kernel's ring in registers (its shared-memory ring, which frees room
      // for a second launch set of the same batch, crowds five concurrent chunks:
      // e2e 4990 -> 5045 pairs/s with the register ring here)
      if ((r = de::dense_dev(&c->cfg, dp.data() + bound[k], bound[k + 1] - bound[k],
                             dws + woff[k], woff[k + 1] - woff[k], sk,
                             nch > 1 ? 1 : g_batch_streams, nch > 1)))
        return r;
      DE_CUDA(cudaMemcpyAsync(&hstat[k], dws + woff[k], sizeof(int), cudaMemcpyDeviceToHost, sk));
      DE_CUDA(cudaEventRecord(c->ev_done[k], sk));
      if (k == 0) {                                   // the other chunks' inputs, now
        for (int j = 1; j < nch; ++j) {
          const std::vector<Io> in = inputs(bound[j], bound[j + 1]);
          stage(in);
          for (const Io& io : in) DE_CUDA(move(io, true, c->upload));
          DE_CUDA(cudaEventRecord(c->ev_in[j], c->upload));
        }
        outs = outputs();
      }
      DE_CUDA(cudaStreamWaitEvent(c->copy, c->ev_done[k], 0));
      for (const Io& io : outs)
        if (io.pair >= bound[k] && io.pair < bound[k + 1]) DE_CUDA(move(io, false, c->copy));
    }
    return DE_OK;
  };
  // whatever was enqueued finishes before the call returns, on success or not
  rc = enqueue();
  cudaError_t e1 = cudaSuccess;
  for (int k = 0; k < de_ctx::kChunks; ++k) {
    const cudaError_t ek = cudaStreamSynchronize(c->cs[k]);
    if (e1 == cudaSuccess) e1 = ek;
  }
  const cudaError_t e2 = cudaStreamSynchronize(c->copy);
  const cudaError_t e3 = cudaStreamSynchronize(c->upload);
  if (rc) return rc;
  if (e1 != cudaSuccess) return cuda_fail(e1, "cudaStreamSynchronize");
  if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamSynchronize");
  if (e3 != cudaSuccess) return cuda_fail(e3, "cudaStreamSynchronize");
  int status = 0;
  for (int k = 0; k < nch && !status; ++k) status = hstat[k];
  if (status) return fail(DE_ERR_TIMEOUT, "a bounded device wait ran out (status %d)", status);
  std::vector<de::HostCopy> jobs;
  for (const Io& io : outs)
    if (!io.pinned) jobs.push_back({io.host, Hb + io.off, io.bytes});
  de::parallel_copy(jobs);
  return DE_OK;
}

int de_ctx_keypoints(de_ctx* c, const uint8_t* L, int W, int H, const de_det_cfg* det,
                     const float* disp, const float* margin, de_kp_disparity* out, int cap,
                     int* n_out, int* n_detected) {
  if (!c || !L || !det || !disp || !n_out || cap < 0 || (cap > 0 && !out))
    return fail(DE_ERR_ARG, "bad arguments");
  DE_CUDA(cudaSetDevice(c->device));
  const size_t WH = size_t(W) * H;
  const size_t ws = de::detect_ws_bytes(W, H, det);
  const int kcap = 1 << 16;
  // device block: L | disp | margin | keypoints | readout | counts
  const size_t oL = 0, oD = align_up(oL + WH), oM = align_up(oD + WH * 4),
               oK = align_up(oM + WH * 4), oR = align_up(oK + size_t(kcap) * 16),
               oN = align_up(oR + size_t(kcap) * 16), end = align_up(oN + 16);
  int rc;
  if ((rc = grow_dev(&c->dws, &c->dws_cap, ws))) return rc;
  if ((rc = grow_dev(&c->dio, &c->dio_cap, end))) return rc;
  if ((rc = grow_host(&c->hio, &c->hio_cap, end))) return rc;
  uint8_t* Hb = static_cast<uint8_t*>(c->hio);
  uint8_t* Db = static_cast<uint8_t*>(c->dio);
  std::memcpy(Hb + oL, L, WH);
  std::memcpy(Hb + oD, disp, WH * 4);
  if (margin) std::memcpy(Hb + oM, margin, WH * 4);
  else std::memset(Hb + oM, 0, WH * 4);
  DE_CUDA(cudaMemcpyAsync(Db, Hb, oK, cudaMemcpyHostToDevice, c->stream));
  de_keypoint* kp = reinterpret_cast<de_keypoint*>(Db + oK);
  int* counts = reinterpret_cast<int*>(Db + oN);
  if ((rc = de::detect_fast_dev(Db + oL, W, H, det, kp, kcap, counts, c->dws, c->dws_cap,
                                c->stream)))
    return rc;
  if ((rc = de::kp_readout_dev(kp, kcap, counts, reinterpret_cast<const float*>(Db + oD),
                               reinterpret_cast<const float*>(Db + oM), W, H,
                               reinterpret_cast<de_kp_disparity*>(Db + oR), kcap, counts + 1,
                               c->stream)))
    return rc;
  DE_CUDA(cudaMemcpyAsync(Hb + oR, Db + oR, end - oR, cudaMemcpyDeviceToHost, c->stream));
  DE_CUDA(cudaStreamSynchronize(c->stream));
  int cnt[2];
  std::memcpy(cnt, Hb + oN, sizeof(cnt));
  if (cnt[0] < 0) return fail(DE_ERR_TIMEOUT, "keypoint suppression did not settle");
  if (n_detected) *n_detected = cnt[0];
  *n_out = cnt[1];
  std::memcpy(out, Hb + oR, size_t(std::min(cnt[1], cap)) * sizeof(de_kp_disparity));
  return DE_OK;
}

int de_ctx_dense_prior(de_ctx* c, const uint8_t* L, const uint8_t* R, int W, int H,
                       const float* prior, int band, float* disp, float* margin,
                       uint8_t* conf, float* cand) {
  if (!c || !L || !R || !prior) return fail(DE_ERR_ARG, "bad arguments");
  const size_t WH = size_t(W) * H;
  for (size_t i = 0; i < WH; ++i)
    if (!std::isfinite(prior[i]))
      return fail(DE_ERR_ARG, "the prior has holes (non-finite values); fill them first");
  DE_CUDA(cudaSetDevice(c->device));
  de_pair p{};
  p.L = L; p.R = R; p.W = W; p.H = H;
  size_t ws = 0;
  int rc = de_dense_prior_workspace_bytes(&c->cfg, &p, &ws);
  if (rc) return rc;
  const size_t oL = 0, oR = align_up(WH), oP = align_up(oR + WH), oD = align_up(oP + WH * 4),
               oM = align_up(oD + WH * 4), oC = align_up(oM + WH * 4),
               oX = align_up(oC + WH), end = align_up(oX + (cand ? WH * 24 : 0));
  if ((rc = grow_dev(&c->dws, &c->dws_cap, ws))) return rc;
  if ((rc = grow_dev(&c->dio, &c->dio_cap, end))) return rc;
  if ((rc = grow_host(&c->hio, &c->hio_cap, end))) return rc;
  uint8_t* Hb = static_cast<uint8_t*>(c->hio);
  uint8_t* Db = static_cast<uint8_t*>(c->dio);
  std::memcpy(Hb + oL, L, WH);
  std::memcpy(Hb + oR, R, WH);
  std::memcpy(Hb + oP, prior, WH * 4);
  DE_CUDA(cudaMemcpyAsync(Db, Hb, oD, cudaMemcpyHostToDevice, c->stream));
  de_pair dp{};
  dp.L = Db + oL; dp.R = Db + oR; dp.W = W; dp.H = H;
  dp.disp = reinterpret_cast<float*>(Db + oD);
  dp.margin = reinterpret_cast<float*>(Db + oM);
  dp.conf = Db + oC;
  dp.cand = cand ? reinterpret_cast<float*>(Db + oX) : nullptr;
  if ((rc = de_dense_prior_dev(&c->cfg, &dp, reinterpret_cast<const float*>(Db + oP), band,
                               c->dws, c->dws_cap, c->stream)))
    return rc;
  DE_CUDA(cudaMemcpyAsync(Hb + oD, Db + oD, end - oD, cudaMemcpyDeviceToHost, c->stream));
  int status = 0;
  DE_CUDA(cudaMemcpyAsync(&status, c->dws, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  DE_CUDA(cudaStreamSynchronize(c->stream));
  if (status) return fail(DE_ERR_TIMEOUT, "a bounded device wait ran out (status %d)", status);
  if (disp) std::memcpy(disp, Hb + oD, WH * 4);
  if (margin) std::memcpy(margin, Hb + oM, WH * 4);
  if (conf) std::memcpy(conf, Hb + oC, WH);
  if (cand) std::memcpy(cand, Hb + oX, WH * 24);
  return DE_OK;
}

int de_ctx_dense(de_ctx* c, const uint8_t* L, const uint8_t* R, int W, int H, float* disp,
                 float* margin, uint8_t* conf, float* cand) {
  de_pair p{};
  p.L = L; p.R = R; p.W = W; p.H = H; p.dmax = 0;
  p.disp = disp; p.margin = margin; p.conf = conf; p.cand = cand;
  return de_ctx_dense_batch(c, &p, 1);
}

}  // extern "C"

// ---------------------------------------------------------------------------------
// Host-pointer forms of the stage and sparse entry points: inputs copied up into the
// context's I/O block, the device entry point run on the context's stream, outputs
// copied back; each call has finished when it returns.
namespace {

struct Carve {                                       // consecutive 256-byte aligned slices
  size_t end = 0;
  size_t take(size_t n) {
    const size_t o = end;
    end = align_up(end + std::max<size_t>(n, 1));
    return o;
  }
};

int ctx_io(de_ctx* c, size_t io_bytes, size_t ws_bytes) {
  DE_CUDA(cudaSetDevice(c->device));
  if (int rc = grow_dev(&c->dio, &c->dio_cap, io_bytes)) return rc;
  return grow_dev(&c->dws, &c->dws_cap, std::max<size_t>(ws_bytes, 256));
}

int ctx_up(de_ctx* c, size_t off, const void* src, size_t n) {
  if (!n) return DE_OK;
  DE_CUDA(cudaMemcpyAsync(static_cast<uint8_t*>(c->dio) + off, src, n, cudaMemcpyHostToDevice,
                          c->stream));
  return DE_OK;
}

int ctx_down(de_ctx* c, void* dst, size_t off, size_t n) {
  if (!n || !dst) return DE_OK;
  DE_CUDA(cudaMemcpyAsync(dst, static_cast<uint8_t*>(c->dio) + off, n, cudaMemcpyDeviceToHost,
                          c->stream));
  return DE_OK;
}

template <typename T = void>
T* dptr(de_ctx* c, size_t off) {
  return reinterpret_cast<T*>(static_cast<uint8_t*>(c->dio) + off);
}

}  // namespace

extern "C" {

int de_ctx_census(de_ctx* c, const uint8_t* img, int W, int H, int hw, int hh,
                  uint64_t* bits) {
  if (!c || !img || !bits) return fail(DE_ERR_ARG, "NULL argument");
  if (int rc = check_dims(W, H)) return rc;
  const size_t WH = size_t(W) * H;
  Carve k;
  const size_t oi = k.take(WH), ob = k.take(WH * 8), ob2 = k.take(WH * 8);
  const size_t oax = k.take(WH * 2), oay = k.take(WH * 2);
  if (int rc = ctx_io(c, k.end, 0)) return rc;
  de_cfg cfg = c->cfg;
  cfg.census_hw = hw;
  cfg.census_hh = hh;
  int rc = ctx_up(c, oi, img, WH);
  if (!rc) rc = de_census_dev(&cfg, dptr<uint8_t>(c, oi), dptr<uint8_t>(c, oi), W, H,
                              dptr<uint64_t>(c, ob), dptr<uint64_t>(c, ob2),
                              dptr<uint16_t>(c, oax), dptr<uint16_t>(c, oay), c->stream);
  if (!rc) rc = ctx_down(c, bits, ob, WH * 8);
  if (rc) return rc;
  DE_CUDA(cudaStreamSynchronize(c->stream));
  return DE_OK;
}

int de_ctx_census_at(de_ctx* c, const uint8_t* img, int W, int H, const de_keypoint* kp,
                     int n, int hw, int hh, uint64_t* desc, uint8_t* ok) {
  if (!c || !img || n < 0 || (n > 0 && (!kp || !desc))) return fail(DE_ERR_ARG, "bad argument");
  if (W < 1 || H < 1) return fail(DE_ERR_ARG, "image %dx%d", W, H);
  if (n == 0) return DE_OK;
  const size_t WH = size_t(W) * H;
  Carve k;
  const size_t oi = k.take(WH), ok_ = k.take(sizeof(de_keypoint) * n);
  const size_t od = k.take(8 * size_t(n)), oo = k.take(size_t(n));
  if (int rc = ctx_io(c, k.end, 0)) return rc;
  int rc = ctx_up(c, oi, img, WH);
  if (!rc) rc = ctx_up(c, ok_, kp, sizeof(de_keypoint) * n);
  if (!rc) rc = de_census_at_dev(dptr<uint8_t>(c, oi), W, H, dptr<de_keypoint>(c, ok_), n,
                                 nullptr, hw, hh, dptr<uint64_t>(c, od), dptr<uint8_t>(c, oo),
                                 c->stream);
  if (!rc) rc = ctx_down(c, desc, od, 8 * size_t(n));
  if (!rc) rc = ctx_down(c, ok, oo, size_t(n));
  if (rc) return rc;
  DE_CUDA(cudaStreamSynchronize(c->stream));
  return DE_OK;
}

int de_ctx_detect_fast(de_ctx* c, const uint8_t* img, int W, int H, const de_det_cfg* cfg,
                       de_keypoint* out, int cap, int* n) {
  if (!c || !img || !cfg || !n || cap < 0 || (cap > 0 && !out))
    return fail(DE_ERR_ARG, "bad argument");
  size_t ws = 0;
  if (int rc = de_detect_workspace_bytes(W, H, cfg, &ws)) return rc;
  const size_t WH = size_t(W) * H;
  Carve k;
  const size_t oi = k.take(WH), oo = k.take(sizeof(de_keypoint) * size_t(std::max(cap, 1)));
  const size_t on = k.take(sizeof(int));
  if (int rc = ctx_io(c, k.end, ws)) return rc;
  int rc = ctx_up(c, oi, img, WH);
  if (!rc) rc = de_detect_fast_dev(dptr<uint8_t>(c, oi), W, H, cfg, dptr<de_keypoint>(c, oo),
                                   cap, dptr<int>(c, on), c->dws, c->dws_cap, c->stream);
  if (!rc) rc = ctx_down(c, n, on, sizeof(int));
  if (rc) return rc;
  DE_CUDA(cudaStreamSynchronize(c->stream));
  if (*n < 0) return fail(DE_ERR_UNSUPPORTED, "keypoint suppression exceeded its work bound");
  const int got = std::min(*n, cap);
  if (got > 0) {
    DE_CUDA(cudaMemcpy(out, dptr(c, oo), sizeof(de_keypoint) * size_t(got),
                       cudaMemcpyDeviceToHost));
  }
  return DE_OK;
}

int de_ctx_match_masda(de_ctx* c, const de_keypoint* kl, const uint64_t* dl, int nl,
                       const de_keypoint* kr, const uint64_t* dr, int nr,
                       const de_match_cfg* cfg, const de_match_prior* prior, de_match* out,
                       int cap, int* n_out, de_match_stats* stats) {
  if (!c || !cfg || !n_out || nl < 0 || nr < 0 || cap < 0 || (cap > 0 && !out))
    return fail(DE_ERR_ARG, "bad argument");
  size_t ws = 0;
  if (int rc = de_match_workspace_bytes(nl, nr, cfg, &ws)) return rc;
  Carve k;
  const size_t okl = k.take(sizeof(de_keypoint) * nl), odl = k.take(8 * size_t(nl));
  const size_t okr = k.take(sizeof(de_keypoint) * nr), odr = k.take(8 * size_t(nr));
  const size_t oout = k.take(sizeof(de_match) * size_t(std::max(cap, 1)));
  const size_t on = k.take(sizeof(int)), ost = k.take(sizeof(de_match_stats));
  const size_t pn = 4 * size_t(nl);
  const size_t pcd = k.take(pn), pcs = k.take(pn), psd = k.take(pn), pss = k.take(pn);
  if (int rc = ctx_io(c, k.end, ws)) return rc;
  int rc = ctx_up(c, okl, kl, sizeof(de_keypoint) * nl);
  if (!rc) rc = ctx_up(c, odl, dl, 8 * size_t(nl));
  if (!rc) rc = ctx_up(c, okr, kr, sizeof(de_keypoint) * nr);
  if (!rc) rc = ctx_up(c, odr, dr, 8 * size_t(nr));
  de_match_prior dp{};
  if (!rc && prior) {
    dp.w_coarse = prior->w_coarse;
    dp.w_smooth = prior->w_smooth;
    if (prior->coarse_sd) {
      if (!prior->coarse_d) return fail(DE_ERR_ARG, "coarse prior sigma without disparities");
      rc = ctx_up(c, pcd, prior->coarse_d, pn);
      if (!rc) rc = ctx_up(c, pcs, prior->coarse_sd, pn);
      dp.coarse_d = dptr<float>(c, pcd);
      dp.coarse_sd = dptr<float>(c, pcs);
    }
    if (!rc && prior->smooth_sd) {
      if (!prior->smooth_d) return fail(DE_ERR_ARG, "smooth prior sigma without disparities");
      rc = ctx_up(c, psd, prior->smooth_d, pn);
      if (!rc) rc = ctx_up(c, pss, prior->smooth_sd, pn);
      dp.smooth_d = dptr<float>(c, psd);
      dp.smooth_sd = dptr<float>(c, pss);
    }
  }
  if (!rc) rc = de_match_masda_prior_dev(dptr<de_keypoint>(c, okl), dptr<uint64_t>(c, odl), nl,
                                         nullptr, dptr<de_keypoint>(c, okr),
                                         dptr<uint64_t>(c, odr), nr, nullptr, cfg,
                                         prior ? &dp : nullptr, dptr<de_match>(c, oout), cap,
                                         dptr<int>(c, on), dptr<de_match_stats>(c, ost), c->dws,
                                         c->dws_cap, c->stream);
  if (!rc) rc = ctx_down(c, n_out, on, sizeof(int));
  if (!rc) rc = ctx_down(c, stats, ost, sizeof(de_match_stats));
  if (rc) return rc;
  DE_CUDA(cudaStreamSynchronize(c->stream));
  const int got = std::min(*n_out, cap);
  if (got > 0) {
    DE_CUDA(cudaMemcpy(out, dptr(c, oout), sizeof(de_match) * size_t(got),
                       cudaMemcpyDeviceToHost));
  }
  return DE_OK;
}

int de_ctx_solve(de_ctx* c, const de_cfg* cfg, int W, int H, const float* cs, const int* cd,
                 const int* cn, const int16_t* cnb, float* disp, float* margin, float* lrc2) {
  if (!c || !cs || !cd || !cn || !disp) return fail(DE_ERR_ARG, "NULL buffer");
  if (W < 1 || H < 1) return fail(DE_ERR_ARG, "candidates %dx%d", W, H);
  const size_t WH = size_t(W) * H;
  Carve k;
  const size_t ocs = k.take(WH * 8), ocd = k.take(WH * 8), ocn = k.take(WH * 4);
  const size_t onb = k.take(WH * 4), od = k.take(WH * 4), om = k.take(WH * 4);
  const size_t ol = k.take(WH * 4);
  if (int rc = ctx_io(c, k.end, 0)) return rc;
  int rc = ctx_up(c, ocs, cs, WH * 8);
  if (!rc) rc = ctx_up(c, ocd, cd, WH * 8);
  if (!rc) rc = ctx_up(c, ocn, cn, WH * 4);
  if (!rc && cnb) rc = ctx_up(c, onb, cnb, WH * 4);
  if (!rc) rc = de_solve_dev(cfg, W, H, dptr<float>(c, ocs), dptr<int>(c, ocd),
                             dptr<int>(c, ocn), cnb ? dptr<int16_t>(c, onb) : nullptr,
                             dptr<float>(c, od), dptr<float>(c, om),
                             lrc2 ? dptr<float>(c, ol) : nullptr, c->stream);
  if (!rc) rc = ctx_down(c, disp, od, WH * 4);
  if (!rc) rc = ctx_down(c, margin, om, WH * 4);
  if (!rc) rc = ctx_down(c, lrc2, ol, WH * 4);
  if (rc) return rc;
  DE_CUDA(cudaStreamSynchronize(c->stream));
  return DE_OK;
}

}  // extern "C"
