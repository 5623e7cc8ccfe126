// Serving: a request loop that matches stereo pairs arriving from many camera
// streams, batching whatever is waiting into the dense pipeline as device memory and
// launch slots free up.
//
// The reference's live path is one process per camera pair handling one frame at a
// time (core/tools/de_dense_cuda.cu:670-770, "DEIR" pairs in, "DEDD" maps out).  Here
// one server owns the device:
//   * requests (a left/right pair of any supported size, tagged with its camera
//     stream) are submitted from any thread and copied into the request;
//   * a worker thread admits waiting requests, first come first served, into one of
//     several lanes (a CUDA stream with a fixed device arena and a pinned mirror,
//     sized from the HBM budget at creation: nothing is allocated per request), as
//     many as fit the lane's arena and the batch limit, and launches them as one
//     batched pipeline; while one lane computes, the next lane is filled from what
//     arrived meanwhile (continuous batching across lanes);
//   * completion is signalled from the stream (a host callback), results are copied
//     out of the pinned mirror, and per-request latency (submit to result) is kept for
//     the p50/p99 report;
//   * each camera stream keeps device state: its last two disparity maps (the frame
//     just delivered and the one in flight), readable without a host round trip by
//     device consumers and on request by the host;
//   * results are those of the plain pipeline bit for bit: batching changes which
//     pairs share a launch, never the arithmetic (each pair's work is independent).
// The DEDD encoding of the live path (Q4 int16 disparity, -32768 where the matcher
// declined, u8 confidence zeroed there) is produced on the device with the outputs.

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "de_internal.h"

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

namespace de {
namespace {

// DEDD planes (core/tools/de_dense_cuda.cu:729-746): Q4 disparity, lround(d * 16) for
// finite d > 0, else -32768; confidence 0 wherever the disparity is -32768.
__global__ void k_dedd(const float* disp, const uint8_t* conf, long long n, int16_t* q4,
                       uint8_t* qconf) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float d = disp[i];
    const bool ok = d > 0.f && isfinite(d);
    q4[i] = ok ? int16_t(lroundf(d * 16.0f)) : int16_t(-32768);
    if (qconf) qconf[i] = ok ? (conf ? conf[i] : uint8_t(0)) : uint8_t(0);
  }
}

}  // namespace

int dedd_encode_dev(const float* disp, const uint8_t* conf, int W, int H, int16_t* q4,
                    uint8_t* qconf, cudaStream_t s) {
  if (!disp || !q4 || W < 1 || H < 1) return set_error(DE_ERR_ARG, "NULL plane or bad size");
  const long long n = (long long)W * H;
  k_dedd<<<int(std::min<long long>((n + 255) / 256, 148 * 8)), 256, 0, s>>>(disp, conf, n, q4,
                                                                          qconf);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(DE_ERR_CUDA, "dedd: %s", cudaGetErrorString(e));
  return DE_OK;
}

}  // namespace de

namespace {

struct Req {
  uint64_t ticket = 0;
  int stream = 0, W = 0, H = 0, dmax = 0;
  unsigned planes = 0;                 // DE_PLANE_* the client will read
  std::vector<uint8_t> L, R;
  std::vector<float> disp, margin;
  std::vector<uint8_t> conf, qconf;
  std::vector<int16_t> q4;
  double t_submit = 0, t_launch = 0, t_done = 0;
  int status = 1;                      // 1 pending, 0 done, < 0 error code
};

struct Slot {                          // one request's place in a lane's arena
  size_t L, R, disp, margin, conf, q4, qconf;
};

struct Lane {
  cudaStream_t s = nullptr;
  uint8_t* dev = nullptr;              // I/O block, then the pipeline workspace
  size_t dev_cap = 0;
  uint8_t* pin = nullptr;              // pinned mirror of the I/O block
  size_t pin_cap = 0;
  std::vector<Req*> batch;
  std::vector<Slot> slots;
  size_t in_end = 0, out_begin = 0, out_end = 0;
  bool busy = false;
  bool finished = false;               // set by the stream callback
  struct de_server* owner = nullptr;
};

struct StreamState {
  int W = 0, H = 0;
  float* buf[2] = {nullptr, nullptr};  // last two disparity maps on the device
  cudaEvent_t ev[2] = {nullptr, nullptr};
  uint64_t frames = 0;                 // frames launched
};

}  // namespace

struct de_server {
  de_cfg cfg{};
  de_server_cfg scfg{};
  int device = 0;
  std::vector<Lane> lanes;
  std::mutex mu;
  std::condition_variable cv_work;     // new request, finished lane or stop
  std::condition_variable cv_done;     // a request finished
  std::deque<Req*> pending;
  std::unordered_map<uint64_t, Req*> reqs;
  uint64_t next_ticket = 1;
  std::unordered_map<int, StreamState> streams;
  std::vector<Req*> pool;              // finished requests kept with their buffers
  std::vector<double> lat;
  uint64_t batches = 0, batched_pairs = 0, completed = 0, failed = 0;
  size_t max_pending = 0;
  bool stop = false;
  int fatal = 0;
  std::thread worker;
};

namespace {

void CUDART_CB lane_done(void* p) {
  Lane* l = static_cast<Lane*>(p);
  de_server* sv = l->owner;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    l->finished = true;
  }
  sv->cv_work.notify_all();
}

// Arena layout of a prospective batch; returns the device bytes needed (I/O block +
// workspace), and in *out_end the I/O block's size (the pinned mirror's share, plus
// 256 bytes for the status word).
size_t plan_batch(const de_server* sv, const std::vector<Req*>& b, std::vector<Slot>* slots,
                  size_t* in_end, size_t* out_begin, size_t* out_end, size_t* ws_bytes) {
  std::vector<Slot> s(b.size());
  size_t o = 0;
  for (size_t i = 0; i < b.size(); ++i) {
    const size_t WH = size_t(b[i]->W) * b[i]->H;
    s[i].L = o;  o = align256(o + WH);
    s[i].R = o;  o = align256(o + WH);
  }
  const size_t ie = o;
  for (size_t i = 0; i < b.size(); ++i) {
    const size_t WH = size_t(b[i]->W) * b[i]->H;
    s[i].disp = o;    o = align256(o + WH * 4);
    s[i].margin = o;  o = align256(o + WH * 4);
    s[i].conf = o;    o = align256(o + WH);
    s[i].q4 = o;      o = align256(o + WH * 2);
    s[i].qconf = o;   o = align256(o + WH);
  }
  const size_t oe = o;
  std::vector<de_pair> pairs(b.size());
  for (size_t i = 0; i < b.size(); ++i) {
    pairs[i] = de_pair{};
    pairs[i].L = pairs[i].R = reinterpret_cast<const uint8_t*>(1);
    pairs[i].W = b[i]->W;
    pairs[i].H = b[i]->H;
    pairs[i].dmax = b[i]->dmax;
  }
  size_t ws = 0;
  if (de_dense_workspace_bytes(&sv->cfg, pairs.data(), int(pairs.size()), &ws)) return ~size_t(0);
  if (slots) *slots = std::move(s);
  if (in_end) *in_end = ie;
  if (out_begin) *out_begin = ie;
  if (out_end) *out_end = oe;
  if (ws_bytes) *ws_bytes = ws;
  return align256(oe) + ws;
}

// Enqueues one batch on a free lane.  Called by the worker without the lock held;
// the requests are already owned by the lane.
int launch(de_server* sv, Lane& l) {
  size_t ws = 0;
  plan_batch(sv, l.batch, &l.slots, &l.in_end, &l.out_begin, &l.out_end, &ws);
  const size_t ws_off = align256(l.out_end);
  std::vector<de_pair> dp(l.batch.size());
  std::vector<de::HostCopy> jobs;
  for (size_t i = 0; i < l.batch.size(); ++i) {
    Req* r = l.batch[i];
    const Slot& s = l.slots[i];
    const size_t WH = size_t(r->W) * r->H;
    jobs.push_back({l.pin + s.L, r->L.data(), WH});
    jobs.push_back({l.pin + s.R, r->R.data(), WH});
    dp[i] = de_pair{};
    dp[i].L = l.dev + s.L;
    dp[i].R = l.dev + s.R;
    dp[i].W = r->W;
    dp[i].H = r->H;
    dp[i].dmax = r->dmax;
    dp[i].disp = reinterpret_cast<float*>(l.dev + s.disp);
    dp[i].margin = reinterpret_cast<float*>(l.dev + s.margin);
    dp[i].conf = l.dev + s.conf;
    r->t_launch = now_ms();
  }
  de::parallel_copy(jobs);
  cudaError_t e = cudaMemcpyAsync(l.dev, l.pin, l.in_end, cudaMemcpyHostToDevice, l.s);
  if (e != cudaSuccess) return de::set_error(DE_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
  int rc = de_dense_dev(&sv->cfg, dp.data(), int(dp.size()), l.dev + ws_off, ws, l.s);
  if (rc) return rc;
  for (size_t i = 0; i < l.batch.size(); ++i) {
    Req* r = l.batch[i];
    const Slot& s = l.slots[i];
    rc = de::dedd_encode_dev(reinterpret_cast<float*>(l.dev + s.disp), l.dev + s.conf, r->W,
                             r->H, reinterpret_cast<int16_t*>(l.dev + s.q4), l.dev + s.qconf,
                             l.s);
    if (rc) return rc;
    // per-stream device state: this frame's disparity into the stream's next buffer
    std::lock_guard<std::mutex> lk(sv->mu);
    StreamState* st = &sv->streams[r->stream];
    const size_t bytes = size_t(r->W) * r->H * 4;
    if (st->W != r->W || st->H != r->H) {
      for (int k = 0; k < 2; ++k) {
        if (st->buf[k]) cudaFree(st->buf[k]);
        st->buf[k] = nullptr;
        if (!st->ev[k]) cudaEventCreateWithFlags(&st->ev[k], cudaEventDisableTiming);
      }
      e = cudaMalloc(&st->buf[0], bytes);
      if (e == cudaSuccess) e = cudaMalloc(&st->buf[1], bytes);
      if (e != cudaSuccess)
        return de::set_error(DE_ERR_OOM, "stream state: %s", cudaGetErrorString(e));
      st->W = r->W;
      st->H = r->H;
    }
    const int k = int(st->frames & 1);
    e = cudaMemcpyAsync(st->buf[k], l.dev + s.disp, bytes, cudaMemcpyDeviceToDevice, l.s);
    if (e == cudaSuccess) e = cudaEventRecord(st->ev[k], l.s);
    if (e != cudaSuccess) return de::set_error(DE_ERR_CUDA, "state: %s", cudaGetErrorString(e));
    ++st->frames;
  }
  // only the planes each request asked for come back
  for (size_t i = 0; i < l.batch.size() && e == cudaSuccess; ++i) {
    const Req* r = l.batch[i];
    const Slot& s = l.slots[i];
    const size_t WH = size_t(r->W) * r->H;
    const struct { unsigned bit; size_t off, bytes; } planes[] = {
        {DE_PLANE_DISP, s.disp, WH * 4}, {DE_PLANE_MARGIN, s.margin, WH * 4},
        {DE_PLANE_CONF, s.conf, WH}, {DE_PLANE_Q4, s.q4, WH * 2}, {DE_PLANE_QCONF, s.qconf, WH}};
    for (const auto& pl : planes)
      if ((r->planes & pl.bit) && e == cudaSuccess)
        e = cudaMemcpyAsync(l.pin + pl.off, l.dev + pl.off, pl.bytes, cudaMemcpyDeviceToHost, l.s);
  }
  // the pipeline's status word (set by a bounded device wait that ran out)
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(l.pin + align256(l.out_end), l.dev + ws_off, sizeof(int),
                        cudaMemcpyDeviceToHost, l.s);
  if (e == cudaSuccess) e = cudaLaunchHostFunc(l.s, lane_done, &l);
  if (e != cudaSuccess) return de::set_error(DE_ERR_CUDA, "download: %s", cudaGetErrorString(e));
  return DE_OK;
}

// Copies a finished lane's results into its requests.  Lock held.
void deliver(de_server* sv, Lane& l) {
  int word = 0;
  std::memcpy(&word, l.pin + align256(l.out_end), sizeof(int));
  const int status = word ? DE_ERR_TIMEOUT : 0;
  const double t = now_ms();
  for (size_t i = 0; i < l.batch.size(); ++i) {
    Req* r = l.batch[i];
    const Slot& s = l.slots[i];
    const size_t WH = size_t(r->W) * r->H;
    auto take = [&](unsigned bit, auto& v, size_t off, size_t esz) {
      if (!(r->planes & bit)) return;
      v.resize(WH);
      std::memcpy(v.data(), l.pin + off, WH * esz);
    };
    take(DE_PLANE_DISP, r->disp, s.disp, 4);
    take(DE_PLANE_MARGIN, r->margin, s.margin, 4);
    take(DE_PLANE_CONF, r->conf, s.conf, 1);
    take(DE_PLANE_Q4, r->q4, s.q4, 2);
    take(DE_PLANE_QCONF, r->qconf, s.qconf, 1);
    r->status = status;
    r->t_done = t;
    if (status) {
      ++sv->failed;
    } else {
      sv->lat.push_back(t - r->t_submit);
      ++sv->completed;
    }
  }
  l.batch.clear();
  l.busy = false;
  l.finished = false;
}

void fail_batch(de_server* sv, Lane& l, int rc) {
  for (Req* r : l.batch) {
    r->status = rc;
    r->t_done = now_ms();
    ++sv->failed;
  }
  l.batch.clear();
  l.busy = false;
}

void worker_main(de_server* sv) {
  cudaSetDevice(sv->device);
  std::unique_lock<std::mutex> lk(sv->mu);
  for (;;) {
    bool any_busy = false;
    for (Lane& l : sv->lanes) {
      if (l.busy && l.finished) {
        deliver(sv, l);
        sv->cv_done.notify_all();
      }
      any_busy |= l.busy;
    }
    bool launched = false;
    for (Lane& l : sv->lanes) {
      if (l.busy || sv->pending.empty() || sv->fatal) continue;
      // admit first come first served while the batch fits the lane
      std::vector<Req*> b;
      while (!sv->pending.empty() && int(b.size()) < sv->scfg.max_batch) {
        b.push_back(sv->pending.front());
        size_t io = 0;
        const size_t need = plan_batch(sv, b, nullptr, nullptr, nullptr, &io, nullptr);
        if (need > l.dev_cap || align256(io) + 256 > l.pin_cap) {
          b.pop_back();
          if (b.empty()) {                       // alone it does not fit: refuse it
            Req* r = sv->pending.front();
            sv->pending.pop_front();
            r->status = DE_ERR_OOM;
            r->t_done = now_ms();
            ++sv->failed;
            sv->cv_done.notify_all();
            continue;
          }
          break;
        }
        sv->pending.pop_front();
      }
      if (b.empty()) continue;
      l.batch = b;
      l.busy = true;
      l.finished = false;
      ++sv->batches;
      sv->batched_pairs += b.size();
      lk.unlock();
      const int rc = launch(sv, l);
      lk.lock();
      if (rc) {
        fail_batch(sv, l, rc);
        sv->cv_done.notify_all();
      } else {
        launched = true;
        any_busy = true;
      }
    }
    if (sv->stop && sv->pending.empty() && !any_busy) break;
    if (!launched) {
      bool work = false;
      for (Lane& l : sv->lanes) work |= (l.busy && l.finished);
      bool free_lane = false;
      for (Lane& l : sv->lanes) free_lane |= !l.busy;
      if (!work && !(free_lane && !sv->pending.empty()))
        sv->cv_work.wait_for(lk, std::chrono::milliseconds(50));
    }
  }
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  const size_t k = std::min(v.size() - 1, size_t(q * double(v.size() - 1) + 0.5));
  std::nth_element(v.begin(), v.begin() + k, v.end());
  return v[k];
}

}  // namespace

extern "C" {

void de_server_cfg_default(de_server_cfg* c) {
  if (!c) return;
  c->device = 0;
  c->hbm_budget = size_t(8) << 30;
  c->max_batch = 16;
  c->lanes = 2;
}

int de_server_create(const de_cfg* cfg, const de_server_cfg* scfg, de_server** out) {
  if (!cfg || !scfg || !out) return de::set_error(DE_ERR_ARG, "NULL argument");
  de_pair probe{};
  probe.L = probe.R = reinterpret_cast<const uint8_t*>(1);
  probe.W = 64;
  probe.H = 64;
  size_t dummy = 0;
  if (int rc = de_dense_workspace_bytes(cfg, &probe, 1, &dummy)) return rc;
  if (scfg->lanes < 1 || scfg->lanes > 8 || scfg->max_batch < 1 ||
      scfg->max_batch > 4096 || scfg->hbm_budget < (size_t(64) << 20))
    return de::set_error(DE_ERR_ARG, "lanes 1..8, max_batch 1..4096, budget >= 64 MiB");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || scfg->device < 0 || scfg->device >= ndev)
    return de::set_error(DE_ERR_ARG, "no CUDA device %d", scfg->device);
  cudaSetDevice(scfg->device);
  de_server* sv = new de_server;
  sv->cfg = *cfg;
  sv->scfg = *scfg;
  sv->device = scfg->device;
  sv->lanes.resize(scfg->lanes);
  const size_t per = (scfg->hbm_budget / scfg->lanes) & ~size_t(255);
  for (Lane& l : sv->lanes) {
    l.owner = sv;
    cudaError_t e = cudaStreamCreateWithFlags(&l.s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&l.dev, per);
    // the pinned mirror holds the I/O block only: at most ~14 bytes per pixel of a
    // pair whose workspace (>= 2*W*H*64 bytes) also fits the arena
    const size_t pin = std::max<size_t>(per / 8, size_t(16) << 20);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&l.pin), pin,
                                            cudaHostAllocDefault);
    if (e != cudaSuccess) {
      de_server_destroy(sv);
      return de::set_error(DE_ERR_OOM, "server lane: %s", cudaGetErrorString(e));
    }
    l.dev_cap = per;
    l.pin_cap = pin;
  }
  sv->worker = std::thread(worker_main, sv);
  *out = sv;
  return DE_OK;
}

int de_server_submit(de_server* sv, int stream, const uint8_t* L, const uint8_t* R, int W,
                     int H, int dmax, unsigned planes, unsigned long long* ticket) {
  if (!sv || !L || !R || !ticket) return de::set_error(DE_ERR_ARG, "NULL argument");
  de_pair probe{};
  probe.L = L;
  probe.R = R;
  probe.W = W;
  probe.H = H;
  probe.dmax = dmax;
  size_t dummy = 0;
  if (int rc = de_dense_workspace_bytes(&sv->cfg, &probe, 1, &dummy)) return rc;
  Req* r = nullptr;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (!sv->pool.empty()) {
      r = sv->pool.back();
      sv->pool.pop_back();
    }
  }
  if (!r) r = new Req;
  r->planes = planes ? planes : DE_PLANE_ALL;
  r->status = 1;
  r->stream = stream;
  r->W = W;
  r->H = H;
  r->dmax = dmax;
  const size_t WH = size_t(W) * H;
  r->L.resize(WH);
  r->R.resize(WH);
  std::memcpy(r->L.data(), L, WH);
  std::memcpy(r->R.data(), R, WH);
  r->t_submit = now_ms();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) {
      delete r;
      return de::set_error(DE_ERR_CLOSED, "server is shutting down");
    }
    r->ticket = sv->next_ticket++;
    sv->reqs[r->ticket] = r;
    sv->pending.push_back(r);
    sv->max_pending = std::max(sv->max_pending, sv->pending.size());
    *ticket = r->ticket;
  }
  sv->cv_work.notify_all();
  return DE_OK;
}

int de_server_wait(de_server* sv, unsigned long long ticket, int timeout_ms, float* disp, float* margin,
                   uint8_t* conf, int16_t* q4, uint8_t* qconf, double* latency_ms) {
  if (!sv) return de::set_error(DE_ERR_ARG, "server is NULL");
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(ticket);
  if (it == sv->reqs.end()) return de::set_error(DE_ERR_ARG, "unknown ticket %llu",
                                                 (unsigned long long)ticket);
  Req* r = it->second;
  const auto until = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
  while (r->status == 1)
    if (sv->cv_done.wait_until(lk, until) == std::cv_status::timeout && r->status == 1)
      return de::set_error(DE_ERR_TIMEOUT, "request %llu not finished after %d ms",
                           (unsigned long long)ticket, timeout_ms);
  const int status = r->status;
  if (status == 0) {
    const size_t WH = size_t(r->W) * r->H;
    const unsigned p = r->planes;
    if (disp && (p & DE_PLANE_DISP)) std::memcpy(disp, r->disp.data(), WH * 4);
    if (margin && (p & DE_PLANE_MARGIN)) std::memcpy(margin, r->margin.data(), WH * 4);
    if (conf && (p & DE_PLANE_CONF)) std::memcpy(conf, r->conf.data(), WH);
    if (q4 && (p & DE_PLANE_Q4)) std::memcpy(q4, r->q4.data(), WH * 2);
    if (qconf && (p & DE_PLANE_QCONF)) std::memcpy(qconf, r->qconf.data(), WH);
    if (latency_ms) *latency_ms = r->t_done - r->t_submit;
  }
  sv->reqs.erase(it);
  if (sv->pool.size() < 256) sv->pool.push_back(r); else delete r;
  if (status) return de::set_error(status, "request failed (%d)", status);
  return DE_OK;
}

int de_server_stats(de_server* sv, de_server_report* out) {
  if (!sv || !out) return de::set_error(DE_ERR_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(sv->mu);
  out->completed = sv->completed;
  out->failed = sv->failed;
  out->batches = sv->batches;
  out->mean_batch = sv->batches ? double(sv->batched_pairs) / double(sv->batches) : 0.0;
  out->p50_ms = percentile(sv->lat, 0.50);
  out->p99_ms = percentile(sv->lat, 0.99);
  out->max_ms = sv->lat.empty() ? 0.0 : *std::max_element(sv->lat.begin(), sv->lat.end());
  out->max_pending = sv->max_pending;
  return DE_OK;
}

int de_server_reset_stats(de_server* sv) {
  if (!sv) return de::set_error(DE_ERR_ARG, "server is NULL");
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->lat.clear();
  sv->completed = sv->failed = sv->batches = sv->batched_pairs = 0;
  sv->max_pending = 0;
  return DE_OK;
}

int de_server_last_disparity(de_server* sv, int stream, float* host, int W, int H) {
  if (!sv || !host) return de::set_error(DE_ERR_ARG, "NULL argument");
  float* src = nullptr;
  cudaEvent_t ev = nullptr;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->streams.find(stream);
    if (it == sv->streams.end() || it->second.frames == 0)
      return de::set_error(DE_ERR_ARG, "stream %d has no frame yet", stream);
    StreamState& st = it->second;
    if (st.W != W || st.H != H)
      return de::set_error(DE_ERR_ARG, "stream %d is %dx%d", stream, st.W, st.H);
    const int k = int((st.frames - 1) & 1);       // the newest launched frame
    src = st.buf[k];
    ev = st.ev[k];
  }
  cudaSetDevice(sv->device);
  cudaError_t e = cudaEventSynchronize(ev);
  if (e == cudaSuccess) e = cudaMemcpy(host, src, size_t(W) * H * 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return de::set_error(DE_ERR_CUDA, "state read: %s", cudaGetErrorString(e));
  return DE_OK;
}

int de_server_destroy(de_server* sv) {
  if (!sv) return DE_OK;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  if (sv->worker.joinable()) sv->worker.join();
  cudaSetDevice(sv->device);
  for (Lane& l : sv->lanes) {
    if (l.s) cudaStreamSynchronize(l.s);
    if (l.dev) cudaFree(l.dev);
    if (l.pin) cudaFreeHost(l.pin);
    if (l.s) cudaStreamDestroy(l.s);
  }
  for (auto& kv : sv->streams)
    for (int k = 0; k < 2; ++k) {
      if (kv.second.buf[k]) cudaFree(kv.second.buf[k]);
      if (kv.second.ev[k]) cudaEventDestroy(kv.second.ev[k]);
    }
  for (auto& kv : sv->reqs) delete kv.second;
  for (Req* r : sv->pool) delete r;
  delete sv;
  return DE_OK;
}

int de_dedd_encode_dev(const float* disp, const uint8_t* conf, int W, int H, int16_t* q4,
                       uint8_t* qconf, void* stream) {
  return de::dedd_encode_dev(disp, conf, W, H, q4, qconf, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
