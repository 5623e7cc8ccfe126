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
//   * each camera stream keeps device state: its last two disparity maps (allocated at
//     the stream's first frame of a size, kept until the server is destroyed),
//     readable on request by the host;
//   * a stream can be given a temporal prior (de_server_stream_prior): its frames are
//     then matched through the prior path (core/tools/de_dense.cpp:797-853, --prior)
//     with its previous map, hole-filled on the device
//     (article/coarse_to_fine.py:58-76), as the prior, one at a time and in order;
//   * results are those of the plain (or prior) pipeline bit for bit: batching changes
//     which pairs share a launch, never the arithmetic (each pair's work is
//     independent).
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
  int band = 0;                        // temporal prior band of its stream at admission
  unsigned planes = 0;                 // DE_PLANE_* the client will read
  // page-locked block holding the inputs and the requested outputs (ReqLayout), kept
  // with the request when it returns to the pool
  uint8_t* pin = nullptr;
  size_t pin_cap = 0;
  double t_submit = 0, t_launch = 0, t_done = 0;
  int status = 1;                      // 1 pending, 0 done, < 0 error code
};

struct Slot {                          // one request's place in a lane's arena
  size_t L, R, disp, margin, conf, q4, qconf;
};

// A request's page-locked block: L | R | disp | margin | conf | q4 | qconf, each
// 256-byte aligned, so the inputs move up in one copy into an arena slot laid out the
// same way and each output plane comes straight back into the block.
Slot req_layout(int W, int H, size_t* total) {
  const size_t WH = size_t(W) * H;
  Slot s;
  size_t o = 0;
  s.L = o;       o = align256(o + WH);
  s.R = o;       o = align256(o + WH);
  s.disp = o;    o = align256(o + WH * 4);
  s.margin = o;  o = align256(o + WH * 4);
  s.conf = o;    o = align256(o + WH);
  s.q4 = o;      o = align256(o + WH * 2);
  s.qconf = o;   o = align256(o + WH);
  if (total) *total = o;
  return s;
}

// Arena of one batch: [inputs | outputs | status words] [plain workspace] [one-at-a-
// time workspace].  Requests of streams without a prior run as one batched launch
// set in the plain workspace; requests of streams with a prior run one at a time, in
// order, reusing the one-at-a-time workspace (a filled prior map, the fill's scratch
// and the prior path's workspace, or a single pair's dense workspace).
struct Plan {
  std::vector<Slot> slots;
  std::vector<int> plain, seq;         // request indices, in batch order
  size_t in_end = 0, out_end = 0;      // I/O block: inputs [0, in_end), outputs to out_end
  size_t status = 0;                   // status words: [0] plain batch, [1 + i] seq[i]
  size_t io_end = 0;                   // end of the I/O block (the pinned mirror's share)
  size_t ws_plain = 0, ws_plain_bytes = 0;
  size_t ws_seq = 0, ws_seq_bytes = 0;
  size_t total = 0;
};

struct Lane {
  cudaStream_t s = nullptr;
  uint8_t* dev = nullptr;              // I/O block, then the pipeline workspaces
  size_t dev_cap = 0;
  uint8_t* pin = nullptr;              // page-locked copy of the batch's status words
  size_t pin_cap = 0;
  std::vector<Req*> batch;
  std::vector<int> status_of;          // per request of a finished batch
  Plan plan;
  bool busy = false;
  bool finished = false;               // set by the stream callback
  struct de_server* owner = nullptr;
};

// Per camera stream, on the device: the last two disparity maps (slot frames & 1 takes
// frame number `frames`).  Each slot's last write and last host read are events, so a
// write waits for the slot's previous write and read, whichever lanes issued them.
struct StreamState {
  int W = 0, H = 0;
  float* buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};   // last write of the slot
  cudaEvent_t rd[2] = {nullptr, nullptr};   // last host read of the slot
  bool read_issued[2] = {false, false};
  uint64_t frames = 0;                      // maps written since the last size change
  int band = 0;                             // temporal prior band, 0 = off
};

}  // namespace

struct de_server {
  de_cfg cfg{};
  de_server_cfg scfg{};
  int device = 0;
  std::vector<Lane> lanes;
  std::mutex mu;                       // requests, lanes, statistics
  std::condition_variable cv_work;     // new request, finished lane or stop
  std::condition_variable cv_done;     // a request finished
  std::deque<Req*> pending;
  std::unordered_map<uint64_t, Req*> reqs;
  uint64_t next_ticket = 1;
  // Stream state has its own lock, never held while taking `mu` (order: mu, then
  // state_mu).  Device work on stream state is enqueued under it, so the order of
  // writes and reads of a slot is the order they were enqueued in.  Nothing is freed
  // while the server runs: maps replaced after a size change are retired and freed at
  // destruction, so a read already enqueued never sees freed memory.
  std::mutex state_mu;
  std::unordered_map<int, StreamState> streams;
  std::vector<float*> retired;
  cudaStream_t state_s = nullptr;      // host reads of stream state
  std::mutex rd_mu;                    // one host read at a time, through rd_pin
  float* rd_pin = nullptr;
  size_t rd_cap = 0;
  std::vector<Req*> pool;              // finished requests kept with their buffers
  std::vector<uint8_t*> retired_pin;   // replaced request blocks, freed at destruction
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

de_pair pair_of(const Req* r) {
  de_pair p{};
  p.L = p.R = reinterpret_cast<const uint8_t*>(1);   // sizing only
  p.W = r->W;
  p.H = r->H;
  p.dmax = r->dmax;
  return p;
}

// Arena layout of a prospective batch; false if a pair is outside the pipeline's limits.
bool plan_batch(const de_server* sv, const std::vector<Req*>& b, Plan* pl) {
  Plan P;
  P.slots.resize(b.size());
  size_t o = 0;
  for (size_t i = 0; i < b.size(); ++i) {
    const size_t WH = size_t(b[i]->W) * b[i]->H;
    P.slots[i].L = o;  o = align256(o + WH);
    P.slots[i].R = o;  o = align256(o + WH);
    (b[i]->band > 0 ? P.seq : P.plain).push_back(int(i));
  }
  P.in_end = o;
  for (size_t i = 0; i < b.size(); ++i) {
    const size_t WH = size_t(b[i]->W) * b[i]->H;
    Slot& s = P.slots[i];
    s.disp = o;    o = align256(o + WH * 4);
    s.margin = o;  o = align256(o + WH * 4);
    s.conf = o;    o = align256(o + WH);
    s.q4 = o;      o = align256(o + WH * 2);
    s.qconf = o;   o = align256(o + WH);
  }
  P.out_end = o;
  P.status = o;
  o = align256(o + (1 + P.seq.size()) * sizeof(int));
  P.io_end = o;
  std::vector<de_pair> pairs;
  for (int i : P.plain) pairs.push_back(pair_of(b[i]));
  if (!pairs.empty() &&
      de_dense_workspace_bytes(&sv->cfg, pairs.data(), int(pairs.size()), &P.ws_plain_bytes))
    return false;
  for (int i : P.seq) {
    const de_pair p = pair_of(b[i]);
    size_t dense = 0, prior = 0;
    if (de_dense_workspace_bytes(&sv->cfg, &p, 1, &dense) ||
        de_dense_prior_workspace_bytes(&sv->cfg, &p, &prior))
      return false;
    const size_t map = align256(size_t(p.W) * p.H * 4);
    P.ws_seq_bytes = std::max({P.ws_seq_bytes, dense,
                               map + de::fill_ws_bytes(p.W, p.H) + align256(prior)});
  }
  P.ws_plain = P.io_end;
  P.ws_seq = align256(P.ws_plain + P.ws_plain_bytes);
  P.total = P.ws_seq + P.ws_seq_bytes;
  *pl = std::move(P);
  return true;
}

de_pair device_pair(const Lane& l, const Req* r, const Slot& s) {
  de_pair p{};
  p.L = l.dev + s.L;
  p.R = l.dev + s.R;
  p.W = r->W;
  p.H = r->H;
  p.dmax = r->dmax;
  p.disp = reinterpret_cast<float*>(l.dev + s.disp);
  p.margin = reinterpret_cast<float*>(l.dev + s.margin);
  p.conf = l.dev + s.conf;
  return p;
}

// The stream's map slot for this request's frame, (re)allocated at a size change;
// called on the worker thread with state_mu held.  A replaced map is retired, not
// freed (a read may still be queued on it).
int ensure_state(de_server* sv, StreamState* st, int W, int H) {
  for (int k = 0; k < 2; ++k) {
    if (!st->ev[k] && cudaEventCreateWithFlags(&st->ev[k], cudaEventDisableTiming) != cudaSuccess)
      return de::set_error(DE_ERR_CUDA, "stream state event");
    if (!st->rd[k] && cudaEventCreateWithFlags(&st->rd[k], cudaEventDisableTiming) != cudaSuccess)
      return de::set_error(DE_ERR_CUDA, "stream state event");
  }
  if (st->W == W && st->H == H && st->buf[0]) return DE_OK;
  float* nb[2] = {nullptr, nullptr};
  const size_t bytes = size_t(W) * H * 4;
  cudaError_t e = cudaMalloc(&nb[0], bytes);
  if (e == cudaSuccess) e = cudaMalloc(&nb[1], bytes);
  if (e != cudaSuccess) {
    if (nb[0]) sv->retired.push_back(nb[0]);
    return de::set_error(DE_ERR_OOM, "stream state: %s", cudaGetErrorString(e));
  }
  for (int k = 0; k < 2; ++k) {
    if (st->buf[k]) sv->retired.push_back(st->buf[k]);
    st->buf[k] = nb[k];
  }
  st->W = W;
  st->H = H;
  st->frames = 0;
  return DE_OK;
}

// This frame's disparity map into the stream's next slot, after the slot's previous
// write and read.
int record_state(de_server* sv, cudaStream_t s, const Req* r, const float* disp) {
  std::lock_guard<std::mutex> lk(sv->state_mu);
  StreamState* st = &sv->streams[r->stream];
  if (int rc = ensure_state(sv, st, r->W, r->H)) return rc;
  const int k = int(st->frames & 1);
  cudaError_t e = cudaStreamWaitEvent(s, st->ev[k], 0);
  if (e == cudaSuccess && st->read_issued[k]) e = cudaStreamWaitEvent(s, st->rd[k], 0);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(st->buf[k], disp, size_t(r->W) * r->H * 4, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaEventRecord(st->ev[k], s);
  if (e != cudaSuccess) return de::set_error(DE_ERR_CUDA, "state: %s", cudaGetErrorString(e));
  ++st->frames;
  return DE_OK;
}

// The previous map of a prior stream, if it has one of this size: its device address,
// with `s` made to wait for its write.  nullptr: match this frame without a prior.
const float* previous_map(de_server* sv, cudaStream_t s, const Req* r) {
  std::lock_guard<std::mutex> lk(sv->state_mu);
  auto it = sv->streams.find(r->stream);
  if (it == sv->streams.end()) return nullptr;
  StreamState& st = it->second;
  if (st.frames == 0 || st.W != r->W || st.H != r->H) return nullptr;
  const int k = int((st.frames - 1) & 1);
  if (cudaStreamWaitEvent(s, st.ev[k], 0) != cudaSuccess) return nullptr;
  return st.buf[k];
}

// Enqueues one batch on a free lane.  Called by the worker without `mu` held; the
// requests are already owned by the lane.
int launch(de_server* sv, Lane& l) {
  if (!plan_batch(sv, l.batch, &l.plan)) return de::set_error(DE_ERR_ARG, "batch plan");
  const Plan& P = l.plan;
  cudaError_t e = cudaSuccess;
  for (size_t i = 0; i < l.batch.size() && e == cudaSuccess; ++i) {
    Req* r = l.batch[i];
    const Slot rl = req_layout(r->W, r->H, nullptr);
    e = cudaMemcpyAsync(l.dev + P.slots[i].L, r->pin + rl.L, rl.R + size_t(r->W) * r->H,
                        cudaMemcpyHostToDevice, l.s);
    r->t_launch = now_ms();
  }
  if (e == cudaSuccess)
    e = cudaMemsetAsync(l.dev + P.status, 0, (1 + P.seq.size()) * sizeof(int), l.s);
  if (e != cudaSuccess) return de::set_error(DE_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
  int* status = reinterpret_cast<int*>(l.dev + P.status);
  auto finish = [&](int i) -> int {                  // DEDD planes and stream state
    Req* r = l.batch[i];
    const Slot& s = P.slots[i];
    if (int rc = de::dedd_encode_dev(reinterpret_cast<float*>(l.dev + s.disp), l.dev + s.conf,
                                     r->W, r->H, reinterpret_cast<int16_t*>(l.dev + s.q4),
                                     l.dev + s.qconf, l.s))
      return rc;
    return record_state(sv, l.s, r, reinterpret_cast<float*>(l.dev + s.disp));
  };
  // streams without a prior: one batched launch set
  if (!P.plain.empty()) {
    std::vector<de_pair> dp;
    for (int i : P.plain) dp.push_back(device_pair(l, l.batch[i], P.slots[i]));
    // the lanes already overlap one another's batches: one launch set each
    if (int rc = de::dense_dev(&sv->cfg, dp.data(), int(dp.size()), l.dev + P.ws_plain,
                               P.ws_plain_bytes, l.s, 1))
      return rc;
    e = cudaMemcpyAsync(status, l.dev + P.ws_plain, sizeof(int), cudaMemcpyDeviceToDevice, l.s);
    if (e != cudaSuccess) return de::set_error(DE_ERR_CUDA, "status: %s", cudaGetErrorString(e));
    for (int i : P.plain)
      if (int rc = finish(i)) return rc;
  }
  // streams with a prior: one at a time, each after its stream's previous frame
  for (size_t q = 0; q < P.seq.size(); ++q) {
    const int i = P.seq[q];
    const Req* r = l.batch[i];
    const de_pair dp = device_pair(l, r, P.slots[i]);
    uint8_t* ws = l.dev + P.ws_seq;
    const float* prev = previous_map(sv, l.s, r);
    int rc;
    if (prev) {
      float* prior = reinterpret_cast<float*>(ws);
      const size_t map = align256(size_t(r->W) * r->H * 4);
      const size_t fill = de::fill_ws_bytes(r->W, r->H);
      rc = de::fill_holes_dev(prev, prior, r->W, r->H, ws + map, fill, l.s);
      if (!rc) rc = de_dense_prior_dev(&sv->cfg, &dp, prior, r->band, ws + map + fill,
                                       P.ws_seq_bytes - map - fill, l.s);
      ws += map + fill;                               // the status word's workspace
    } else {
      rc = de_dense_dev(&sv->cfg, &dp, 1, ws, P.ws_seq_bytes, l.s);
    }
    if (rc) return rc;
    e = cudaMemcpyAsync(status + 1 + q, ws, sizeof(int), cudaMemcpyDeviceToDevice, l.s);
    if (e != cudaSuccess) return de::set_error(DE_ERR_CUDA, "status: %s", cudaGetErrorString(e));
    if ((rc = finish(i))) return rc;
  }
  // only the planes each request asked for come back
  for (size_t i = 0; i < l.batch.size() && e == cudaSuccess; ++i) {
    const Req* r = l.batch[i];
    const Slot& s = P.slots[i];
    const Slot h = req_layout(r->W, r->H, nullptr);
    const size_t WH = size_t(r->W) * r->H;
    const struct { unsigned bit; size_t dev, host, bytes; } planes[] = {
        {DE_PLANE_DISP, s.disp, h.disp, WH * 4}, {DE_PLANE_MARGIN, s.margin, h.margin, WH * 4},
        {DE_PLANE_CONF, s.conf, h.conf, WH}, {DE_PLANE_Q4, s.q4, h.q4, WH * 2},
        {DE_PLANE_QCONF, s.qconf, h.qconf, WH}};
    for (const auto& pl : planes)
      if ((r->planes & pl.bit) && e == cudaSuccess)
        e = cudaMemcpyAsync(r->pin + pl.host, l.dev + pl.dev, pl.bytes, cudaMemcpyDeviceToHost,
                            l.s);
  }
  // the status words (a bounded device wait that ran out sets one)
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(l.pin, status, (1 + P.seq.size()) * sizeof(int),
                        cudaMemcpyDeviceToHost, l.s);
  if (e == cudaSuccess) e = cudaLaunchHostFunc(l.s, lane_done, &l);
  if (e != cudaSuccess) return de::set_error(DE_ERR_CUDA, "download: %s", cudaGetErrorString(e));
  return DE_OK;
}

// A finished lane's status words, one per request (the outputs are already in each
// request's page-locked block).  The server lock is not needed.
void copy_results(Lane& l) {
  const Plan& P = l.plan;
  std::vector<int> words(1 + P.seq.size());
  std::memcpy(words.data(), l.pin, words.size() * sizeof(int));
  l.status_of.assign(l.batch.size(), words[0] ? DE_ERR_TIMEOUT : 0);
  for (size_t q = 0; q < P.seq.size(); ++q)
    l.status_of[P.seq[q]] = words[1 + q] ? DE_ERR_TIMEOUT : 0;
}

// Publishes a finished lane's requests and frees the lane.  Lock held.
void deliver(de_server* sv, Lane& l) {
  const double t = now_ms();
  for (size_t i = 0; i < l.batch.size(); ++i) {
    Req* r = l.batch[i];
    const int status = l.status_of[i];
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
        lk.unlock();
        copy_results(l);
        lk.lock();
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
        Req* front = sv->pending.front();
        {
          std::lock_guard<std::mutex> sl(sv->state_mu);
          auto it = sv->streams.find(front->stream);
          front->band = it == sv->streams.end() ? 0 : it->second.band;
        }
        b.push_back(front);
        Plan plan;
        if (!plan_batch(sv, b, &plan) || plan.total > l.dev_cap ||
            (1 + plan.seq.size()) * sizeof(int) > l.pin_cap) {
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
      // a launch that failed part-way may have copies into its requests' blocks in
      // flight: let them finish before the requests are handed back (no host callback
      // of this lane is queued, so this cannot wait on the lock)
      if (rc) cudaStreamSynchronize(l.s);
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
    const size_t pin = align256((1 + size_t(scfg->max_batch)) * sizeof(int));
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&l.pin), pin,
                                            cudaHostAllocDefault);
    if (e != cudaSuccess) {
      de_server_destroy(sv);
      return de::set_error(DE_ERR_OOM, "server lane: %s", cudaGetErrorString(e));
    }
    l.dev_cap = per;
    l.pin_cap = pin;
  }
  if (cudaStreamCreateWithFlags(&sv->state_s, cudaStreamNonBlocking) != cudaSuccess) {
    de_server_destroy(sv);
    return de::set_error(DE_ERR_CUDA, "server state stream");
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
  size_t need = 0;
  const Slot rl = req_layout(W, H, &need);
  Req* r = nullptr;
  {
    // a pooled request whose block is large enough, else any pooled one
    std::lock_guard<std::mutex> lk(sv->mu);
    size_t pick = sv->pool.size();
    for (size_t i = 0; i < sv->pool.size(); ++i)
      if (sv->pool[i]->pin_cap >= need &&
          (pick == sv->pool.size() || sv->pool[i]->pin_cap < sv->pool[pick]->pin_cap))
        pick = i;
    if (pick == sv->pool.size() && !sv->pool.empty()) pick = sv->pool.size() - 1;
    if (pick < sv->pool.size()) {
      r = sv->pool[pick];
      sv->pool.erase(sv->pool.begin() + long(pick));
    }
  }
  if (!r) r = new Req;
  if (r->pin_cap < need) {
    // a bigger block; the old one is freed with the server (freeing page-locked memory
    // can wait for the device, which this submitting thread should not)
    uint8_t* nb = nullptr;
    if (cudaHostAlloc(reinterpret_cast<void**>(&nb), need, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->pool.push_back(r);
      return de::set_error(DE_ERR_OOM, "page-locked request buffer of %zu bytes", need);
    }
    if (r->pin) {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->retired_pin.push_back(r->pin);
    }
    r->pin = nb;
    r->pin_cap = need;
  }
  r->planes = planes ? planes : DE_PLANE_ALL;
  r->status = 1;
  r->stream = stream;
  r->W = W;
  r->H = H;
  r->dmax = dmax;
  const size_t WH = size_t(W) * H;
  std::memcpy(r->pin + rl.L, L, WH);
  std::memcpy(r->pin + rl.R, R, WH);
  r->t_submit = now_ms();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) {
      sv->pool.push_back(r);
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
    // the copies run in the caller's thread without the lock: the request stays
    // registered (so nothing reuses it) until they are done
    lk.unlock();
    const size_t WH = size_t(r->W) * r->H;
    const unsigned p = r->planes;
    const Slot h = req_layout(r->W, r->H, nullptr);
    if (disp && (p & DE_PLANE_DISP)) std::memcpy(disp, r->pin + h.disp, WH * 4);
    if (margin && (p & DE_PLANE_MARGIN)) std::memcpy(margin, r->pin + h.margin, WH * 4);
    if (conf && (p & DE_PLANE_CONF)) std::memcpy(conf, r->pin + h.conf, WH);
    if (q4 && (p & DE_PLANE_Q4)) std::memcpy(q4, r->pin + h.q4, WH * 2);
    if (qconf && (p & DE_PLANE_QCONF)) std::memcpy(qconf, r->pin + h.qconf, WH);
    if (latency_ms) *latency_ms = r->t_done - r->t_submit;
    lk.lock();
  }
  sv->reqs.erase(it);
  sv->pool.push_back(r);
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

int de_server_stream_prior(de_server* sv, int stream, int band) {
  if (!sv) return de::set_error(DE_ERR_ARG, "server is NULL");
  if (band < 0 || band > DE_MAX_D) return de::set_error(DE_ERR_ARG, "band %d outside 0..%d",
                                                        band, DE_MAX_D);
  if (band > 0 && (sv->cfg.census_hw != 3 || sv->cfg.census_hh != 3))
    return de::set_error(DE_ERR_ARG, "the prior path is the reference's 7x7-census path");
  std::lock_guard<std::mutex> lk(sv->state_mu);
  sv->streams[stream].band = band;
  return DE_OK;
}

int de_server_last_disparity(de_server* sv, int stream, float* host, int W, int H) {
  if (!sv || !host || W < 1 || H < 1) return de::set_error(DE_ERR_ARG, "bad argument");
  const size_t bytes = size_t(W) * H * 4;
  std::lock_guard<std::mutex> rl(sv->rd_mu);         // one reader at a time owns rd_pin
  cudaSetDevice(sv->device);
  if (sv->rd_cap < bytes) {
    if (sv->rd_pin) cudaFreeHost(sv->rd_pin);
    sv->rd_pin = nullptr;
    sv->rd_cap = 0;
    if (cudaHostAlloc(reinterpret_cast<void**>(&sv->rd_pin), bytes, cudaHostAllocDefault) !=
        cudaSuccess)
      return de::set_error(DE_ERR_OOM, "state read buffer");
    sv->rd_cap = bytes;
  }
  cudaEvent_t done = nullptr;
  {
    // the copy is enqueued under state_mu, after the slot's write and before the
    // slot's next write (which waits for this read's event)
    std::lock_guard<std::mutex> lk(sv->state_mu);
    auto it = sv->streams.find(stream);
    if (it == sv->streams.end() || it->second.frames == 0)
      return de::set_error(DE_ERR_ARG, "stream %d has no frame yet", stream);
    StreamState& st = it->second;
    if (st.W != W || st.H != H)
      return de::set_error(DE_ERR_ARG, "stream %d is %dx%d", stream, st.W, st.H);
    const int k = int((st.frames - 1) & 1);          // the newest launched frame
    cudaError_t e = cudaStreamWaitEvent(sv->state_s, st.ev[k], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(sv->rd_pin, st.buf[k], bytes, cudaMemcpyDeviceToHost, sv->state_s);
    if (e == cudaSuccess) e = cudaEventRecord(st.rd[k], sv->state_s);
    if (e != cudaSuccess) return de::set_error(DE_ERR_CUDA, "state read: %s", cudaGetErrorString(e));
    st.read_issued[k] = true;
    done = st.rd[k];
  }
  // rd events are recorded only by readers, and readers are serialised by rd_mu
  if (cudaEventSynchronize(done) != cudaSuccess)
    return de::set_error(DE_ERR_CUDA, "state read: %s", cudaGetErrorString(cudaGetLastError()));
  std::memcpy(host, sv->rd_pin, bytes);
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
  if (sv->state_s) cudaStreamSynchronize(sv->state_s);
  for (auto& kv : sv->streams)
    for (int k = 0; k < 2; ++k) {
      if (kv.second.buf[k]) cudaFree(kv.second.buf[k]);
      if (kv.second.ev[k]) cudaEventDestroy(kv.second.ev[k]);
      if (kv.second.rd[k]) cudaEventDestroy(kv.second.rd[k]);
    }
  for (float* p : sv->retired) cudaFree(p);
  if (sv->rd_pin) cudaFreeHost(sv->rd_pin);
  if (sv->state_s) cudaStreamDestroy(sv->state_s);
  for (auto& kv : sv->reqs) {
    if (kv.second->pin) cudaFreeHost(kv.second->pin);
    delete kv.second;
  }
  for (Req* r : sv->pool) {
    if (r->pin) cudaFreeHost(r->pin);
    delete r;
  }
  for (uint8_t* p : sv->retired_pin) cudaFreeHost(p);
  delete sv;
  return DE_OK;
}

int de_dedd_encode_dev(const float* disp, const uint8_t* conf, int W, int H, int16_t* q4,
                       uint8_t* qconf, void* stream) {
  return de::dedd_encode_dev(disp, conf, W, H, q4, qconf, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
