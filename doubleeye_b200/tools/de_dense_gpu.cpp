// de_dense_gpu: the reference's dense matcher tools on the B200 path.
//
//   de_dense_gpu L.y8 R.y8 W H [flags]        core/tools/de_dense.cpp:1610-2040
//   de_dense_gpu - - W H --stream [flags]     core/tools/de_dense_cuda.cu:670-770
//
// Same argv and the same output bytes: --out writes the W*H float32 disparity map (NaN
// where the matcher declined), --out-conf the six W*H float32 planes s1, s2, d1, d2,
// lrc, lrc2; the last stdout line containing "total" carries the stage times.  With
// --stream, "DEIR" frames (14-byte header + Y8) arrive on stdin, are paired by frame
// number (stream 1 is the left camera), and each pair leaves on stdout as "DEDD"
// (16-byte header, the left Y8, W*H int16 disparity in sixteenths of a pixel with
// -32768 where declined, and W*H u8 confidence unless --no-confidence).  --keypoints
// F.csv writes the sparse feature set read out of the dense map (x, y, disparity,
// margin at FAST keypoints of the left image), as de_dense_cuda does.
// Everything runs through the library's C ABI; flags of the reference's measured
// negative paths (guided/box filters, --csct, --simd, --c2f, --topk != 2, --dump-vol)
// are refused.  --prior F [--band N] runs the prior-masked path (sub-pixel off).

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "doubleeye_b200.h"

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

bool load_y8(const std::string& p, size_t n, std::vector<uint8_t>* out) {
  FILE* f = std::fopen(p.c_str(), "rb");
  if (!f) return false;
  out->resize(n);
  const size_t got = std::fread(out->data(), 1, n, f);
  std::fclose(f);
  return got == n;
}

bool dump(const std::string& p, const float* v, size_t n) {
  FILE* f = std::fopen(p.c_str(), "wb");
  const size_t w = f ? std::fwrite(v, sizeof(float), n, f) : 0;
  if (f) std::fclose(f);
  if (w == n) return true;
  std::fprintf(stderr, "could not write %s (%zu of %zu floats)\n", p.c_str(), w, n);
  return false;
}

bool read_all(void* p, size_t n) { return std::fread(p, 1, n, stdin) == n; }

bool write_all(const void* p, size_t n) { return std::fwrite(p, 1, n, stdout) == n; }

// ---- --prior ------------------------------------------------------------------
// The prior file holds float32 disparities, either one per pixel (W*H) or one per
// 2x2 block (floor(W/2) * floor(H/2)), the latter read as nearest-neighbour samples
// at twice the disparity.  A non-finite value is a hole, and a prior with holes is
// refused.  Interface: core/tools/de_dense.cpp --prior (flag at :1756).
bool slurp(const std::string& path, std::vector<unsigned char>* bytes) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  unsigned char chunk[1 << 16];
  size_t n;
  while ((n = std::fread(chunk, 1, sizeof(chunk), f)) > 0) bytes->insert(bytes->end(), chunk, chunk + n);
  const bool ok = !std::ferror(f);
  std::fclose(f);
  return ok;
}

bool load_prior(const std::string& path, int W, int H, std::vector<float>* prior,
                std::string* why) {
  std::vector<unsigned char> raw;
  if (!slurp(path, &raw)) {
    *why = "not readable";
    return false;
  }
  const size_t full = size_t(W) * H;
  const int hw = W / 2, hh = H / 2;
  const size_t half = size_t(hw) * hh;
  const size_t count = raw.size() / sizeof(float);
  if (raw.size() % sizeof(float) != 0 || (count != full && count != half)) {
    *why = std::to_string(raw.size()) + " bytes; want " + std::to_string(full * 4) +
           " (" + std::to_string(W) + "x" + std::to_string(H) + " float32) or " +
           std::to_string(half * 4) + " (" + std::to_string(hw) + "x" + std::to_string(hh) +
           ", half resolution)";
    return false;
  }
  std::vector<float> src(count);
  std::memcpy(src.data(), raw.data(), count * sizeof(float));
  prior->assign(full, 0.f);
  if (count == full) {
    *prior = std::move(src);
  } else {
    // each full-resolution pixel samples the block it falls in (the last block row /
    // column also covers an odd trailing pixel), disparity scaled to full resolution
    for (int y = 0; y < H; ++y) {
      const float* srow = src.data() + size_t(y / 2 < hh ? y / 2 : hh - 1) * hw;
      float* drow = prior->data() + size_t(y) * W;
      for (int x = 0; x < W; ++x) drow[x] = 2.f * srow[x / 2 < hw ? x / 2 : hw - 1];
    }
  }
  const size_t bad = size_t(std::count_if(prior->begin(), prior->end(),
                                          [](float v) { return !std::isfinite(v); }));
  if (bad) {
    *why = std::to_string(bad) + " of " + std::to_string(full) +
           " values are holes (non-finite); fill them before matching";
    return false;
  }
  return true;
}

// ---- --stream -----------------------------------------------------------------
// Wire format (interface of core/tools/de_dense_cuda.cu:44-59):
//   in   "DEIR" | width u16 | height u16 | camera u8 | flags u8 | frame u32 | Y8 image
//   out  "DEDD" | width u16 | height u16 | frame u32 | flags u32 | left Y8 |
//        W*H int16 disparity in 1/16 px (-32768 = declined) | W*H u8 confidence if
//        flags & 1
// Camera 1 is the left image.  Two images with the same frame number from the two
// cameras make a pair; a later image from the same camera replaces the earlier one.
// At most kWaiting frames wait for their partner; when a ninth arrives, the lowest
// frame number of the nine is given up.
constexpr int kWaiting = 8;

struct FrameSlot {
  bool used = false;
  uint32_t frame = 0;
  bool has[2] = {false, false};   // [0] right camera, [1] left camera
  std::vector<uint8_t> img[2];
};

class FramePairer {
 public:
  explicit FramePairer(size_t bytes) : bytes_(bytes) {
    for (FrameSlot& s : slots_) { s.img[0].resize(bytes); s.img[1].resize(bytes); }
  }
  // Stores the image that was read into scratch(); returns the slot if that
  // completed a pair, else nullptr.
  FrameSlot* offer(uint32_t frame, int camera) {
    const int side = camera == 1 ? 1 : 0;
    FrameSlot* s = find(frame);
    if (!s) s = claim(frame);
    if (!s) { ++discarded_; return nullptr; }   // older than every waiting frame
    std::swap(s->img[side], scratch_);
    if (scratch_.size() != bytes_) scratch_.resize(bytes_);
    s->has[side] = true;
    return (s->has[0] && s->has[1]) ? s : nullptr;
  }
  void release(FrameSlot* s) { s->used = false; s->has[0] = s->has[1] = false; }
  uint8_t* scratch() { if (scratch_.size() != bytes_) scratch_.resize(bytes_); return scratch_.data(); }
  long discarded() const { return discarded_; }

 private:
  FrameSlot* find(uint32_t frame) {
    for (FrameSlot& s : slots_) if (s.used && s.frame == frame) return &s;
    return nullptr;
  }
  // A free slot, else the slot of the lowest waiting frame number, which is given up;
  // nullptr when the new frame itself is the lowest (it is the one given up).
  FrameSlot* claim(uint32_t frame) {
    FrameSlot* victim = nullptr;
    for (FrameSlot& s : slots_) {
      if (!s.used) { victim = &s; break; }
      if (!victim || s.frame < victim->frame) victim = &s;
    }
    if (victim->used && frame < victim->frame) return nullptr;
    if (victim->used) ++discarded_;
    release(victim);
    victim->used = true;
    victim->frame = frame;
    return victim;
  }
  size_t bytes_;
  FrameSlot slots_[kWaiting];
  std::vector<uint8_t> scratch_;
  long discarded_ = 0;
};

template <typename T>
T get_le(const unsigned char* p) {
  T v;
  std::memcpy(&v, p, sizeof(T));
  return v;
}
template <typename T>
void put_le(unsigned char* p, T v) { std::memcpy(p, &v, sizeof(T)); }

// Sixteenths of a pixel, round half up; -32768 (and confidence 0) where the matcher
// gave no positive, finite disparity.
void encode_q4(const std::vector<float>& disp, std::vector<int16_t>* q4,
               std::vector<uint8_t>* conf) {
  for (size_t i = 0; i < disp.size(); ++i) {
    const float d = disp[i];
    const bool ok = std::isfinite(d) && d > 0.f;
    (*q4)[i] = ok ? int16_t(std::floor(double(d) * 16.0 + 0.5)) : int16_t(-32768);
    if (!ok && conf) (*conf)[i] = 0;
  }
}

int serve_stream(de_ctx* ctx, int W, int H, bool want_conf) {
  const size_t WH = size_t(W) * H;
  FramePairer pairer(WH);
  std::vector<float> disp(WH);
  std::vector<int16_t> q4(WH);
  std::vector<uint8_t> conf(WH);
  long served = 0;
  double last_note = now_ms();
  unsigned char in[14];
  while (read_all(in, sizeof(in))) {
    if (std::memcmp(in, "DEIR", 4) != 0) {
      std::fprintf(stderr, "de_dense_gpu: input is not a DEIR frame header; giving up\n");
      return 1;
    }
    const int fw = get_le<uint16_t>(in + 4), fh = get_le<uint16_t>(in + 6);
    const int camera = in[8];
    const uint32_t frame = get_le<uint32_t>(in + 10);
    if (fw != W || fh != H) {
      std::fprintf(stderr, "de_dense_gpu: frame %u is %dx%d; the matcher runs at %dx%d\n",
                   frame, fw, fh, W, H);
      return 1;
    }
    if (!read_all(pairer.scratch(), WH)) break;          // truncated image: end of input
    FrameSlot* pair = pairer.offer(frame, camera);
    if (!pair) continue;
    const uint8_t* left = pair->img[1].data();
    const uint8_t* right = pair->img[0].data();
    if (de_ctx_dense(ctx, left, right, W, H, disp.data(), nullptr,
                     want_conf ? conf.data() : nullptr, nullptr) != DE_OK) {
      std::fprintf(stderr, "de_dense_gpu: frame %u: %s\n", frame, de_last_error());
      return 1;
    }
    encode_q4(disp, &q4, want_conf ? &conf : nullptr);
    unsigned char out[16];
    std::memcpy(out, "DEDD", 4);
    put_le<uint16_t>(out + 4, uint16_t(W));
    put_le<uint16_t>(out + 6, uint16_t(H));
    put_le<uint32_t>(out + 8, frame);
    put_le<uint32_t>(out + 12, want_conf ? 1u : 0u);
    const bool wrote = write_all(out, sizeof(out)) && write_all(left, WH) &&
                       write_all(q4.data(), WH * sizeof(int16_t)) &&
                       (!want_conf || write_all(conf.data(), WH));
    pairer.release(pair);
    if (!wrote) break;                                   // reader went away
    std::fflush(stdout);
    ++served;
    const double t = now_ms();
    if (t - last_note > 5000.0) {
      std::fprintf(stderr, "de_dense_gpu: served %ld frame pairs (%ld images had no partner)\n",
                   served, pairer.discarded());
      last_note = t;
    }
  }
  std::fprintf(stderr, "de_dense_gpu: end of input after %ld frame pairs (%ld images had no "
                       "partner)\n", served, pairer.discarded());
  return 0;
}

int usage(const char* argv0) {
  std::fprintf(stderr,
               "usage: %s L.y8 R.y8 W H [--dmax N] [--iters N] [--lambda F] [--gamma F]\n"
               "       [--damping F] [--sigma-s F] [--sigma-r F] [--ad F] [--ad-trunc N]\n"
               "       [--min-margin F] [--min-ratio F] [--subpixel|--no-subpixel]\n"
               "       [--fit-eq|--fit-parabola] [--lrc] [--out F] [--out-conf F]\n"
               "       [--keypoints F.csv] [--prior F.f32 [--band N]] [--frames N]\n"
               "       [--device N]\n"
               "       [--stream [--no-confidence]]\n",
               argv0);
  return 2;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 5) return usage(argv[0]);
  const std::string lp = argv[1], rp = argv[2];
  const int W = std::atoi(argv[3]), H = std::atoi(argv[4]);
  de_cfg cfg;
  de_cfg_default(&cfg);
  std::string outp, confp, kpp, priorp;
  int band = 2;
  bool stream_mode = false, want_conf = true;
  int frames = 1, device = 0;
  for (int i = 5; i < argc; ++i) {
    const std::string a = argv[i];
    const bool has = i + 1 < argc;
    if (a == "--dmax" && has) cfg.dmax = std::atoi(argv[++i]);
    else if (a == "--iters" && has) cfg.iters = std::atoi(argv[++i]);
    else if (a == "--lambda" && has) cfg.lambda = float(std::atof(argv[++i]));
    else if (a == "--gamma" && has) cfg.gamma = float(std::atof(argv[++i]));
    else if (a == "--damping" && has) cfg.damping = float(std::atof(argv[++i]));
    else if (a == "--sigma-s" && has) cfg.sigma_s = float(std::atof(argv[++i]));
    else if (a == "--sigma-r" && has) cfg.sigma_r = float(std::atof(argv[++i]));
    else if (a == "--ad" && has) cfg.ad = float(std::atof(argv[++i]));
    else if (a == "--ad-trunc" && has) cfg.ad_trunc = std::atoi(argv[++i]);
    else if (a == "--min-margin" && has) cfg.min_margin = float(std::atof(argv[++i]));
    else if (a == "--min-ratio" && has) cfg.min_ratio = float(std::atof(argv[++i]));
    else if (a == "--subpixel") cfg.subpixel = 1;
    else if (a == "--no-subpixel") cfg.subpixel = 0;
    else if (a == "--fit-eq") cfg.fit_eq = 1;
    else if (a == "--fit-parabola") cfg.fit_eq = 0;
    else if (a == "--lrc") cfg.lrc = 1;
    else if (a == "--out" && has) outp = argv[++i];
    else if (a == "--out-conf" && has) confp = argv[++i];
    else if (a == "--keypoints" && has) kpp = argv[++i];
    else if (a == "--prior" && has) priorp = argv[++i];
    else if (a == "--band" && has) band = std::atoi(argv[++i]);
    else if (a == "--frames" && has) frames = std::max(1, std::atoi(argv[++i]));
    else if (a == "--device" && has) device = std::atoi(argv[++i]);
    else if (a == "--stream") stream_mode = true;
    else if (a == "--no-confidence") want_conf = false;
    else if (a == "--threads" && has) ++i;          // CPU thread count: nothing to set
    else if (a == "--agg" && has) ++i;              // accepted for flag compatibility
    else if (a == "--rf") {}                        // the recursive filter is the path
    else if (a == "--topk" && has && std::atoi(argv[i + 1]) == 2) ++i;
    else {
      std::fprintf(stderr, "unknown or unsupported flag: %s\n", a.c_str());
      return 2;
    }
  }
  if (W <= 0 || H <= 0) return usage(argv[0]);
  de_ctx* ctx = nullptr;
  if (de_ctx_create(&cfg, device, &ctx) != DE_OK) {
    std::fprintf(stderr, "de_dense_gpu: %s\n", de_last_error());
    return 1;
  }
  const size_t WH = size_t(W) * H;
  std::vector<float> disp(WH), margin(WH);
  std::vector<uint8_t> conf(WH);

  if (stream_mode) {
    const int rc = serve_stream(ctx, W, H, want_conf);
    de_ctx_destroy(ctx);
    return rc;
  }

  std::vector<uint8_t> L, R;
  if (!load_y8(lp, WH, &L) || !load_y8(rp, WH, &R)) {
    std::fprintf(stderr, "failed to load %s / %s at %dx%d\n", lp.c_str(), rp.c_str(), W, H);
    de_ctx_destroy(ctx);
    return 1;
  }
  std::vector<float> prior;
  if (!priorp.empty()) {
    std::string why;
    if (!load_prior(priorp, W, H, &prior, &why)) {
      std::fprintf(stderr, "de_dense_gpu: --prior %s: %s\n", priorp.c_str(), why.c_str());
      de_ctx_destroy(ctx);
      return 1;
    }
    if (cfg.subpixel)
      std::fprintf(stderr, "de_dense_gpu: --prior runs without sub-pixel refinement "
                           "(disparities are whole pixels)\n");
  }
  std::vector<float> cand(confp.empty() ? 0 : WH * 6);
  de_stage_timing(1);
  double t_total = 0;
  for (int f = 0; f < frames; ++f) {
    const double t0 = now_ms();
    const int rc0 =
        prior.empty()
            ? de_ctx_dense(ctx, L.data(), R.data(), W, H, disp.data(), margin.data(),
                           conf.data(), cand.empty() ? nullptr : cand.data())
            : de_ctx_dense_prior(ctx, L.data(), R.data(), W, H, prior.data(), band,
                                 disp.data(), margin.data(), conf.data(),
                                 cand.empty() ? nullptr : cand.data());
    if (rc0 != DE_OK) {
      std::fprintf(stderr, "de_dense_gpu: %s\n", de_last_error());
      de_ctx_destroy(ctx);
      return 1;
    }
    t_total = now_ms() - t0;
  }
  float stage[4] = {0, 0, 0, 0};
  int groups = 0;
  de_stage_times(stage, 4, &groups);
  de_stage_timing(0);
  const float g = groups > 0 ? float(groups) : 1.f;
  size_t filled = 0;
  for (float v : disp) filled += std::isfinite(v) ? 1 : 0;
  std::printf("%dx%d  D=%d  iters=%d  device=%d  frames=%d\n", W, H,
              cfg.dmax - cfg.dmin + 1, cfg.iters, device, frames);
  std::printf("census %.1f ms  cost %.1f ms  solve %.1f ms  total %.1f ms  agg=0 iters=%d  "
              "filled %.1f%%\n",
              stage[0] / g, (stage[1] + stage[2]) / g, stage[3] / g, t_total, cfg.iters,
              100.0 * double(filled) / double(WH));
  int rc = 0;
  if (!outp.empty() && !dump(outp, disp.data(), WH)) rc = 1;
  if (!confp.empty() && !dump(confp, cand.data(), WH * 6)) rc = 1;
  if (!kpp.empty()) {
    // the sparse feature set read out of the dense map (de_dense_cuda --keypoints)
    de_det_cfg det;
    de_det_cfg_default(&det);
    std::vector<de_kp_disparity> kd(1 << 16);
    int n = 0, detected = 0;
    const double tk0 = now_ms();
    if (de_ctx_keypoints(ctx, L.data(), W, H, &det, disp.data(), margin.data(), kd.data(),
                         int(kd.size()), &n, &detected) != DE_OK) {
      std::fprintf(stderr, "de_dense_gpu: %s\n", de_last_error());
      de_ctx_destroy(ctx);
      return 1;
    }
    const double tk1 = now_ms();
    FILE* f = std::fopen(kpp.c_str(), "w");
    if (!f) {
      std::fprintf(stderr, "cannot write %s\n", kpp.c_str());
      de_ctx_destroy(ctx);
      return 1;
    }
    std::fprintf(f, "x,y,disparity,margin\n");
    for (int k = 0; k < std::min(n, int(kd.size())); ++k)
      std::fprintf(f, "%.2f,%.2f,%.4f,%.4f\n", kd[k].x, kd[k].y, kd[k].disparity,
                   kd[k].margin);
    std::fclose(f);
    std::printf("keypoints: %d detected in %.1f ms, %d carried a disparity (%.1f%%) -> %s\n",
                detected, tk1 - tk0, n, detected ? 100.0 * n / detected : 0.0, kpp.c_str());
  }
  de_ctx_destroy(ctx);
  return rc;
}
