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
#include <map>
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
    struct Pending { std::vector<uint8_t> img; int stream; };
    std::map<uint32_t, Pending> pending;
    std::vector<int16_t> q(WH);
    long pairs = 0, dropped = 0;
    for (;;) {
      unsigned char hdr[14];
      if (!read_all(hdr, sizeof(hdr))) break;
      if (std::memcmp(hdr, "DEIR", 4) != 0) {
        std::fprintf(stderr, "de_dense_gpu: lost sync (bad magic), stopping\n");
        de_ctx_destroy(ctx);
        return 1;
      }
      uint16_t pw, ph;
      uint32_t num;
      std::memcpy(&pw, hdr + 4, 2);
      std::memcpy(&ph, hdr + 6, 2);
      const int st = hdr[8];
      std::memcpy(&num, hdr + 10, 4);
      if (int(pw) != W || int(ph) != H) {
        std::fprintf(stderr, "de_dense_gpu: stream is %dx%d, this was started for %dx%d\n",
                     int(pw), int(ph), W, H);
        de_ctx_destroy(ctx);
        return 1;
      }
      std::vector<uint8_t> img(WH);
      if (!read_all(img.data(), WH)) break;
      auto it = pending.find(num);
      if (it == pending.end()) {
        pending[num] = Pending{std::move(img), st};
        while (pending.size() > 8) { pending.erase(pending.begin()); ++dropped; }
        continue;
      }
      if (it->second.stream == st) { it->second.img = std::move(img); continue; }
      const std::vector<uint8_t>& lft = (st == 1) ? img : it->second.img;
      const std::vector<uint8_t>& rgt = (st == 1) ? it->second.img : img;
      if (de_ctx_dense(ctx, lft.data(), rgt.data(), W, H, disp.data(), nullptr,
                       want_conf ? conf.data() : nullptr, nullptr) != DE_OK) {
        std::fprintf(stderr, "de_dense_gpu: %s\n", de_last_error());
        de_ctx_destroy(ctx);
        return 1;
      }
      for (size_t i = 0; i < WH; ++i) {
        const float d = disp[i];
        q[i] = (d > 0.f && std::isfinite(d)) ? int16_t(std::lround(d * 16.0f))
                                               : int16_t(-32768);
        if (want_conf && q[i] == int16_t(-32768)) conf[i] = 0;
      }
      unsigned char out[16];
      std::memcpy(out, "DEDD", 4);
      std::memcpy(out + 4, &pw, 2);
      std::memcpy(out + 6, &ph, 2);
      std::memcpy(out + 8, &num, 4);
      const uint32_t flags = want_conf ? 1u : 0u;
      std::memcpy(out + 12, &flags, 4);
      if (!write_all(out, sizeof(out)) || !write_all(lft.data(), WH) ||
          !write_all(q.data(), WH * sizeof(int16_t)) ||
          (want_conf && !write_all(conf.data(), WH)))
        break;
      std::fflush(stdout);
      pending.erase(it);
      if (++pairs % 30 == 0) {
        size_t filled = 0;
        for (size_t i = 0; i < WH; ++i) filled += q[i] != int16_t(-32768);
        std::fprintf(stderr, "de_dense_gpu: %ld pairs, %ld unpaired dropped, %.0f%% filled\n",
                     pairs, dropped, 100.0 * double(filled) / double(WH));
      }
    }
    std::fprintf(stderr, "de_dense_gpu: %ld pairs, %ld unpaired dropped\n", pairs, dropped);
    de_ctx_destroy(ctx);
    return 0;
  }

  std::vector<uint8_t> L, R;
  if (!load_y8(lp, WH, &L) || !load_y8(rp, WH, &R)) {
    std::fprintf(stderr, "failed to load %s / %s at %dx%d\n", lp.c_str(), rp.c_str(), W, H);
    de_ctx_destroy(ctx);
    return 1;
  }
  // --prior F: W*H floats, or (W/2)*(H/2) upsampled by nearest neighbour with the
  // disparity doubled; holes are refused (core/tools/de_dense.cpp:1756-1813)
  std::vector<float> prior;
  if (!priorp.empty()) {
    FILE* f = std::fopen(priorp.c_str(), "rb");
    if (!f) {
      std::fprintf(stderr, "cannot open prior %s\n", priorp.c_str());
      de_ctx_destroy(ctx);
      return 1;
    }
    std::fseek(f, 0, SEEK_END);
    const size_t n = size_t(std::ftell(f)) / sizeof(float);
    std::fseek(f, 0, SEEK_SET);
    std::vector<float> raw(n);
    const size_t got = std::fread(raw.data(), sizeof(float), n, f);
    std::fclose(f);
    const int W2 = W / 2, H2 = H / 2;
    if (got != n || (n != WH && n != size_t(W2) * H2)) {
      std::fprintf(stderr, "prior %s has %zu floats, expected %zu (full) or %zu (half)\n",
                   priorp.c_str(), n, WH, size_t(W2) * H2);
      de_ctx_destroy(ctx);
      return 1;
    }
    prior.resize(WH);
    if (n == WH) {
      prior = raw;
    } else {
      for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
          prior[size_t(y) * W + x] =
              2.f * raw[size_t(std::min(H2 - 1, y / 2)) * W2 + std::min(W2 - 1, x / 2)];
    }
    size_t holes = 0;
    for (float v : prior) holes += std::isfinite(v) ? 0 : 1;
    if (holes) {
      std::fprintf(stderr, "prior has %zu holes of %zu; fill them first\n", holes, WH);
      de_ctx_destroy(ctx);
      return 1;
    }
    if (cfg.subpixel)
      std::fprintf(stderr, "note: --prior disables sub-pixel (masked planes break the "
                           "neighbour invariant); disparities are integer\n");
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
