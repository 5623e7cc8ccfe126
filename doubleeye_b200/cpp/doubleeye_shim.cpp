// The reference's C++ call surface (include/doubleeye/*.hpp) over this build's C ABI.
//
// Every function here moves the caller's host data through a per-thread host-pointer
// context (de_ctx, device 0 unless DOUBLEEYE_DEVICE names another) into the sm_100a
// kernels and back; nothing is computed on the host beyond argument conversion,
// except pair_score and the DisparityPrior lookups, which are the scoring formula
// and a table read the device applies inside match_masda.  Errors from the C ABI are
// thrown as std::runtime_error with de_last_error()'s reason.

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "doubleeye/dense_solve.hpp"
#include "doubleeye/match.hpp"
#include "doubleeye/preproc.hpp"
#include "doubleeye_b200.h"

namespace doubleeye {
namespace {

void check(int rc, const char* what) {
  if (rc != DE_OK) throw std::runtime_error(std::string(what) + ": " + de_last_error());
}

struct CtxDeleter {
  void operator()(de_ctx* c) const { de_ctx_destroy(c); }
};

// The calling thread's context (a de_ctx is used by one thread at a time).
de_ctx* ctx() {
  thread_local std::unique_ptr<de_ctx, CtxDeleter> c;
  if (!c) {
    de_cfg cfg;
    de_cfg_default(&cfg);
    const char* dev = std::getenv("DOUBLEEYE_DEVICE");
    de_ctx* raw = nullptr;
    check(de_ctx_create(&cfg, dev ? std::atoi(dev) : 0, &raw), "doubleeye context");
    c.reset(raw);
  }
  return c.get();
}

de_det_cfg det_cfg(const DetectorConfig& d) {
  de_det_cfg c;
  c.grad_window = d.grad_window;
  c.cell = d.cell;
  c.per_cell = d.per_cell;
  c.min_response = d.min_response;
  c.min_local_std = d.min_local_std;
  c.border = d.border;
  c.subpixel = d.subpixel ? 1 : 0;
  c.fast_threshold = d.fast_threshold;
  c.nms_radius = d.nms_radius;
  return c;
}

// The score scale of match_masda: the reference scales every descriptor distance by 48
// bits (core/src/match.cpp:339), whatever the census window.
constexpr int kMatchCensusBits = 48;

de_match_cfg match_cfg(const MatchConfig& m) {
  de_match_cfg c;
  de_match_cfg_default(&c);
  c.max_dy = m.max_dy;
  c.min_disparity = m.min_disparity;
  c.max_disparity = m.max_disparity;
  c.max_candidates = m.max_candidates;
  c.sigma_y = m.sigma_y;
  c.w_y = m.w_y;
  c.iterations = m.iterations;
  c.damping = m.damping;
  c.lambda = m.lambda;
  c.gamma = m.gamma;
  c.converge_eps = m.converge_eps;
  c.census_bits = kMatchCensusBits;
  return c;
}

static_assert(sizeof(Keypoint) == sizeof(de_keypoint), "Keypoint is de_keypoint's layout");

}  // namespace

// ---- preproc ----------------------------------------------------------------------

CensusImage census_transform(const Image8& img, CensusConfig cfg) {
  CensusImage out;
  out.width = img.width;
  out.height = img.height;
  out.config = cfg;
  if (img.empty()) return out;
  out.bits.assign(img.pixels(), 0ull);
  out.valid.assign(img.pixels(), 0);
  if (cfg.bits() > 64) return out;
  check(de_ctx_census(ctx(), img.data.data(), img.width, img.height, cfg.half_w, cfg.half_h,
                      out.bits.data()),
        "census_transform");
  for (int y = cfg.half_h; y < img.height - cfg.half_h; ++y)
    for (int x = cfg.half_w; x < img.width - cfg.half_w; ++x)
      out.valid[size_t(y) * img.width + x] = 1;
  return out;
}

uint64_t census_at(const Image8& img, int x, int y, CensusConfig cfg, bool* ok) {
  const bool inside = x >= cfg.half_w && y >= cfg.half_h && x < img.width - cfg.half_w &&
                      y < img.height - cfg.half_h;
  if (ok) *ok = inside;
  if (!inside || cfg.bits() > 64) return 0ull;
  de_keypoint kp{float(x), float(y), 0.f, 0.f};
  uint64_t desc = 0;
  uint8_t good = 0;
  check(de_ctx_census_at(ctx(), img.data.data(), img.width, img.height, &kp, 1, cfg.half_w,
                         cfg.half_h, &desc, &good),
        "census_at");
  return desc;
}

std::vector<Keypoint> detect_keypoints_fast(const Image8& img, const DetectorConfig& cfg,
                                            DetectProfile* prof) {
  std::vector<Keypoint> out;
  if (img.empty()) return out;
  const de_det_cfg c = det_cfg(cfg);
  // every cell keeps at most per_cell points, which bounds the output
  const int cells = ((img.width + cfg.cell - 1) / std::max(1, cfg.cell)) *
                    ((img.height + cfg.cell - 1) / std::max(1, cfg.cell));
  out.resize(size_t(std::max(1, cells * std::max(1, cfg.per_cell))));
  int n = 0;
  check(de_ctx_detect_fast(ctx(), img.data.data(), img.width, img.height, &c,
                           reinterpret_cast<de_keypoint*>(out.data()), int(out.size()), &n),
        "detect_keypoints_fast");
  out.resize(size_t(std::min<int>(n, int(out.size()))));
  if (prof) *prof = DetectProfile{};
  return out;
}

// ---- match ------------------------------------------------------------------------

bool DisparityPrior::lookup(float x, float y, float* d, float* sd) const {
  if (cols <= 0 || rows <= 0) return false;
  const int cx = std::min(cols - 1, std::max(0, int(x) / cell));
  const int cy = std::min(rows - 1, std::max(0, int(y) / cell));
  const size_t i = size_t(cy) * cols + cx;
  if (!valid[i]) return false;
  if (d) *d = disparity[i];
  if (sd) *sd = sigma[i];
  return true;
}

float DisparityPrior::coverage() const {
  if (valid.empty()) return 0.f;
  size_t n = 0;
  for (uint8_t v : valid) n += v ? 1 : 0;
  return float(n) / float(valid.size());
}

float pair_score(const Keypoint& l, const Keypoint& r, uint64_t dl, uint64_t dr,
                 int census_bits, const MatchConfig& cfg, int left_index) {
  const float half = 0.5f * float(census_bits);
  const float desc = (half - float(hamming(dl, dr))) / half;
  const float dy = (l.y - r.y) / (cfg.sigma_y > 0 ? cfg.sigma_y : 1.f);
  float score = desc - cfg.w_y * dy * dy;
  float d_pred = 0.f, sd = 1.f;
  if (cfg.prior && cfg.prior->lookup(l.x, l.y, &d_pred, &sd) && sd > 0.f) {
    const float e = ((l.x - r.x) - d_pred) / sd;
    score -= cfg.w_prior * e * e;
  }
  if (cfg.smooth && left_index >= 0 && size_t(left_index) < cfg.smooth->valid.size() &&
      cfg.smooth->valid[left_index]) {
    const float s2 = cfg.smooth->sigma[left_index];
    if (s2 > 0.f) {
      const float e = ((l.x - r.x) - cfg.smooth->disparity[left_index]) / s2;
      score -= cfg.w_smooth * e * e;
    }
  }
  return score;
}

std::vector<Match> match_masda(const std::vector<Keypoint>& left,
                               const std::vector<uint64_t>& desc_left,
                               const std::vector<Keypoint>& right,
                               const std::vector<uint64_t>& desc_right,
                               const MatchConfig& cfg, MatchStats* stats) {
  if (desc_left.size() != left.size() || desc_right.size() != right.size())
    throw std::invalid_argument("match_masda: descriptors must parallel their keypoints");
  const int nl = int(left.size()), nr = int(right.size());
  const de_match_cfg c = match_cfg(cfg);
  // the priors, resolved per left keypoint (sigma 0 = no term there)
  std::vector<float> cd, csd, sd, ssd;
  de_match_prior prior{};
  prior.w_coarse = cfg.w_prior;
  prior.w_smooth = cfg.w_smooth;
  if (cfg.prior) {
    cd.assign(size_t(nl), 0.f);
    csd.assign(size_t(nl), 0.f);
    for (int i = 0; i < nl; ++i) {
      float d = 0.f, s = 0.f;
      if (cfg.prior->lookup(left[i].x, left[i].y, &d, &s) && s > 0.f) { cd[i] = d; csd[i] = s; }
    }
    prior.coarse_d = cd.data();
    prior.coarse_sd = csd.data();
  }
  if (cfg.smooth) {
    sd.assign(size_t(nl), 0.f);
    ssd.assign(size_t(nl), 0.f);
    for (int i = 0; i < nl && size_t(i) < cfg.smooth->valid.size(); ++i)
      if (cfg.smooth->valid[i] && cfg.smooth->sigma[i] > 0.f) {
        sd[i] = cfg.smooth->disparity[i];
        ssd[i] = cfg.smooth->sigma[i];
      }
    prior.smooth_d = sd.data();
    prior.smooth_sd = ssd.data();
  }
  // each left keypoint is matched at most once
  std::vector<Match> out(size_t(std::max(1, nl)));
  int n = 0;
  de_match_stats st{};
  check(de_ctx_match_masda(ctx(), reinterpret_cast<const de_keypoint*>(left.data()),
                           desc_left.data(), nl,
                           reinterpret_cast<const de_keypoint*>(right.data()),
                           desc_right.data(), nr, &c, (cfg.prior || cfg.smooth) ? &prior : nullptr,
                           reinterpret_cast<de_match*>(out.data()), int(out.size()), &n, &st),
        "match_masda");
  out.resize(size_t(std::min<int>(n, int(out.size()))));
  if (stats) {
    stats->left = st.left;
    stats->right = st.right;
    stats->candidates = st.candidates;
    stats->iterations_run = st.iterations_run;
    stats->converged = st.converged != 0;
    stats->final_max_delta = st.final_max_delta;
    stats->oscillating = st.oscillating;
  }
  return out;
}

// ---- dense_solve ------------------------------------------------------------------

void solve_row_sparse(int W, int D, int K, const Cfg& cfg, const float* vol, float* cs,
                      int* cd, int* cn, float* /*beta*/, float* /*rho*/, float* out_disp,
                      float* out_margin, int /*hw*/, int* /*bstart*/, int* /*bitems*/,
                      int* /*cursor*/, float* /*best*/, int* /*bestj*/, int* /*order*/,
                      char* /*taken*/, const float* cnb, float* out_lrc) {
  if (W < 1 || K < 1) return;
  if (vol || K != 2)
    throw std::invalid_argument("solve_row_sparse: this build runs the K = 2 candidate path "
                                "(vol == nullptr)");
  de_cfg c;
  de_cfg_default(&c);
  c.dmin = cfg.dmin;
  c.dmax = std::max(cfg.dmax, cfg.dmin + D - 1);
  c.iters = cfg.iters;
  c.sigma_s = cfg.sigma_s;
  c.sigma_r = cfg.sigma_r;
  c.ad = cfg.ad;
  c.ad_trunc = cfg.ad_trunc;
  c.lambda = cfg.lambda;
  c.gamma = cfg.gamma;
  c.damping = cfg.damping;
  c.min_margin = cfg.min_margin;
  c.min_ratio = cfg.min_ratio;
  c.subpixel = cfg.subpixel ? 1 : 0;
  c.fit_eq = cfg.fit_eq ? 1 : 0;
  std::vector<int16_t> nb;
  if (cnb) {                                         // Q14 costs, -32768 for none
    nb.resize(size_t(W) * 2);
    for (size_t i = 0; i < nb.size(); ++i)
      nb[i] = (cnb[i] > -1e29f) ? int16_t(std::lrint(double(cnb[i]) * 16384.0)) : int16_t(-32768);
  }
  std::vector<float> margin(out_margin ? 0 : size_t(W));
  check(de_ctx_solve(ctx(), &c, W, 1, cs, cd, cn, cnb ? nb.data() : nullptr, out_disp,
                     out_margin ? out_margin : margin.data(), out_lrc),
        "solve_row_sparse");
}

}  // namespace doubleeye
