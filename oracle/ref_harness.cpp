// Test infrastructure only.  Exposes the reference implementation (mayio/doubleeye,
// compiled from its own sources in place by oracle/Makefile) through a flat C ABI,
// so the golden-vector script can call the reference's own functions, including the
// ones core/tools/de_dense.cpp keeps in an anonymous namespace.  The reference file
// is #included, not copied: this translation unit IS the reference tool with its
// main() renamed, plus the thin extern "C" shims below.
//
// Built only where the reference tree exists; the output lives in oracle/_ref/.

#define main de_dense_tool_main
#include "de_dense.cpp"   // core/tools/de_dense.cpp, found via -iquote
#undef main

#include "doubleeye/match.hpp"
#include "../include/doubleeye_b200.h"

#include <cstring>

using namespace doubleeye;

namespace {

Image8 wrap(const uint8_t* p, int W, int H) {
  Image8 im(W, H);
  std::memcpy(im.data.data(), p, size_t(W) * H);
  return im;
}

Cfg to_cfg(const de_cfg* c) {
  Cfg cfg;                       // reference defaults for everything not mirrored
  cfg.dmin = c->dmin;
  cfg.dmax = c->dmax;
  cfg.iters = c->iters;
  cfg.sigma_s = c->sigma_s;
  cfg.sigma_r = c->sigma_r;
  cfg.ad = c->ad;
  cfg.ad_trunc = c->ad_trunc;
  cfg.lambda = c->lambda;
  cfg.gamma = c->gamma;
  cfg.damping = c->damping;
  cfg.min_margin = c->min_margin;
  cfg.min_ratio = c->min_ratio;
  cfg.subpixel = c->subpixel != 0;
  cfg.fit_eq = c->fit_eq != 0;
  cfg.lrc = c->lrc != 0;
  return cfg;
}

}  // namespace

extern "C" {

// census_image (core/tools/de_dense.cpp:186-227), one thread.
void ref_census_image(const uint8_t* img, int W, int H, int hw, int hh, uint64_t* out) {
  const Image8 im = wrap(img, W, H);
  const std::vector<uint64_t> c = census_image(im, hw, hh, 1);
  std::memcpy(out, c.data(), c.size() * sizeof(uint64_t));
}

// rf_coeffs (core/tools/de_dense.cpp:531-561), one thread.
void ref_rf_coeffs(const uint8_t* img, int W, int H, float sigma_s, float sigma_r,
                   uint16_t* ax, uint16_t* ay) {
  rf_coeffs(img, ax, ay, W, H, sigma_s, sigma_r, 1);
}

// rf_filter_i16 (core/tools/de_dense.cpp:485-508), in place.
void ref_rf_filter_i16(int16_t* plane, const uint16_t* ax, const uint16_t* ay, int W,
                       int H) {
  rf_filter_i16(plane, ax, ay, W, H);
}

// rf_filter, the float variant (core/tools/de_dense.cpp:510-527), in place.
void ref_rf_filter_f32(float* plane, const uint16_t* ax, const uint16_t* ay, int W,
                       int H) {
  rf_filter(plane, ax, ay, W, H);
}

// run_dense (core/tools/de_dense.cpp:738-1608) on the default path.  cand (6*W*H)
// may be NULL.  Returns the stage wall times through t3 = {census, cost, solve} ms.
void ref_run_dense(const uint8_t* L, const uint8_t* R, int W, int H, const de_cfg* c,
                   int nthreads, float* disp, float* margin, float* cand, double* t3) {
  const Image8 li = wrap(L, W, H), ri = wrap(R, W, H);
  const Cfg cfg = to_cfg(c);
  std::vector<float> d, m, cd;
  LevelTimes T;
  run_dense(li, ri, cfg, nthreads < 1 ? 1 : nthreads, {}, "", &d, &m, &T,
            cand ? &cd : nullptr);
  std::memcpy(disp, d.data(), d.size() * sizeof(float));
  if (margin) std::memcpy(margin, m.data(), m.size() * sizeof(float));
  if (cand) std::memcpy(cand, cd.data(), cd.size() * sizeof(float));
  if (t3) { t3[0] = T.census; t3[1] = T.cost; t3[2] = T.solve; }
}

// run_dense with a full-resolution disparity prior as the per-plane mask
// (core/tools/de_dense.cpp:738-1608 with prior; cfg.band = band, sub-pixel off as the
// tool forces it under --prior, :1824-1839).
void ref_run_dense_prior(const uint8_t* L, const uint8_t* R, int W, int H, const de_cfg* c,
                         int band, const float* prior, int nthreads, float* disp,
                         float* margin, float* cand) {
  const Image8 li = wrap(L, W, H), ri = wrap(R, W, H);
  Cfg cfg = to_cfg(c);
  cfg.band = band;
  cfg.subpixel = false;
  std::vector<float> pr(prior, prior + size_t(W) * H);
  std::vector<float> d, m, cd;
  LevelTimes T;
  run_dense(li, ri, cfg, nthreads < 1 ? 1 : nthreads, pr, "", &d, &m, &T,
            cand ? &cd : nullptr);
  std::memcpy(disp, d.data(), d.size() * sizeof(float));
  if (margin) std::memcpy(margin, m.data(), m.size() * sizeof(float));
  if (cand) std::memcpy(cand, cd.data(), cd.size() * sizeof(float));
}

float ref_confidence(float s1, float s2, float lambda, float lrc, float lrc_tol) {
  return confidence(s1, s2, lambda, lrc, lrc_tol);
}

unsigned ref_confidence_u8(float s1, float s2, float lambda, float lrc, float lrc_tol) {
  return confidence_u8(s1, s2, lambda, lrc, lrc_tol);
}

// census_at (core/src/preproc.cpp:142-162).
uint64_t ref_census_at(const uint8_t* img, int W, int H, int x, int y, int hw, int hh,
                       int* ok) {
  const Image8 im = wrap(img, W, H);
  CensusConfig cc;
  cc.half_w = hw;
  cc.half_h = hh;
  bool okb = false;
  const uint64_t v = census_at(im, x, y, cc, &okb);
  if (ok) *ok = okb ? 1 : 0;
  return v;
}

// detect_keypoints_fast (core/src/preproc.cpp:442-545).  Returns the count; writes
// at most cap keypoints.
int ref_detect_fast(const uint8_t* img, int W, int H, const de_det_cfg* c,
                    de_keypoint* out, int cap) {
  const Image8 im = wrap(img, W, H);
  DetectorConfig d;
  d.grad_window = c->grad_window;
  d.cell = c->cell;
  d.per_cell = c->per_cell;
  d.min_response = c->min_response;
  d.min_local_std = c->min_local_std;
  d.border = c->border;
  d.subpixel = c->subpixel != 0;
  d.fast_threshold = c->fast_threshold;
  d.nms_radius = c->nms_radius;
  const std::vector<Keypoint> kp = detect_keypoints_fast(im, d);
  const int n = int(kp.size());
  for (int i = 0; i < n && i < cap; ++i)
    out[i] = de_keypoint{kp[i].x, kp[i].y, kp[i].response, kp[i].local_std};
  return n;
}

// match_masda (core/src/match.cpp:334-417).  Returns the match count; writes at
// most cap matches in the reference's emission order.
int ref_match_masda(const de_keypoint* kl, const uint64_t* dl, int nl,
                    const de_keypoint* kr, const uint64_t* dr, int nr,
                    const de_match_cfg* c, de_match* out, int cap,
                    de_match_stats* st) {
  std::vector<Keypoint> L(nl), R(nr);
  for (int i = 0; i < nl; ++i) L[i] = Keypoint{kl[i].x, kl[i].y, kl[i].response, kl[i].local_std};
  for (int j = 0; j < nr; ++j) R[j] = Keypoint{kr[j].x, kr[j].y, kr[j].response, kr[j].local_std};
  std::vector<uint64_t> DL(dl, dl + nl), DR(dr, dr + nr);
  MatchConfig m;
  m.max_dy = c->max_dy;
  m.min_disparity = c->min_disparity;
  m.max_disparity = c->max_disparity;
  m.max_candidates = c->max_candidates;
  m.sigma_y = c->sigma_y;
  m.w_y = c->w_y;
  m.iterations = c->iterations;
  m.damping = c->damping;
  m.lambda = c->lambda;
  m.gamma = c->gamma;
  m.converge_eps = c->converge_eps;
  MatchStats s;
  const std::vector<Match> res = match_masda(L, DL, R, DR, m, &s);
  const int n = int(res.size());
  for (int i = 0; i < n && i < cap; ++i)
    out[i] = de_match{res[i].left, res[i].right, res[i].score, res[i].belief,
                      res[i].disparity, res[i].dy, res[i].margin};
  if (st) *st = de_match_stats{s.left, s.right, s.candidates, s.iterations_run,
                               s.converged ? 1 : 0, s.final_max_delta, s.oscillating};
  return n;
}

// match_brute_force (core/src/match.cpp:480-545), for optimality checks.
int ref_match_brute_force(const de_keypoint* kl, const uint64_t* dl, int nl,
                          const de_keypoint* kr, const uint64_t* dr, int nr,
                          const de_match_cfg* c, de_match* out, int cap) {
  std::vector<Keypoint> L(nl), R(nr);
  for (int i = 0; i < nl; ++i) L[i] = Keypoint{kl[i].x, kl[i].y, kl[i].response, kl[i].local_std};
  for (int j = 0; j < nr; ++j) R[j] = Keypoint{kr[j].x, kr[j].y, kr[j].response, kr[j].local_std};
  std::vector<uint64_t> DL(dl, dl + nl), DR(dr, dr + nr);
  MatchConfig m;
  m.max_dy = c->max_dy;
  m.min_disparity = c->min_disparity;
  m.max_disparity = c->max_disparity;
  m.max_candidates = c->max_candidates;
  m.sigma_y = c->sigma_y;
  m.w_y = c->w_y;
  m.iterations = c->iterations;
  m.damping = c->damping;
  m.lambda = c->lambda;
  m.gamma = c->gamma;
  m.converge_eps = c->converge_eps;
  const std::vector<Match> res = match_brute_force(L, DL, R, DR, m);
  const int n = int(res.size());
  for (int i = 0; i < n && i < cap; ++i)
    out[i] = de_match{res[i].left, res[i].right, res[i].score, res[i].belief,
                      res[i].disparity, res[i].dy, res[i].margin};
  return n;
}

}  // extern "C"
