// doubleeye_b200 -- the C++14 call surface of core/include/doubleeye/dense_solve.hpp
// (mayio/doubleeye): the dense matcher's configuration, confidence and row solve,
// backed by the B200 build.
//
// Same namespace, type names, members, defaults and signatures as the reference
// header.  Cfg keeps every field of the reference's (fields of paths this build does
// not run -- guided and box filters, --csct, --simd, --c2f, the full-volume path -- are
// carried and ignored).
//
// Defined by this build:
//   confidence, confidence_u8   inline, over de_confidence (the same float arithmetic
//                               as the reference's)
//   solve_row_sparse            one row through the GPU row solve (de_ctx_solve): the
//                               path the dense tools take, K = 2 candidates from the
//                               cost stage (vol == nullptr).  The scratch arguments
//                               (beta ... taken) are accepted and unused: the device
//                               keeps its own.  cnb values are the cost stage's Q14
//                               costs (multiples of 1/16384) or -1e30.  A full volume
//                               (vol != nullptr) or K != 2 throws std::invalid_argument.

#ifndef DOUBLEEYE_DENSE_SOLVE_HPP
#define DOUBLEEYE_DENSE_SOLVE_HPP

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "doubleeye_b200.h"

namespace doubleeye {

struct Cfg {
  int dmin = 1, dmax = 60, iters = 0, agg = 3;
  bool rf = true;              // recursive edge-aware filter
  float sigma_s = 8.f, sigma_r = 0.20f;
  bool fit_eq = true;          // equiangular sub-pixel fit (parabola when false)
  bool subpixel = true;
  bool guided = true;
  float eps = 0.0025f;
  int fgf = 1;
  int topk = 2;                // candidates per pixel
  int band = 2;                // prior band, +-band around the prior
  bool csct = false;
  float ad = 0.15f;            // weight of the truncated absolute difference
  int ad_trunc = 10;
  float lambda = -0.1f, gamma = -0.1f, damping = 0.4f, min_margin = 0.f;
  float min_ratio = 0.f;
  bool lrc = false;
  int threads = 0;
  bool simd = false;
  bool c2f = false;
  bool noblock = false;
};

// The calibrated probability that a pixel's answer is right, from its two best scores
// (and a reverse-match residual above lrc_tol, which caps it).
inline float confidence(float s1, float s2, float lambda, float lrc = 0.f,
                        float lrc_tol = 1.f) {
  return de_confidence(s1, s2, lambda, lrc, lrc_tol);
}

inline uint8_t confidence_u8(float s1, float s2, float lambda, float lrc = 0.f,
                             float lrc_tol = 1.f) {
  return uint8_t(std::lround(confidence(s1, s2, lambda, lrc, lrc_tol) * 255.f));
}

// Best and runner-up of a set, with the best's index: "the largest message except
// my own" is excl(me).
struct Top2 {
  float b1 = -1e30f, b2 = -1e30f;
  int i1 = -1;
  inline void push(float v, int i) {
    if (v > b1) { b2 = b1; b1 = v; i1 = i; }
    else if (v > b2) { b2 = v; }
  }
  inline float excl(int i) const { return i == i1 ? b2 : b1; }
};

void solve_row_sparse(int W, int D, int K, const Cfg& cfg, const float* vol,
                      float* cs, int* cd, int* cn,
                      float* beta, float* rho,
                      float* out_disp, float* out_margin, int hw,
                      int* bstart, int* bitems, int* cursor,
                      float* best, int* bestj, int* order, char* taken,
                      const float* cnb = nullptr, float* out_lrc = nullptr);

}  // namespace doubleeye

#endif  // DOUBLEEYE_DENSE_SOLVE_HPP
