/*
 * ORACLE -- test infrastructure, not product code.  See de_oracle.h.
 *
 * The dense path in double precision, for the error statement of the fixed-point
 * filter and the single-precision row solve against exact arithmetic:
 *
 *   or_cost_top2_f64   the cost stage with the four filter passes in double and no
 *                      rounding (or_filter_f64), top-2 and sub-pixel neighbours by the
 *                      same insertion rule as or_cost_top2
 *                      (core/tools/de_dense.cpp:1156-1297)
 *   or_solve_row_f64   solve_row_sparse (core/include/doubleeye/dense_solve.hpp:213-434,
 *                      K = 2, candidates from the cost stage) in double
 *   or_dense_f64       both, one image
 *
 * Candidate values are in score units (Q14 / 16384).  Missing candidates and
 * neighbours are -1e300.  Claim order: belief descending, then x (the index
 * tie-break of the single-precision oracle).
 */
#include "de_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NONE64 (-1e300)

static inline double dmax2(double a, double b) { return (a < b) ? b : a; }

void or_cost_top2_f64(const de_cfg* cfg, const uint8_t* L, const uint8_t* R, int W, int H,
                      double* cs, int* cd, int* cn, double* nb) {
  const size_t WH = (size_t)W * H;
  const int D = cfg->dmax - cfg->dmin + 1;
  const int hw = cfg->census_hw, hh = cfg->census_hh;
  uint64_t* cl = malloc(WH * sizeof(uint64_t));
  uint64_t* cr = malloc(WH * sizeof(uint64_t));
  uint16_t* ax = malloc(WH * sizeof(uint16_t));
  uint16_t* ay = malloc(WH * sizeof(uint16_t));
  int16_t* sc = malloc(WH * sizeof(int16_t));
  double* cur = malloc(WH * sizeof(double));
  double* prv = malloc(WH * sizeof(double));
  double* s0 = malloc(WH * sizeof(double));
  double* s1 = malloc(WH * sizeof(double));
  double* nm = malloc(WH * sizeof(double));
  double* np = malloc(WH * sizeof(double));
  int* k0 = malloc(WH * sizeof(int));
  int* k1 = malloc(WH * sizeof(int));
  uint16_t lut[256];
  or_census(L, W, H, hw, hh, cl);
  or_census(R, W, H, hw, hh, cr);
  or_rf_lut(cfg->sigma_s, cfg->sigma_r, lut);
  or_rf_coeffs(L, W, H, lut, ax, ay);
  for (size_t i = 0; i < WH; ++i) {
    s0[i] = s1[i] = nm[i] = np[i] = NONE64;
    k0[i] = k1[i] = -1;
  }
  for (int k = 0; k < D; ++k) {
    const int d = cfg->dmin + k;
    or_score_plane(cfg, L, R, cl, cr, W, H, k, sc);
    for (size_t i = 0; i < WH; ++i) cur[i] = (double)sc[i];
    or_filter_f64(cur, ax, ay, W, H);
    for (int y = hh; y < H - hh; ++y)
      for (int x = hw + d; x < W - hw; ++x) {
        const size_t i = (size_t)y * W + x;
        const double v = cur[i] / 16384.0;
        if (k0[i] == k - 1) np[i] = v;                 /* right neighbour of the best */
        if (v > s0[i]) { nm[i] = (k > 0) ? prv[i] / 16384.0 : NONE64; np[i] = NONE64; }
        if (v <= s1[i]) continue;
        if (v > s0[i]) { s1[i] = s0[i]; k1[i] = k0[i]; s0[i] = v; k0[i] = k; }
        else { s1[i] = v; k1[i] = k; }
      }
    double* t = cur; cur = prv; prv = t;
  }
  for (size_t i = 0; i < WH; ++i) {
    int n = 0;
    cs[2 * i] = cs[2 * i + 1] = NONE64;
    cd[2 * i] = cd[2 * i + 1] = -1;
    if (k0[i] >= 0) { cs[2 * i] = s0[i]; cd[2 * i] = k0[i]; n = 1; }
    if (k1[i] >= 0) { cs[2 * i + 1] = s1[i]; cd[2 * i + 1] = k1[i]; n = 2; }
    cn[i] = n;
    nb[2 * i] = (cfg->subpixel && n > 0) ? nm[i] : NONE64;
    nb[2 * i + 1] = (cfg->subpixel && n > 0) ? np[i] : NONE64;
  }
  free(cl); free(cr); free(ax); free(ay); free(sc); free(cur); free(prv);
  free(s0); free(s1); free(nm); free(np); free(k0); free(k1);
}

typedef struct { double best; int x; } rank64_t;
static int rank64_cmp(const void* pa, const void* pb) {
  const rank64_t* a = pa; const rank64_t* b = pb;
  if (a->best > b->best) return -1;
  if (a->best < b->best) return 1;
  return (a->x > b->x) - (a->x < b->x);
}

/* Best and runner-up over a set, with the index of the best: what "the largest
 * message excluding my own" needs (dense_solve.hpp:174-182). */
typedef struct { double b1, b2; int i1; } top2_64;
static void t64_push(top2_64* t, double v, int i) {
  if (v > t->b1) { t->b2 = t->b1; t->b1 = v; t->i1 = i; }
  else if (v > t->b2) t->b2 = v;
}

void or_solve_row_f64(const de_cfg* cfg, int W, const double* cs, const int* cd,
                      const int* cn, const double* nb, double* disp, double* best_out) {
  const int K = 2, dmin = cfg->dmin;
  const double lam = cfg->lambda, gam = cfg->gamma, damp = cfg->damping;
  const double keep = 1.0 - damp;
  double* beta = calloc((size_t)W * K, sizeof(double));
  double* rho = calloc((size_t)W * K, sizeof(double));
  double* best = malloc((size_t)W * sizeof(double));
  double* margin = malloc((size_t)W * sizeof(double));
  int* bestj = malloc((size_t)W * sizeof(int));
  int* start = calloc((size_t)W + 1, sizeof(int));
  int* items = malloc((size_t)W * K * sizeof(int));
  int* fillp = calloc((size_t)W, sizeof(int));
  char* taken = calloc((size_t)W, 1);
  rank64_t* order = malloc((size_t)W * sizeof(rank64_t));
  /* margin: best minus the larger of the runner-up and lambda (:263-268) */
  for (int x = 0; x < W; ++x) {
    const double alt = cn[x] < 2 ? lam : dmax2(cs[2 * x + 1], lam);
    margin[x] = cn[x] ? cs[2 * x] - alt : 0.0;
  }
  /* the candidates of each right pixel xr = x - d, in (x, j) order (:270-284) */
  for (int x = 0; x < W; ++x)
    for (int j = 0; j < cn[x]; ++j) {
      const int xr = x - (dmin + cd[2 * x + j]);
      if (xr >= 0 && xr < W) ++start[xr + 1];
    }
  for (int xr = 0; xr < W; ++xr) start[xr + 1] += start[xr];
  for (int x = 0; x < W; ++x)
    for (int j = 0; j < cn[x]; ++j) {
      const int xr = x - (dmin + cd[2 * x + j]);
      if (xr >= 0 && xr < W) items[start[xr] + fillp[xr]++] = 2 * x + j;
    }
  /* damped max-sum: rho over a left pixel's candidates, beta over a right pixel's
   * claimants, each against the best other message or the clutter cost (:318-341) */
  for (int it = 0; it < cfg->iters; ++it) {
    for (int x = 0; x < W; ++x) {
      top2_64 t = {NONE64, NONE64, -1};
      for (int j = 0; j < cn[x]; ++j) t64_push(&t, beta[2 * x + j], j);
      for (int j = 0; j < cn[x]; ++j) {
        const double other = (j == t.i1) ? t.b2 : t.b1;
        rho[2 * x + j] = keep * (cs[2 * x + j] - dmax2(lam, other)) + damp * rho[2 * x + j];
      }
    }
    for (int xr = 0; xr < W; ++xr) {
      top2_64 t = {NONE64, NONE64, -1};
      for (int p = start[xr]; p < start[xr + 1]; ++p) t64_push(&t, rho[items[p]], p);
      for (int p = start[xr]; p < start[xr + 1]; ++p) {
        const int c = items[p];
        const double other = (p == t.i1) ? t.b2 : t.b1;
        beta[c] = keep * (cs[c] - dmax2(gam, other)) + damp * beta[c];
      }
    }
  }
  /* belief of each candidate scoring above lambda; the pixel's best (:343-358) */
  for (int x = 0; x < W; ++x) {
    best[x] = NONE64;
    bestj[x] = -1;
    for (int j = 0; j < cn[x]; ++j) {
      const int c = 2 * x + j;
      if (cs[c] <= lam) continue;
      const double b = cfg->iters > 0 ? beta[c] + rho[c] - cs[c] : cs[c];
      if (b > best[x]) { best[x] = b; bestj[x] = j; }
    }
    order[x].best = best[x];
    order[x].x = x;
  }
  qsort(order, (size_t)W, sizeof(rank64_t), rank64_cmp);
  /* one-to-one claim in belief order with the margin / ratio gates, then the
   * sub-pixel fit of the winner against its neighbours (:360-434) */
  for (int r = 0; r < W; ++r) {
    const int x = order[r].x;
    disp[x] = NAN;
    if (bestj[x] < 0) continue;
    if (cfg->min_margin > 0.f && margin[x] < cfg->min_margin) continue;
    if (cfg->min_ratio > 0.f) {
      const double s2 = cn[x] > 1 ? dmax2(cs[2 * x + 1], lam) : lam;
      if ((1.0 - s2) / dmax2(1.0 - cs[2 * x], 1e-6) < cfg->min_ratio) continue;
    }
    const int d = dmin + cd[2 * x + bestj[x]];
    const int xr = x - d;
    if (xr < 0 || taken[xr]) continue;
    taken[xr] = 1;
    double off = 0.0;
    const double cm = nb[2 * x], cp = nb[2 * x + 1], c0 = cs[2 * x];
    if (cfg->subpixel && bestj[x] == 0 && cm > -1e29 && cp > -1e29) {
      const double den = cfg->fit_eq ? c0 - (cm < cp ? cm : cp) : 2.0 * c0 - cm - cp;
      if (den > 1e-6) {
        off = 0.5 * (cp - cm) / den;
        off = off > 0.5 ? 0.5 : (off < -0.5 ? -0.5 : off);
      }
    }
    disp[x] = (double)d + off;
  }
  if (best_out) memcpy(best_out, best, (size_t)W * sizeof(double));
  free(beta); free(rho); free(best); free(margin); free(bestj); free(start); free(items);
  free(fillp); free(taken); free(order);
}

void or_dense_f64(const de_cfg* cfg, const uint8_t* L, const uint8_t* R, int W, int H,
                  double* disp, double* best) {
  const size_t WH = (size_t)W * H;
  double* cs = malloc(WH * 2 * sizeof(double));
  double* nb = malloc(WH * 2 * sizeof(double));
  int* cd = malloc(WH * 2 * sizeof(int));
  int* cn = malloc(WH * sizeof(int));
  or_cost_top2_f64(cfg, L, R, W, H, cs, cd, cn, nb);
  for (int y = 0; y < H; ++y)
    or_solve_row_f64(cfg, W, cs + (size_t)y * W * 2, cd + (size_t)y * W * 2, cn + (size_t)y * W,
                     nb + (size_t)y * W * 2, disp + (size_t)y * W,
                     best ? best + (size_t)y * W : NULL);
  free(cs); free(nb); free(cd); free(cn);
}
