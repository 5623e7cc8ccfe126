/*
 * ORACLE -- test infrastructure, not product code.  See de_oracle.h.
 *
 * Single-threaded C restatement of the reference dense matcher, written to the
 * semantics of `de_dense --threads 1` (the reference's own bit-exact oracle,
 * core/tools/de_dense.cpp with nthreads = 1).  Float arithmetic is plain IEEE
 * single precision without contraction (built with -ffp-contract=off), as in the
 * reference's x86-64 build.
 */
#include "de_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define Q14 16384
#define NEG_BIG (-1e30f)

static inline float fmax_ref(float a, float b) { return (a < b) ? b : a; } /* std::max */
static inline float fmin_ref(float a, float b) { return (b < a) ? b : a; } /* std::min */
static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* Census: core/tools/de_dense.cpp:94-129 (7x7 byte-plane form), :196-226 (any
 * window), core/src/preproc.cpp:142-162 (census_at).  Bit b counts window
 * positions in row-major order with the centre skipped and is set where that
 * neighbour is strictly darker than the centre; pixels whose window leaves the
 * image are 0. */
void or_census(const uint8_t* img, int W, int H, int hw, int hh, uint64_t* out) {
  memset(out, 0, sizeof(uint64_t) * (size_t)W * (size_t)H);
  for (int y = hh; y < H - hh; ++y)
    for (int x = hw; x < W - hw; ++x) {
      const uint8_t c = img[(size_t)y * W + x];
      uint64_t v = 0;
      int b = 0;
      for (int dy = -hh; dy <= hh; ++dy)
        for (int dx = -hw; dx <= hw; ++dx) {
          if (dx == 0 && dy == 0) continue;
          if (img[(size_t)(y + dy) * W + (x + dx)] < c) v |= 1ull << b;
          ++b;
        }
      out[(size_t)y * W + x] = v;
    }
}

/* Filter coefficient per byte difference: core/tools/de_dense.cpp:533-546 (same
 * expression, float, std::exp = expf, truncating conversion). */
void or_rf_lut(float sigma_s, float sigma_r, uint16_t lut[256]) {
  const float kk = -sqrtf(2.f) / sigma_s;
  const float rs = sigma_s / sigma_r;
  for (int d = 0; d < 256; ++d) {
    const float c = expf(kk * (1.f + rs * ((float)d / 255.f)));
    lut[d] = (uint16_t)fmin_ref(32767.f, c * 32768.f + 0.5f);
  }
}

/* Coefficient planes: core/tools/de_dense.cpp:548-558.  ax[y][x] steps into x from
 * x-1, ay[y][x] into y from y-1; the first column / row take lut[0]. */
void or_rf_coeffs(const uint8_t* L, int W, int H, const uint16_t lut[256], uint16_t* ax,
                  uint16_t* ay) {
  for (int y = 0; y < H; ++y) {
    const uint8_t* r = L + (size_t)y * W;
    const uint8_t* u = L + (size_t)(y > 0 ? y - 1 : 0) * W;
    uint16_t* axr = ax + (size_t)y * W;
    uint16_t* ayr = ay + (size_t)y * W;
    axr[0] = lut[0];
    for (int x = 1; x < W; ++x) axr[x] = lut[abs((int)r[x] - (int)r[x - 1])];
    for (int x = 0; x < W; ++x) ayr[x] = (y == 0) ? lut[0] : lut[abs((int)r[x] - (int)u[x])];
  }
}

/* Q14 score tables: core/tools/de_dense.cpp:1201-1223.  tbl[h] = (half-h)*2^14/half
 * with C truncating division (half = bits/2 = 24 for 7x7); adt[v] is the truncated
 * absolute difference mapped to +-2^14.  Returns wq = weight of the AD term in 1/1024. */
int or_score_tables(const de_cfg* cfg, int16_t tbl[65], int16_t adt[256]) {
  const int nbits = (2 * cfg->census_hw + 1) * (2 * cfg->census_hh + 1) - 1;
  const int half = nbits / 2;
  memset(tbl, 0, 65 * sizeof(int16_t));
  for (int h = 0; h <= 2 * half && h <= 64; ++h)
    tbl[h] = (int16_t)(((half - h) * Q14) / half);
  const int T = imax(1, cfg->ad_trunc);
  for (int v = 0; v < 256; ++v) adt[v] = (int16_t)(Q14 - (2 * Q14 * imin(v, T)) / T);
  return (int)(fmax_ref(0.f, fmin_ref(1.f, cfg->ad)) * 1024.f);
}

/* One recursive-filter step, core/tools/de_dense.cpp:419 (int32 carry, +-2^14
 * rounding, arithmetic shift). */
static inline int32_t rf_step(int32_t c, int32_t f, int32_t a) {
  return c + ((a * (f - c) + (1 << 14)) >> 15);
}

/* rf_filter_i16, core/tools/de_dense.cpp:411-430 and :485-508: per row forward then
 * backward (backward coefficient at x+1), then vertical forward over all rows, then
 * vertical backward (coefficient at y+1).  The whole plane, border included. */
void or_filter_i16(int16_t* C, const uint16_t* ax, const uint16_t* ay, int W, int H) {
  for (int y = 0; y < H; ++y) {
    int16_t* row = C + (size_t)y * W;
    const uint16_t* a = ax + (size_t)y * W;
    int32_t f = row[0];
    for (int x = 1; x < W; ++x) { f = rf_step(row[x], f, a[x]); row[x] = (int16_t)f; }
    f = row[W - 1];
    for (int x = W - 2; x >= 0; --x) { f = rf_step(row[x], f, a[x + 1]); row[x] = (int16_t)f; }
  }
  for (int y = 1; y < H; ++y) {
    int16_t* cur = C + (size_t)y * W;
    const int16_t* prv = C + (size_t)(y - 1) * W;
    const uint16_t* a = ay + (size_t)y * W;
    for (int x = 0; x < W; ++x) cur[x] = (int16_t)rf_step(cur[x], prv[x], a[x]);
  }
  for (int y = H - 2; y >= 0; --y) {
    int16_t* cur = C + (size_t)y * W;
    const int16_t* nxt = C + (size_t)(y + 1) * W;
    const uint16_t* a = ay + (size_t)(y + 1) * W;
    for (int x = 0; x < W; ++x) cur[x] = (int16_t)rf_step(cur[x], nxt[x], a[x]);
  }
}

/* The same four passes in double precision without rounding, the exact-arithmetic
 * counterpart of rf_filter (core/tools/de_dense.cpp:380-396,510-527) used to state
 * the error of the fixed-point filter. */
void or_filter_f64(double* C, const uint16_t* ax, const uint16_t* ay, int W, int H) {
  const double s = 1.0 / 32768.0;
  for (int y = 0; y < H; ++y) {
    double* row = C + (size_t)y * W;
    const uint16_t* a = ax + (size_t)y * W;
    double f = row[0];
    for (int x = 1; x < W; ++x) { f = row[x] + a[x] * s * (f - row[x]); row[x] = f; }
    f = row[W - 1];
    for (int x = W - 2; x >= 0; --x) { f = row[x] + a[x + 1] * s * (f - row[x]); row[x] = f; }
  }
  for (int y = 1; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      double* c = C + (size_t)y * W + x;
      *c += ay[(size_t)y * W + x] * s * (C[(size_t)(y - 1) * W + x] - *c);
    }
  for (int y = H - 2; y >= 0; --y)
    for (int x = 0; x < W; ++x) {
      double* c = C + (size_t)y * W + x;
      *c += ay[(size_t)(y + 1) * W + x] * s * (C[(size_t)(y + 1) * W + x] - *c);
    }
}

/* Graded score of plane k (disparity d = dmin + k): core/tools/de_dense.cpp:1224-1233.
 * v = (tbl[popcount(cl ^ cr)] * (1024 - wq) + adt[|L - R|] * wq) >> 10 on the valid
 * window y in [hh, H-hh), x in [hw + d, W - hw); 0 elsewhere. */
void or_score_plane(const de_cfg* cfg, const uint8_t* L, const uint8_t* R,
                    const uint64_t* cl, const uint64_t* cr, int W, int H, int k,
                    int16_t* plane) {
  int16_t tbl[65], adt[256];
  const int wq = or_score_tables(cfg, tbl, adt);
  const int hw = cfg->census_hw, hh = cfg->census_hh;
  const int d = cfg->dmin + k;
  memset(plane, 0, sizeof(int16_t) * (size_t)W * H);
  for (int y = hh; y < H - hh; ++y)
    for (int x = hw + d; x < W - hw; ++x) {
      const size_t i = (size_t)y * W + x;
      const int32_t c = tbl[__builtin_popcountll(cl[i] ^ cr[i - d])];
      const int32_t a = adt[abs((int)L[i] - (int)R[i - d])];
      plane[i] = (int16_t)((c * (1024 - wq) + a * wq) >> 10);
    }
}

/* Cost stage with the running top-2: core/tools/de_dense.cpp:1156-1297 at one
 * thread.  Planes in ascending k; insert is strictly-greater (ties keep the smaller
 * k, the runner-up slot takes ties with the best); the sub-pixel neighbours of the
 * running best are captured before each update (:1276-1285), the left one from the
 * previous plane.  Outputs the reference candidate layout of
 * core/tools/de_dense_cuda.cu:286-392; empty slots hold cs = -1e30, cd = -1.
 * rbest_k (may be NULL): per RIGHT pixel the k of the best score any left pixel gave
 * it, first of equals (the --lrc reverse match, :1138-1141,1272-1275), -1 if none. */
void or_cost_top2(const de_cfg* cfg, const uint8_t* L, const uint8_t* R, int W, int H,
                  float* cs, int* cd, int* cn, int16_t* cnb, int16_t* rbest_k) {
  const size_t WH = (size_t)W * H;
  const int D = cfg->dmax - cfg->dmin + 1;
  const int hw = cfg->census_hw, hh = cfg->census_hh;
  const int sub = cfg->subpixel != 0;
  uint64_t* cl = malloc(WH * sizeof(uint64_t));
  uint64_t* cr = malloc(WH * sizeof(uint64_t));
  uint16_t* ax = malloc(WH * sizeof(uint16_t));
  uint16_t* ay = malloc(WH * sizeof(uint16_t));
  int16_t* cur = malloc(WH * sizeof(int16_t));
  int16_t* prv = malloc(WH * sizeof(int16_t));
  int16_t *ts0 = malloc(WH * 2), *ts1 = malloc(WH * 2), *td0 = malloc(WH * 2),
          *td1 = malloc(WH * 2), *tm0 = malloc(WH * 2), *tp0 = malloc(WH * 2),
          *trs = malloc(WH * 2);
  uint16_t lut[256];
  or_census(L, W, H, hw, hh, cl);
  or_census(R, W, H, hw, hh, cr);
  or_rf_lut(cfg->sigma_s, cfg->sigma_r, lut);
  or_rf_coeffs(L, W, H, lut, ax, ay);
  for (size_t i = 0; i < WH; ++i) {
    ts0[i] = ts1[i] = -32768;
    td0[i] = td1[i] = -1;
    tm0[i] = tp0[i] = -32768;
    trs[i] = -32768;
    if (rbest_k) rbest_k[i] = -1;
  }
  for (int k = 0; k < D; ++k) {
    const int d = cfg->dmin + k;
    or_score_plane(cfg, L, R, cl, cr, W, H, k, cur);
    or_filter_i16(cur, ax, ay, W, H);
    for (int y = hh; y < H - hh; ++y)
      for (int x = hw + d; x < W - hw; ++x) {
        const size_t i = (size_t)y * W + x;
        const int16_t v = cur[i];
        if (rbest_k && v > trs[i - d]) { trs[i - d] = v; rbest_k[i - d] = (int16_t)k; }
        if (sub) {
          if (td0[i] == k - 1) tp0[i] = v;
          if (v > ts0[i]) { tm0[i] = (k > 0) ? prv[i] : (int16_t)-32768; tp0[i] = -32768; }
        }
        if (v <= ts1[i]) continue;
        if (v > ts0[i]) { ts1[i] = ts0[i]; td1[i] = td0[i]; ts0[i] = v; td0[i] = (int16_t)k; }
        else { ts1[i] = v; td1[i] = (int16_t)k; }
      }
    int16_t* t = cur; cur = prv; prv = t;
  }
  const float q = 1.f / (float)Q14;
  for (size_t i = 0; i < WH; ++i) {
    int n = 0;
    cs[2 * i] = cs[2 * i + 1] = NEG_BIG;
    cd[2 * i] = cd[2 * i + 1] = -1;
    if (td0[i] >= 0) { cs[2 * i] = (float)ts0[i] * q; cd[2 * i] = td0[i]; n = 1; }
    if (td1[i] >= 0) { cs[2 * i + 1] = (float)ts1[i] * q; cd[2 * i + 1] = td1[i]; n = 2; }
    cn[i] = n;
    if (cnb) {
      cnb[2 * i] = (sub && n > 0) ? tm0[i] : (int16_t)-32768;
      cnb[2 * i + 1] = (sub && n > 0) ? tp0[i] : (int16_t)-32768;
    }
  }
  free(cl); free(cr); free(ax); free(ay); free(cur); free(prv);
  free(ts0); free(ts1); free(td0); free(td1); free(tm0); free(tp0); free(trs);
}

/* Top2 of core/include/doubleeye/dense_solve.hpp:174-182. */
typedef struct { float b1, b2; int i1; } top2_t;
static inline void t2_init(top2_t* t) { t->b1 = NEG_BIG; t->b2 = NEG_BIG; t->i1 = -1; }
static inline void t2_push(top2_t* t, float v, int i) {
  if (v > t->b1) { t->b2 = t->b1; t->b1 = v; t->i1 = i; }
  else if (v > t->b2) t->b2 = v;
}
static inline float t2_excl(const top2_t* t, int i) { return i == t->i1 ? t->b2 : t->b1; }

typedef struct { float best; int x; } rank_t;
/* Claim order: belief descending, then x ascending.  The reference uses std::sort on
 * belief alone (dense_solve.hpp:359), whose order among exact ties is unspecified. */
static int rank_cmp(const void* pa, const void* pb) {
  const rank_t* a = pa; const rank_t* b = pb;
  if (a->best > b->best) return -1;
  if (a->best < b->best) return 1;
  return (a->x > b->x) - (a->x < b->x);
}

/* solve_row_sparse, core/include/doubleeye/dense_solve.hpp:213-452, for the path
 * the dense tools take: K = 2, no volume (candidates from the cost stage), cnb =
 * the winner's neighbour costs.  cnb here is Q14 int16 with -32768 for none (the
 * GPU tool's wire form, dequantised as core/tools/de_dense_cuda.cu:645-649 does). */
static void solve_row_impl(const de_cfg* cfg, int W, const float* cs, const int* cd,
                           const int* cn, const int16_t* cnb, float* disp, float* margin,
                           float* lrc2, float* best_out, int* target_out);

void or_solve_row(const de_cfg* cfg, int W, const float* cs, const int* cd, const int* cn,
                  const int16_t* cnb, float* disp, float* margin, float* lrc2) {
  solve_row_impl(cfg, W, cs, cd, cn, cnb, disp, margin, lrc2, NULL, NULL);
}

/* The same solve, also returning each pixel's belief and the right pixel it would
 * claim (-1 when it is not eligible to claim): what a tie-aware comparison needs to
 * tell an exact-tie claim conflict from a real difference. */
void or_solve_row_debug(const de_cfg* cfg, int W, const float* cs, const int* cd,
                        const int* cn, const int16_t* cnb, float* disp, float* margin,
                        float* lrc2, float* best_out, int* target_out) {
  solve_row_impl(cfg, W, cs, cd, cn, cnb, disp, margin, lrc2, best_out, target_out);
}

static void solve_row_impl(const de_cfg* cfg, int W, const float* cs, const int* cd,
                           const int* cn, const int16_t* cnb, float* disp, float* margin,
                           float* lrc2, float* best_out, int* target_out) {
  const int K = 2;
  const int dmin = cfg->dmin;
  const float keep = 1.f - cfg->damping;
  const float q = 1.f / (float)Q14;
  float* beta = calloc((size_t)W * K, sizeof(float));
  float* rho = calloc((size_t)W * K, sizeof(float));
  int* bstart = calloc((size_t)W + 1, sizeof(int));
  int* bitems = calloc((size_t)W * K, sizeof(int));
  int* cursor = calloc((size_t)W, sizeof(int));
  int* rev = calloc((size_t)W, sizeof(int));
  float* best = calloc((size_t)W, sizeof(float));
  int* bestj = calloc((size_t)W, sizeof(int));
  char* taken = calloc((size_t)W, 1);
  rank_t* order = calloc((size_t)W, sizeof(rank_t));

  /* margin, :263-268 */
  for (int x = 0; x < W; ++x) {
    const float* S = cs + (size_t)x * K;
    const int n = cn[x];
    const float alt = (n < 2) ? cfg->lambda : fmax_ref(S[1], cfg->lambda);
    margin[x] = (n == 0) ? 0.f : S[0] - alt;
  }
  /* claimant buckets by right pixel, counting sort in (x, j) order, :270-284 */
  for (int x = 0; x < W; ++x)
    for (int j = 0; j < cn[x]; ++j) {
      const int xr = x - (dmin + cd[(size_t)x * K + j]);
      if (xr >= 0 && xr < W) ++cursor[xr];
    }
  bstart[0] = 0;
  for (int xr = 0; xr < W; ++xr) bstart[xr + 1] = bstart[xr] + cursor[xr];
  for (int xr = 0; xr < W; ++xr) cursor[xr] = bstart[xr];
  for (int x = 0; x < W; ++x)
    for (int j = 0; j < cn[x]; ++j) {
      const int xr = x - (dmin + cd[(size_t)x * K + j]);
      if (xr >= 0 && xr < W) bitems[cursor[xr]++] = x * K + j;
    }
  /* reverse match over the surviving candidates, :303-313 (first maximum wins) */
  for (int xr = 0; xr < W; ++xr) {
    int bd = -1;
    float bv = NEG_BIG;
    for (int p = bstart[xr]; p < bstart[xr + 1]; ++p) {
      const int idx = bitems[p];
      if (cs[idx] > bv) { bv = cs[idx]; bd = cd[idx]; }
    }
    rev[xr] = bd;
  }
  /* damped max-sum iterations, :318-341 */
  for (int it = 0; it < cfg->iters; ++it) {
    for (int x = 0; x < W; ++x) {
      const int n = cn[x];
      if (n == 0) continue;
      const size_t b = (size_t)x * K;
      top2_t t;
      t2_init(&t);
      for (int j = 0; j < n; ++j) t2_push(&t, beta[b + j], j);
      for (int j = 0; j < n; ++j) {
        const float tgt = cs[b + j] - fmax_ref(cfg->lambda, t2_excl(&t, j));
        rho[b + j] = keep * tgt + cfg->damping * rho[b + j];
      }
    }
    for (int xr = 0; xr < W; ++xr) {
      const int lo = bstart[xr], hi = bstart[xr + 1];
      if (hi <= lo) continue;
      top2_t t;
      t2_init(&t);
      for (int p = lo; p < hi; ++p) t2_push(&t, rho[bitems[p]], p - lo);
      for (int p = lo; p < hi; ++p) {
        const int idx = bitems[p];
        beta[idx] = keep * (cs[idx] - fmax_ref(cfg->gamma, t2_excl(&t, p - lo))) +
                    cfg->damping * beta[idx];
      }
    }
  }
  /* belief (WTA on the score at iters 0), :343-358 */
  for (int x = 0; x < W; ++x) {
    best[x] = NEG_BIG;
    bestj[x] = -1;
    const size_t b = (size_t)x * K;
    for (int j = 0; j < cn[x]; ++j) {
      if (cs[b + j] <= cfg->lambda) continue;
      const float bel = (cfg->iters > 0) ? (beta[b + j] + rho[b + j] - cs[b + j]) : cs[b + j];
      if (bel > best[x]) { best[x] = bel; bestj[x] = j; }
    }
    order[x].best = best[x];
    order[x].x = x;
  }
  qsort(order, (size_t)W, sizeof(rank_t), rank_cmp);
  if (target_out)
    for (int x = 0; x < W; ++x) target_out[x] = -1;
  /* greedy one-to-one claim with gates and sub-pixel fit, :360-434 */
  for (int oi = 0; oi < W; ++oi) {
    const int x = order[oi].x;
    disp[x] = NAN;
    if (bestj[x] < 0) continue;
    if (cfg->min_margin > 0.f && margin[x] < cfg->min_margin) continue;
    const size_t b = (size_t)x * K;
    if (cfg->min_ratio > 0.f) {
      const float s2 = (cn[x] > 1) ? fmax_ref(cs[b + 1], cfg->lambda) : cfg->lambda;
      const float c1 = fmax_ref(1.f - cs[b], 1e-6f);
      if ((1.f - s2) / c1 < cfg->min_ratio) continue;
    }
    const int d = dmin + cd[b + bestj[x]];
    const int xr = x - d;
    if (target_out) target_out[x] = xr;
    if (xr < 0 || taken[xr]) continue;
    taken[xr] = 1;
    float off = 0.f;
    if (cfg->subpixel && cnb && bestj[x] == 0) {
      const float c0 = cs[b];
      const int16_t m = cnb[(size_t)x * 2], p = cnb[(size_t)x * 2 + 1];
      const float cm = (m == -32768) ? NEG_BIG : (float)m * q;
      const float cp = (p == -32768) ? NEG_BIG : (float)p * q;
      if (cm > -1e29f && cp > -1e29f) {
        if (cfg->fit_eq) {
          const float lower = cm < cp ? cm : cp;
          const float den = c0 - lower;
          if (den > 1e-6f) {
            off = 0.5f * (cp - cm) / den;
            if (off > 0.5f) off = 0.5f;
            if (off < -0.5f) off = -0.5f;
          }
        } else {
          const float den = 2.f * c0 - cm - cp;
          if (den > 1e-6f) {
            off = 0.5f * (cp - cm) / den;
            if (off > 0.5f) off = 0.5f;
            if (off < -0.5f) off = -0.5f;
          }
        }
      }
    }
    disp[x] = (float)d + off;
  }
  /* residual against the reverse match, :442-451 */
  if (lrc2)
    for (int x = 0; x < W; ++x) {
      lrc2[x] = NAN;
      const float dl = disp[x];
      if (!(dl == dl)) continue;
      const int xr = x - (int)lroundf(dl);
      if (xr >= 0 && xr < W && rev[xr] >= 0) lrc2[x] = fabsf(dl - (float)(dmin + rev[xr]));
    }
  if (best_out) memcpy(best_out, best, sizeof(float) * (size_t)W);
  free(beta); free(rho); free(bstart); free(bitems); free(cursor); free(rev);
  free(best); free(bestj); free(taken); free(order);
}

/* run_dense on the default path (core/tools/de_dense.cpp:738-1608) at one thread:
 * disp/margin f32[WH]; cand6 (may be NULL) = s1,s2,d1,d2,lrc,lrc2 planes with -1e30
 * in missing candidate slots, lrc NaN/-1e30 as the reference writes it. */
/* Row solves and the --out-conf planes from a cost stage's candidates. */
static void finish_dense(const de_cfg* cfg, int W, int H, const float* cs, const int* cd,
                         const int* cn, const int16_t* cnb, const int16_t* rk, float* disp,
                         float* margin, float* cand6) {
  const size_t WH = (size_t)W * H;
  float* lrc2 = malloc(WH * sizeof(float));
  for (int y = 0; y < H; ++y)
    or_solve_row(cfg, W, cs + (size_t)y * W * 2, cd + (size_t)y * W * 2, cn + (size_t)y * W,
                 (cfg->subpixel && cnb) ? cnb + (size_t)y * W * 2 : NULL, disp + (size_t)y * W,
                 margin + (size_t)y * W, lrc2 + (size_t)y * W);
  if (cand6) {
    for (size_t i = 0; i < WH * 6; ++i) cand6[i] = NEG_BIG;
    for (size_t i = 0; i < WH; ++i) {
      if (cn[i] > 0) { cand6[i] = cs[2 * i]; cand6[2 * WH + i] = (float)(cfg->dmin + cd[2 * i]); }
      if (cn[i] > 1) {
        cand6[WH + i] = cs[2 * i + 1];
        cand6[3 * WH + i] = (float)(cfg->dmin + cd[2 * i + 1]);
      }
      cand6[5 * WH + i] = lrc2[i];
    }
    if (rk)
      for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
          const size_t i = (size_t)y * W + x;
          float r = NAN;
          const float dl = disp[i];
          if (isfinite(dl)) {
            const int xr = x - (int)lroundf(dl);
            if (xr >= 0 && xr < W && rk[(size_t)y * W + xr] >= 0)
              r = fabsf(dl - (float)(cfg->dmin + rk[(size_t)y * W + xr]));
          }
          cand6[4 * WH + i] = r;
        }
  }
  free(lrc2);
}

void or_dense(const de_cfg* cfg, const uint8_t* L, const uint8_t* R, int W, int H,
              float* disp, float* margin, float* cand6) {
  const size_t WH = (size_t)W * H;
  float* cs = malloc(WH * 2 * sizeof(float));
  int* cd = malloc(WH * 2 * sizeof(int));
  int* cn = malloc(WH * sizeof(int));
  int16_t* cnb = malloc(WH * 2 * sizeof(int16_t));
  int16_t* rk = cfg->lrc ? malloc(WH * sizeof(int16_t)) : NULL;
  or_cost_top2(cfg, L, R, W, H, cs, cd, cn, cnb, rk);
  finish_dense(cfg, W, H, cs, cd, cn, cnb, rk, disp, margin, cand6);
  free(cs); free(cd); free(cn); free(cnb); free(rk);
}

/* ---- the disparity prior as a per-plane mask (--prior) ------------------------ */

/* The recursive filter over a sub-rectangle, rows [y0, y1), columns [x0, x1):
 * core/tools/de_dense.cpp:438-483.  The chains start at the rectangle's edges. */
void or_filter_i16_rect(int16_t* C, const uint16_t* ax, const uint16_t* ay, int W, int y0,
                        int y1, int x0, int x1) {
  if (y1 - y0 < 1 || x1 - x0 < 2) return;
  for (int y = y0; y < y1; ++y) {
    int16_t* row = C + (size_t)y * W;
    const uint16_t* a = ax + (size_t)y * W;
    int32_t f = row[x0];
    for (int x = x0 + 1; x < x1; ++x) {
      const int32_t c = row[x];
      f = c + (((int32_t)a[x] * (f - c) + (1 << 14)) >> 15);
      row[x] = (int16_t)f;
    }
    f = row[x1 - 1];
    for (int x = x1 - 2; x >= x0; --x) {
      const int32_t c = row[x];
      f = c + (((int32_t)a[x + 1] * (f - c) + (1 << 14)) >> 15);
      row[x] = (int16_t)f;
    }
  }
  for (int y = y0 + 1; y < y1; ++y) {
    int16_t* cur = C + (size_t)y * W;
    const int16_t* prv = C + (size_t)(y - 1) * W;
    const uint16_t* a = ay + (size_t)y * W;
    for (int x = x0; x < x1; ++x) {
      const int32_t c = cur[x];
      cur[x] = (int16_t)(c + (((int32_t)a[x] * (prv[x] - c) + (1 << 14)) >> 15));
    }
  }
  for (int y = y1 - 2; y >= y0; --y) {
    int16_t* cur = C + (size_t)y * W;
    const int16_t* nxt = C + (size_t)(y + 1) * W;
    const uint16_t* a = ay + (size_t)(y + 1) * W;
    for (int x = x0; x < x1; ++x) {
      const int32_t c = cur[x];
      cur[x] = (int16_t)(c + (((int32_t)a[x] * (nxt[x] - c) + (1 << 14)) >> 15));
    }
  }
}

/* The mask of core/tools/de_dense.cpp:797-853: per row y and plane k the interval
 * [mx0, mx1] of pixels whose band [round(prior) - band, round(prior) + band] (clamped
 * to [dmin, dmax]) contains the plane, and per plane the bounding box of those. */
void or_prior_mask(const de_cfg* cfg, const float* prior, int band, int W, int H,
                   int16_t* mx0, int16_t* mx1, int* pylo, int* pyhi, int* pxlo, int* pxhi) {
  const int D = cfg->dmax - cfg->dmin + 1;
  for (size_t i = 0; i < (size_t)H * D; ++i) { mx0[i] = (int16_t)W; mx1[i] = -1; }
  for (int k = 0; k < D; ++k) { pylo[k] = H; pyhi[k] = -1; pxlo[k] = W; pxhi[k] = -1; }
  for (int y = 0; y < H; ++y) {
    int16_t* r0 = mx0 + (size_t)y * D;
    int16_t* r1 = mx1 + (size_t)y * D;
    for (int x = 0; x < W; ++x) {
      const int dc = (int)lroundf(prior[(size_t)y * W + x]);
      const int klo = imax(cfg->dmin, dc - band) - cfg->dmin;
      const int khi = imin(cfg->dmax, dc + band) - cfg->dmin;
      for (int k = klo; k <= khi; ++k) {
        if (x < r0[k]) r0[k] = (int16_t)x;
        if (x > r1[k]) r1[k] = (int16_t)x;
      }
    }
  }
  for (int y = 0; y < H; ++y)
    for (int k = 0; k < D; ++k) {
      const int a = mx0[(size_t)y * D + k], b = mx1[(size_t)y * D + k];
      if (b < a) continue;
      if (y < pylo[k]) pylo[k] = y;
      if (y > pyhi[k]) pyhi[k] = y;
      if (a < pxlo[k]) pxlo[k] = a;
      if (b > pxhi[k]) pxhi[k] = b;
    }
}

/* Cost stage under the mask: core/tools/de_dense.cpp:1166-1297 with a prior.  A plane
 * no pixel wants is skipped; otherwise its score is filtered over its bounding box
 * padded by 8 (within the valid window) and inserted only inside the row intervals.
 * Sub-pixel neighbours are not captured (the reference turns sub-pixel off here). */
void or_cost_top2_prior(const de_cfg* cfg, const uint8_t* L, const uint8_t* R, int W, int H,
                        const float* prior, int band, float* cs, int* cd, int* cn,
                        int16_t* rbest_k) {
  const size_t WH = (size_t)W * H;
  const int D = cfg->dmax - cfg->dmin + 1;
  const int hw = cfg->census_hw, hh = cfg->census_hh;
  const int MPAD = 8;
  uint64_t* cl = malloc(WH * sizeof(uint64_t));
  uint64_t* cr = malloc(WH * sizeof(uint64_t));
  uint16_t* ax = malloc(WH * sizeof(uint16_t));
  uint16_t* ay = malloc(WH * sizeof(uint16_t));
  int16_t* cur = malloc(WH * sizeof(int16_t));
  int16_t *ts0 = malloc(WH * 2), *ts1 = malloc(WH * 2), *td0 = malloc(WH * 2),
          *td1 = malloc(WH * 2), *trs = malloc(WH * 2);
  int16_t* mx0 = malloc((size_t)H * D * 2);
  int16_t* mx1 = malloc((size_t)H * D * 2);
  int *pylo = malloc(D * sizeof(int)), *pyhi = malloc(D * sizeof(int)),
      *pxlo = malloc(D * sizeof(int)), *pxhi = malloc(D * sizeof(int));
  uint16_t lut[256];
  or_census(L, W, H, hw, hh, cl);
  or_census(R, W, H, hw, hh, cr);
  or_rf_lut(cfg->sigma_s, cfg->sigma_r, lut);
  or_rf_coeffs(L, W, H, lut, ax, ay);
  or_prior_mask(cfg, prior, band, W, H, mx0, mx1, pylo, pyhi, pxlo, pxhi);
  for (size_t i = 0; i < WH; ++i) {
    ts0[i] = ts1[i] = -32768;
    td0[i] = td1[i] = -1;
    trs[i] = -32768;
    if (rbest_k) rbest_k[i] = -1;
  }
  for (int k = 0; k < D; ++k) {
    const int d = cfg->dmin + k;
    if (pyhi[k] < pylo[k]) continue;
    const int rylo = imax(hh, pylo[k] - MPAD), ryhi = imin(H - hh, pyhi[k] + 1 + MPAD);
    const int rxlo = imax(hw + d, pxlo[k] - MPAD), rxhi = imin(W - hw, pxhi[k] + 1 + MPAD);
    if (ryhi - rylo < 1 || rxhi - rxlo < 2) continue;
    or_score_plane(cfg, L, R, cl, cr, W, H, k, cur);
    or_filter_i16_rect(cur, ax, ay, W, rylo, ryhi, rxlo, rxhi);
    for (int y = imax(rylo, pylo[k]); y < imin(ryhi, pyhi[k] + 1); ++y) {
      const int xa = imax(rxlo, mx0[(size_t)y * D + k]);
      const int xb = imin(rxhi, mx1[(size_t)y * D + k] + 1);
      for (int x = xa; x < xb; ++x) {
        const size_t i = (size_t)y * W + x;
        const int16_t v = cur[i];
        if (rbest_k && v > trs[i - d]) { trs[i - d] = v; rbest_k[i - d] = (int16_t)k; }
        if (v <= ts1[i]) continue;
        if (v > ts0[i]) { ts1[i] = ts0[i]; td1[i] = td0[i]; ts0[i] = v; td0[i] = (int16_t)k; }
        else { ts1[i] = v; td1[i] = (int16_t)k; }
      }
    }
  }
  const float q = 1.f / (float)Q14;
  for (size_t i = 0; i < WH; ++i) {
    int n = 0;
    cs[2 * i] = cs[2 * i + 1] = NEG_BIG;
    cd[2 * i] = cd[2 * i + 1] = -1;
    if (td0[i] >= 0) { cs[2 * i] = (float)ts0[i] * q; cd[2 * i] = td0[i]; n = 1; }
    if (td1[i] >= 0) { cs[2 * i + 1] = (float)ts1[i] * q; cd[2 * i + 1] = td1[i]; n = 2; }
    cn[i] = n;
  }
  free(cl); free(cr); free(ax); free(ay); free(cur); free(ts0); free(ts1); free(td0);
  free(td1); free(trs); free(mx0); free(mx1); free(pylo); free(pyhi); free(pxlo); free(pxhi);
}

/* The dense pipeline with a full-resolution prior (run_dense with a prior and
 * cfg.band = band; sub-pixel off, as the tool forces it). */
void or_dense_prior(const de_cfg* cfg_in, const uint8_t* L, const uint8_t* R, int W, int H,
                    const float* prior, int band, float* disp, float* margin, float* cand6) {
  de_cfg cfg = *cfg_in;
  cfg.subpixel = 0;
  const size_t WH = (size_t)W * H;
  float* cs = malloc(WH * 2 * sizeof(float));
  int* cd = malloc(WH * 2 * sizeof(int));
  int* cn = malloc(WH * sizeof(int));
  int16_t* rk = cfg.lrc ? malloc(WH * sizeof(int16_t)) : NULL;
  or_cost_top2_prior(&cfg, L, R, W, H, prior, band, cs, cd, cn, rk);
  finish_dense(&cfg, W, H, cs, cd, cn, NULL, rk, disp, margin, cand6);
  free(cs); free(cd); free(cn); free(rk);
}

/* confidence / confidence_u8, core/include/doubleeye/dense_solve.hpp:158-171. */
float or_confidence(float s1, float s2, float lambda, float lrc, float lrc_tol) {
  if (!(s1 > -1e29f)) return 0.f;
  const float alt = (s2 > -1e29f) ? fmax_ref(s2, lambda) : lambda;
  const float x = logf(fmax_ref((1.f - alt) / fmax_ref(1.f - s1, 1e-6f), 1e-6f));
  const float logit = 0.692684f + 7.936751f * x;
  const float p = 1.f / (1.f + expf(-fmax_ref(-30.f, fmin_ref(30.f, logit))));
  return (lrc > lrc_tol) ? fmin_ref(p, 0.35f) : p;
}

unsigned or_confidence_u8(float s1, float s2, float lambda, float lrc, float lrc_tol) {
  return (unsigned)(uint8_t)lroundf(or_confidence(s1, s2, lambda, lrc, lrc_tol) * 255.f);
}
