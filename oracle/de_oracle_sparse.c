/*
 * ORACLE -- test infrastructure, not product code.  See de_oracle.h.
 *
 * Single-threaded C restatement of the reference's sparse (keypoint) path:
 * census_at, the FAST + Shi-Tomasi detector (core/src/preproc.cpp), the candidate
 * graph and MASDA max-sum matcher (core/src/match.cpp), and the edge-list MASDA of
 * the Python entry points (article/masda_stereo.py), which runs in double precision
 * like NumPy.  Float arithmetic is IEEE single precision without contraction
 * (-ffp-contract=off), as in the reference's x86-64 build.
 *
 * Tie rule.  The reference orders by std::sort / std::partial_sort / NumPy argsort,
 * whose order among exactly equal keys is implementation-defined.  This oracle (and
 * the CUDA path) breaks every such tie by the element's position in the input
 * sequence being sorted, i.e. it behaves like a stable sort.
 */
#include "de_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NEG_BIG (-1e30f)

static inline float fmax_ref(float a, float b) { return (a < b) ? b : a; } /* std::max */
static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* census_at: core/src/preproc.cpp:142-162. */
uint64_t or_census_at(const uint8_t* img, int W, int H, int x, int y, int hw, int hh,
                      int* ok) {
  const int inside = x >= hw && y >= hh && x < W - hw && y < H - hh;
  if (ok) *ok = inside;
  if (!inside || (2 * hw + 1) * (2 * hh + 1) - 1 > 64) return 0ull;
  const uint8_t c = img[(size_t)y * W + x];
  uint64_t v = 0;
  int b = 0;
  for (int dy = -hh; dy <= hh; ++dy)
    for (int dx = -hw; dx <= hw; ++dx) {
      if (dx == 0 && dy == 0) continue;
      if (img[(size_t)(y + dy) * W + x + dx] < c) v |= 1ull << b;
      ++b;
    }
  return v;
}

/* FAST-9 ring, radius-3 Bresenham circle from the top, clockwise:
 * core/src/preproc.cpp:356-357. */
static const int kRingX[16] = {0, 1, 2, 3, 3, 3, 2, 1, 0, -1, -2, -3, -3, -3, -2, -1};
static const int kRingY[16] = {-3, -3, -2, -1, 0, 1, 2, 3, 3, 3, 2, 1, 0, -1, -2, -3};

static int ring_run9(unsigned mask) { /* a circular run of >= 9 set bits in 16 */
  const unsigned twice = mask | (mask << 16);
  for (int i = 0; i < 16; ++i)
    if (((twice >> i) & 0x1FFu) == 0x1FFu) return 1;
  return 0;
}

/* is_fast_corner: core/src/preproc.cpp:373-400 (two-of-four compass pre-test,
 * then a 9-run of brighter or of darker ring pixels). */
int or_is_fast_corner(const uint8_t* img, int W, int H, int x, int y, int thr) {
  if (x < 3 || y < 3 || x >= W - 3 || y >= H - 3) return 0;
  const int c = img[(size_t)y * W + x];
  const int hi = c + thr, lo = c - thr;
  int bright = 0, dark = 0;
  for (int k = 0; k < 16; k += 4) {
    const int v = img[(size_t)(y + kRingY[k]) * W + x + kRingX[k]];
    if (v > hi) ++bright;
    else if (v < lo) ++dark;
  }
  if (bright < 2 && dark < 2) return 0;
  unsigned bm = 0, dm = 0;
  for (int k = 0; k < 16; ++k) {
    const int v = img[(size_t)(y + kRingY[k]) * W + x + kRingX[k]];
    if (v > hi) bm |= 1u << k;
    else if (v < lo) dm |= 1u << k;
  }
  return ring_run9(bm) || ring_run9(dm);
}

/* shi_tomasi_at: core/src/preproc.cpp:402-432.  Sobel/8 gradients over a
 * (2r+1)^2 box, structure tensor mean, smaller eigenvalue. */
float or_shi_tomasi_at(const uint8_t* img, int W, int H, int x, int y, int gw) {
  const int r = imax(1, gw / 2);
  if (x - r - 1 < 0 || y - r - 1 < 0 || x + r + 1 >= W || y + r + 1 >= H) return 0.f;
  float sxx = 0.f, syy = 0.f, sxy = 0.f;
  for (int dy = -r; dy <= r; ++dy)
    for (int dx = -r; dx <= r; ++dx) {
      const int px = x + dx, py = y + dy;
      const uint8_t* rm = img + (size_t)(py - 1) * W;
      const uint8_t* r0 = img + (size_t)py * W;
      const uint8_t* rp = img + (size_t)(py + 1) * W;
      const float gx = ((float)rm[px + 1] - (float)rm[px - 1] +
                        2.f * ((float)r0[px + 1] - (float)r0[px - 1]) + (float)rp[px + 1] -
                        (float)rp[px - 1]) * 0.125f;
      const float gy = ((float)rp[px - 1] - (float)rm[px - 1] +
                        2.f * ((float)rp[px] - (float)rm[px]) + (float)rp[px + 1] -
                        (float)rm[px + 1]) * 0.125f;
      sxx += gx * gx;
      syy += gy * gy;
      sxy += gx * gy;
    }
  const float n = 1.f / (float)((2 * r + 1) * (2 * r + 1));
  const float a = sxx * n, b = syy * n, c = sxy * n;
  const float half_tr = 0.5f * (a + b);
  const float disc = sqrtf(fmax_ref(0.f, 0.25f * (a - b) * (a - b) + c * c));
  return half_tr - disc;
}

/* local_std_at: core/src/preproc.cpp:164-182 (double sums, clamped window). */
float or_local_std_at(const uint8_t* img, int W, int H, int x, int y, int window) {
  if (W <= 0 || H <= 0 || window < 2) return 0.f;
  const int r = window / 2;
  const int x0 = imax(0, x - r), x1 = imin(W - 1, x + r);
  const int y0 = imax(0, y - r), y1 = imin(H - 1, y + r);
  double s1 = 0.0, s2 = 0.0;
  for (int yy = y0; yy <= y1; ++yy)
    for (int xx = x0; xx <= x1; ++xx) {
      const double v = img[(size_t)yy * W + xx];
      s1 += v;
      s2 += v * v;
    }
  const double n = (double)((y1 - y0 + 1) * (x1 - x0 + 1));
  const double mean = s1 / n;
  const double var = s2 / n - mean * mean;
  return var > 0.0 ? (float)sqrt(var) : 0.f;
}

typedef struct { float x, y, response; int xi, yi; } cand_t;

static int cand_cmp(const void* a, const void* b) { /* response desc, then scan order */
  const cand_t* p = (const cand_t*)a;
  const cand_t* q = (const cand_t*)b;
  if (p->response != q->response) return (p->response > q->response) ? -1 : 1;
  if (p->yi != q->yi) return p->yi < q->yi ? -1 : 1;
  return p->xi < q->xi ? -1 : (p->xi > q->xi);
}

/* detect_keypoints_fast: core/src/preproc.cpp:442-545.
 * 1. FAST over [border, W-border) x [border, H-border), border >= 5, Shi-Tomasi
 *    response at each corner, drop response < min_response.
 * 2. Strongest first (ties: scan order), keep a candidate unless a kept one lies in
 *    its (2r+1)^2 square.
 * 3. Per kept point: local_std over 7x7 >= min_local_std, parabola sub-pixel on the
 *    response (offsets within +-0.5 only), bucket by its integer pixel into
 *    cell x cell squares.  Output: cells in row-major order, each cell's first
 *    per_cell points in strength order. */
int or_detect_fast(const uint8_t* img, int W, int H, const de_det_cfg* c, de_keypoint* out,
                   int cap) {
  if (W <= 0 || H <= 0) return 0;
  const int border = imax(c->border, 5);
  size_t ncand = 0, capc = 1024;
  cand_t* cand = (cand_t*)malloc(capc * sizeof(cand_t));
  for (int y = border; y < H - border; ++y)
    for (int x = border; x < W - border; ++x) {
      if (!or_is_fast_corner(img, W, H, x, y, c->fast_threshold)) continue;
      const float r = or_shi_tomasi_at(img, W, H, x, y, c->grad_window);
      if (r < c->min_response) continue;
      if (ncand == capc) {
        capc *= 2;
        cand = (cand_t*)realloc(cand, capc * sizeof(cand_t));
      }
      cand[ncand++] = (cand_t){(float)x, (float)y, r, x, y};
    }
  if (ncand == 0) {
    free(cand);
    return 0;
  }
  qsort(cand, ncand, sizeof(cand_t), cand_cmp);
  const int rad = imax(1, c->nms_radius);
  uint8_t* taken = (uint8_t*)calloc((size_t)W * H, 1);
  const int cell = imax(4, c->cell);
  const int cols = (W + cell - 1) / cell, rows = (H + cell - 1) / cell;
  const int keep = imax(1, c->per_cell);
  int* cnt = (int*)calloc((size_t)cols * rows, sizeof(int));
  de_keypoint* slot = (de_keypoint*)malloc((size_t)cols * rows * keep * sizeof(de_keypoint));
  for (size_t k = 0; k < ncand; ++k) {
    const int xi = cand[k].xi, yi = cand[k].yi;
    int blocked = 0;
    for (int dy = -rad; dy <= rad && !blocked; ++dy) {
      const int py = yi + dy;
      if (py < 0 || py >= H) continue;
      for (int dx = -rad; dx <= rad; ++dx) {
        const int px = xi + dx;
        if (px < 0 || px >= W) continue;
        if (taken[(size_t)py * W + px]) { blocked = 1; break; }
      }
    }
    if (blocked) continue;
    taken[(size_t)yi * W + xi] = 1;
    de_keypoint kp = {cand[k].x, cand[k].y, cand[k].response, 0.f};
    kp.local_std = or_local_std_at(img, W, H, xi, yi, 7);
    if (kp.local_std < c->min_local_std) continue;
    if (c->subpixel) {
      const float cc = kp.response;
      const float l = or_shi_tomasi_at(img, W, H, xi - 1, yi, c->grad_window);
      const float r = or_shi_tomasi_at(img, W, H, xi + 1, yi, c->grad_window);
      const float dxx = l - 2.f * cc + r;
      if (fabsf(dxx) > 1e-12f) {
        const float d = 0.5f * (l - r) / dxx;
        if (fabsf(d) <= 0.5f) kp.x += d;
      }
      const float u = or_shi_tomasi_at(img, W, H, xi, yi - 1, c->grad_window);
      const float dn = or_shi_tomasi_at(img, W, H, xi, yi + 1, c->grad_window);
      const float dyy = u - 2.f * cc + dn;
      if (fabsf(dyy) > 1e-12f) {
        const float d = 0.5f * (u - dn) / dyy;
        if (fabsf(d) <= 0.5f) kp.y += d;
      }
    }
    const int b = (yi / cell) * cols + xi / cell;
    if (cnt[b] < keep) slot[(size_t)b * keep + cnt[b]] = kp;
    ++cnt[b];
  }
  int n = 0;
  for (int b = 0; b < cols * rows; ++b)
    for (int k = 0; k < imin(cnt[b], keep); ++k) {
      if (n < cap) out[n] = slot[(size_t)b * keep + k];
      ++n;
    }
  free(cand);
  free(taken);
  free(cnt);
  free(slot);
  return n;
}

/* ---- keypoint MASDA (core/src/match.cpp) ------------------------------------- */

typedef struct { int i, j; float s, beta, rho; } edge_t;

/* pair_score without priors: core/src/match.cpp:298-332. */
float or_pair_score(const de_keypoint* l, const de_keypoint* r, uint64_t dl, uint64_t dr,
                    const de_match_cfg* c) {
  const float half = 0.5f * (float)c->census_bits;
  const float desc = (half - (float)__builtin_popcountll(dl ^ dr)) / half;
  const float dy = (l->y - r->y) / (c->sigma_y > 0 ? c->sigma_y : 1.f);
  return desc - c->w_y * dy * dy;
}

static const de_keypoint* g_right; /* qsort context (single-threaded oracle) */

static int yorder_cmp(const void* a, const void* b) {
  const int p = *(const int*)a, q = *(const int*)b;
  if (g_right[p].y != g_right[q].y) return g_right[p].y < g_right[q].y ? -1 : 1;
  return p < q ? -1 : (p > q);
}

typedef struct { float s; int j, pos; } scr_t;

static int scr_cmp(const void* a, const void* b) { /* score desc, then position */
  const scr_t* p = (const scr_t*)a;
  const scr_t* q = (const scr_t*)b;
  if (p->s != q->s) return p->s > q->s ? -1 : 1;
  return p->pos < q->pos ? -1 : (p->pos > q->pos);
}

/* build_candidates: core/src/match.cpp:46-102.  Right points in y order; per left
 * point the band [y - max_dy, y + max_dy], disparities within
 * [min_disparity, max_disparity]; more than max_candidates are cut to the best by
 * score, kept in score order, otherwise kept in band order. */
static edge_t* build_edges(const de_keypoint* kl, const uint64_t* dl, int nl,
                           const de_keypoint* kr, const uint64_t* dr, int nr,
                           const de_match_cfg* c, int* n_edges) {
  int* order = (int*)malloc(sizeof(int) * (size_t)(nr > 0 ? nr : 1));
  for (int j = 0; j < nr; ++j) order[j] = j;
  g_right = kr;
  qsort(order, (size_t)nr, sizeof(int), yorder_cmp);
  const int maxc = imax(1, c->max_candidates);
  edge_t* e = (edge_t*)malloc(sizeof(edge_t) * ((size_t)nl * maxc + 1));
  scr_t* scr = (scr_t*)malloc(sizeof(scr_t) * (size_t)(nr > 0 ? nr : 1));
  int ne = 0;
  for (int i = 0; i < nl; ++i) {
    const float ylo = kl[i].y - c->max_dy, yhi = kl[i].y + c->max_dy;
    int lo = 0, hi = nr;
    { /* lower_bound: first with y >= ylo */
      int a = 0, b = nr;
      while (a < b) {
        const int m = (a + b) / 2;
        if (kr[order[m]].y < ylo) a = m + 1; else b = m;
      }
      lo = a;
    }
    { /* upper_bound: first with y > yhi */
      int a = lo, b = nr;
      while (a < b) {
        const int m = (a + b) / 2;
        if (!(yhi < kr[order[m]].y)) a = m + 1; else b = m;
      }
      hi = a;
    }
    int ns = 0;
    for (int p = lo; p < hi; ++p) {
      const int j = order[p];
      const float d = kl[i].x - kr[j].x;
      if (d < c->min_disparity || d > c->max_disparity) continue;
      scr[ns].s = or_pair_score(&kl[i], &kr[j], dl[i], dr[j], c);
      scr[ns].j = j;
      scr[ns].pos = ns;
      ++ns;
    }
    if (ns == 0) continue;
    const int keep = imin(ns, maxc);
    if (ns > keep) qsort(scr, (size_t)ns, sizeof(scr_t), scr_cmp);
    for (int k = 0; k < keep; ++k) e[ne++] = (edge_t){i, scr[k].j, scr[k].s, 0.f, 0.f};
  }
  free(order);
  free(scr);
  *n_edges = ne;
  return e;
}

typedef struct { float best, second; int idx; } top2_t;
static inline void t2_push(top2_t* t, float v, int idx) { /* match.cpp:26-44 */
  if (v > t->best) {
    t->second = t->best;
    t->best = v;
    t->idx = idx;
  } else if (v > t->second) {
    t->second = v;
  }
}

static const float* g_belief;
static const edge_t* g_edges;
static int rest_cmp(const void* a, const void* b) { /* belief desc, s desc, index */
  const int p = *(const int*)a, q = *(const int*)b;
  if (g_belief[p] != g_belief[q]) return g_belief[p] > g_belief[q] ? -1 : 1;
  if (g_edges[p].s != g_edges[q].s) return g_edges[p].s > g_edges[q].s ? -1 : 1;
  return p < q ? -1 : (p > q);
}

/* match_masda: core/src/match.cpp:334-417 (message passing), emit :134-231,
 * row_margins :112-132.  Returns the match count; writes at most cap. */
int or_match_masda(const de_keypoint* kl, const uint64_t* dl, int nl, const de_keypoint* kr,
                   const uint64_t* dr, int nr, const de_match_cfg* c, de_match* out, int cap,
                   de_match_stats* st) {
  int ne = 0;
  edge_t* E = build_edges(kl, dl, nl, kr, dr, nr, c, &ne);
  if (st) {
    st->left = nl;
    st->right = nr;
    st->candidates = ne;
    st->iterations_run = 0;
    st->converged = 0;
    st->final_max_delta = 0.f;
    st->oscillating = 0;
  }
  if (ne == 0) {
    free(E);
    return 0;
  }
  /* column lists in edge order (CSR by j) */
  int* cstart = (int*)calloc((size_t)nr + 1, sizeof(int));
  int* citems = (int*)malloc(sizeof(int) * (size_t)ne);
  for (int e = 0; e < ne; ++e) cstart[E[e].j + 1]++;
  for (int j = 0; j < nr; ++j) cstart[j + 1] += cstart[j];
  {
    int* cur = (int*)malloc(sizeof(int) * (size_t)(nr > 0 ? nr : 1));
    memcpy(cur, cstart, sizeof(int) * (size_t)nr);
    for (int e = 0; e < ne; ++e) citems[cur[E[e].j]++] = e;
    free(cur);
  }
  const float d0 = (c->damping < 0.f) ? 0.f : c->damping; /* std::min(std::max(d, 0), .99) */
  const float d = (0.99f < d0) ? 0.99f : d0;
  float prev = 1e30f;
  for (int it = 0; it < c->iterations; ++it) {
    float md = 0.f;
    for (int a = 0; a < ne;) { /* rows are contiguous runs of the edge list */
      int b = a;
      while (b < ne && E[b].i == E[a].i) ++b;
      top2_t t = {NEG_BIG, NEG_BIG, -1};
      for (int e = a; e < b; ++e) t2_push(&t, E[e].beta, e);
      for (int e = a; e < b; ++e) {
        const float ex = (e == t.idx) ? t.second : t.best;
        const float comp = fmax_ref(c->lambda, ex);
        const float tgt = E[e].s - comp;
        const float up = (1.f - d) * tgt + d * E[e].rho;
        md = fmax_ref(md, fabsf(up - E[e].rho));
        E[e].rho = up;
      }
      a = b;
    }
    for (int j = 0; j < nr; ++j) {
      top2_t t = {NEG_BIG, NEG_BIG, -1};
      for (int q = cstart[j]; q < cstart[j + 1]; ++q) t2_push(&t, E[citems[q]].rho, citems[q]);
      for (int q = cstart[j]; q < cstart[j + 1]; ++q) {
        const int e = citems[q];
        const float ex = (e == t.idx) ? t.second : t.best;
        const float comp = fmax_ref(c->gamma, ex);
        const float tgt = E[e].s - comp;
        const float up = (1.f - d) * tgt + d * E[e].beta;
        md = fmax_ref(md, fabsf(up - E[e].beta));
        E[e].beta = up;
      }
    }
    if (st && md > prev) ++st->oscillating;
    prev = md;
    if (st) {
      st->iterations_run = it + 1;
      st->final_max_delta = md;
    }
    if (md < c->converge_eps) {
      if (st) st->converged = 1;
      break;
    }
  }
  float* belief = (float*)malloc(sizeof(float) * (size_t)ne);
  for (int e = 0; e < ne; ++e) belief[e] = E[e].beta + E[e].rho - E[e].s;

  /* row margins */
  float* margin = (float*)calloc((size_t)(nl > 0 ? nl : 1), sizeof(float));
  {
    float* b1 = (float*)malloc(sizeof(float) * (size_t)(nl > 0 ? nl : 1));
    float* b2 = (float*)malloc(sizeof(float) * (size_t)(nl > 0 ? nl : 1));
    for (int i = 0; i < nl; ++i) b1[i] = b2[i] = NEG_BIG;
    for (int e = 0; e < ne; ++e) {
      const int i = E[e].i;
      if (E[e].s > b1[i]) {
        b2[i] = b1[i];
        b1[i] = E[e].s;
      } else if (E[e].s > b2[i]) {
        b2[i] = E[e].s;
      }
    }
    for (int i = 0; i < nl; ++i) {
      if (b1[i] == NEG_BIG) continue;
      const float alt = (b2[i] == NEG_BIG) ? c->lambda : fmax_ref(b2[i], c->lambda);
      margin[i] = b1[i] - alt;
    }
    free(b1);
    free(b2);
  }
  /* emit: mutual best by belief, then greedy completion */
  int* best_row = (int*)malloc(sizeof(int) * (size_t)(nl > 0 ? nl : 1));
  int* best_col = (int*)malloc(sizeof(int) * (size_t)(nr > 0 ? nr : 1));
  float* bl_row = (float*)malloc(sizeof(float) * (size_t)(nl > 0 ? nl : 1));
  float* bl_col = (float*)malloc(sizeof(float) * (size_t)(nr > 0 ? nr : 1));
  for (int i = 0; i < nl; ++i) { best_row[i] = -1; bl_row[i] = NEG_BIG; }
  for (int j = 0; j < nr; ++j) { best_col[j] = -1; bl_col[j] = NEG_BIG; }
  for (int e = 0; e < ne; ++e) {
    if (E[e].s <= c->lambda) continue;
    const int i = E[e].i, j = E[e].j;
    if (best_row[i] < 0 || belief[e] > bl_row[i]) { best_row[i] = e; bl_row[i] = belief[e]; }
    if (best_col[j] < 0 || belief[e] > bl_col[j]) { best_col[j] = e; bl_col[j] = belief[e]; }
  }
  char* rt = (char*)calloc((size_t)(nl > 0 ? nl : 1), 1);
  char* ct = (char*)calloc((size_t)(nr > 0 ? nr : 1), 1);
  int n = 0;
#define ACCEPT(e_)                                                                      \
  do {                                                                                  \
    const edge_t* x_ = &E[(e_)];                                                        \
    if (n < cap)                                                                        \
      out[n] = (de_match){x_->i, x_->j, x_->s, belief[(e_)], kl[x_->i].x - kr[x_->j].x, \
                          kl[x_->i].y - kr[x_->j].y, margin[x_->i]};                    \
    ++n;                                                                                \
    rt[x_->i] = 1;                                                                      \
    ct[x_->j] = 1;                                                                      \
  } while (0)
  for (int i = 0; i < nl; ++i) {
    const int e = best_row[i];
    if (e < 0 || best_col[E[e].j] != e) continue;
    ACCEPT(e);
  }
  int* rest = (int*)malloc(sizeof(int) * (size_t)ne);
  int nrest = 0;
  for (int e = 0; e < ne; ++e) {
    if (E[e].s <= c->lambda || rt[E[e].i] || ct[E[e].j]) continue;
    rest[nrest++] = e;
  }
  g_belief = belief;
  g_edges = E;
  qsort(rest, (size_t)nrest, sizeof(int), rest_cmp);
  for (int k = 0; k < nrest; ++k) {
    const int e = rest[k];
    if (rt[E[e].i] || ct[E[e].j]) continue;
    ACCEPT(e);
  }
#undef ACCEPT
  free(rest);
  free(rt);
  free(ct);
  free(best_row);
  free(best_col);
  free(bl_row);
  free(bl_col);
  free(margin);
  free(belief);
  free(cstart);
  free(citems);
  free(E);
  return n;
}

/* Candidate edges only (for tests of the graph builder): writes i, j, s in the
 * reference's edge order; returns the count. */
int or_match_edges(const de_keypoint* kl, const uint64_t* dl, int nl, const de_keypoint* kr,
                   const uint64_t* dr, int nr, const de_match_cfg* c, int* ei, int* ej,
                   float* s, int cap) {
  int ne = 0;
  edge_t* E = build_edges(kl, dl, nl, kr, dr, nr, c, &ne);
  for (int e = 0; e < ne && e < cap; ++e) {
    ei[e] = E[e].i;
    ej[e] = E[e].j;
    s[e] = E[e].s;
  }
  free(E);
  return ne;
}

/* ---- edge-list MASDA in double (article/masda_stereo.py:417-492) ------------- */

static const double* g_bel64;
static int bel64_cmp(const void* a, const void* b) { /* argsort(-belief), stable */
  const long p = *(const long*)a, q = *(const long*)b;
  if (g_bel64[p] != g_bel64[q]) return g_bel64[p] > g_bel64[q] ? -1 : 1;
  return p < q ? -1 : (p > q);
}

static inline double dmax_np(double a, double b) { return (a < b) ? b : a; }

/* Per-segment max excluding self (_seg_max_excluding, masda_stereo.py:417-442):
 * the segment max, seen by every element below it and by a maximal element when
 * another element also attains it; otherwise the largest value below the max. */
static void seg_max_excl(const double* v, const int64_t* idx, int64_t E, int64_t n,
                         double* m1, double* m2, int64_t* cnt, double* out) {
  for (int64_t k = 0; k < n; ++k) { m1[k] = -INFINITY; m2[k] = -INFINITY; cnt[k] = 0; }
  for (int64_t e = 0; e < E; ++e) m1[idx[e]] = dmax_np(m1[idx[e]], v[e]);
  for (int64_t e = 0; e < E; ++e) {
    if (v[e] >= m1[idx[e]]) cnt[idx[e]]++;
    else m2[idx[e]] = dmax_np(m2[idx[e]], v[e]);
  }
  for (int64_t e = 0; e < E; ++e) {
    const int64_t k = idx[e];
    const double second = cnt[k] > 1 ? m1[k] : m2[k];
    out[e] = (v[e] >= m1[k]) ? second : m1[k];
  }
}

/* masda_sparse: article/masda_stereo.py:453-492, float64 like NumPy.  assign[i] =
 * matched j or -1; hist gets the per-iteration max change (at most iters values);
 * returns the number of iterations run.  Greedy decision in belief order, ties by
 * edge index (a stable argsort). */
int or_masda_edges(const int64_t* ei, const int64_t* ej, const double* se, int64_t E,
                   int64_t m, int64_t n, double lam, double gam, int iters, double damping,
                   double eps, int64_t* assign, double* hist) {
  double* beta = (double*)calloc((size_t)(E > 0 ? E : 1), sizeof(double));
  double* rho = (double*)calloc((size_t)(E > 0 ? E : 1), sizeof(double));
  double* tmp = (double*)malloc(sizeof(double) * (size_t)(E > 0 ? E : 1));
  double* nr_ = (double*)malloc(sizeof(double) * (size_t)(E > 0 ? E : 1));
  const int64_t big = m > n ? m : n;
  double* m1 = (double*)malloc(sizeof(double) * (size_t)(big > 0 ? big : 1));
  double* m2 = (double*)malloc(sizeof(double) * (size_t)(big > 0 ? big : 1));
  int64_t* cnt = (int64_t*)malloc(sizeof(int64_t) * (size_t)(big > 0 ? big : 1));
  int run = 0;
  for (int it = 0; it < iters && E > 0; ++it) {
    double delta = 0.0;
    seg_max_excl(beta, ei, E, m, m1, m2, cnt, tmp);
    for (int64_t e = 0; e < E; ++e) {
      const double comp = dmax_np(lam, tmp[e]);
      nr_[e] = (1.0 - damping) * (se[e] - comp) + damping * rho[e];
    }
    seg_max_excl(nr_, ej, E, n, m1, m2, cnt, tmp);
    double dr = 0.0, db = 0.0;
    for (int64_t e = 0; e < E; ++e) {
      const double comp = dmax_np(gam, tmp[e]);
      const double nb = (1.0 - damping) * (se[e] - comp) + damping * beta[e];
      dr = dmax_np(dr, fabs(nr_[e] - rho[e]));
      db = dmax_np(db, fabs(nb - beta[e]));
      rho[e] = nr_[e];
      beta[e] = nb;
    }
    delta = dmax_np(dr, db);
    hist[run++] = delta;
    if (delta < eps) break;
  }
  for (int64_t i = 0; i < m; ++i) assign[i] = -1;
  if (E > 0) {
    double* bel = tmp;
    for (int64_t e = 0; e < E; ++e) bel[e] = beta[e] + rho[e] - se[e];
    long* order = (long*)malloc(sizeof(long) * (size_t)E);
    for (int64_t e = 0; e < E; ++e) order[e] = (long)e;
    g_bel64 = bel;
    qsort(order, (size_t)E, sizeof(long), bel64_cmp);
    char* uj = (char*)calloc((size_t)(n > 0 ? n : 1), 1);
    for (int64_t k = 0; k < E; ++k) {
      const long e = order[k];
      if (se[e] <= lam) continue;
      if (assign[ei[e]] >= 0 || uj[ej[e]]) continue;
      assign[ei[e]] = ej[e];
      uj[ej[e]] = 1;
    }
    free(uj);
    free(order);
  }
  free(beta);
  free(rho);
  free(tmp);
  free(nr_);
  free(m1);
  free(m2);
  free(cnt);
  return run;
}
