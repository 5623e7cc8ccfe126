/*
 * ORACLE -- test infrastructure, not product code.
 *
 * A plain-C, single-threaded restatement of the reference algorithm for the
 * stereo hot path (mayio/doubleeye core/tools/de_dense.cpp,
 * core/include/doubleeye/dense_solve.hpp, core/src/preproc.cpp,
 * core/src/match.cpp).  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg load it, and only as the checker.  Each function cites the
 * reference lines it restates.
 *
 * Pinned: tests/test_oracle_golden.py checks every function below against
 * golden vectors produced by the reference itself (oracle/_ref, built from the
 * reference sources by oracle/Makefile; fixtures made by
 * tests/golden/make_golden.py).
 *
 * Deliberate difference: where the reference orders by std::sort (unstable;
 * libstdc++'s tie order is implementation-defined), this oracle uses a total
 * order with an index tie-break.  Results agree except between exactly tied
 * claimants.
 */
#ifndef DE_ORACLE_H
#define DE_ORACLE_H

#include <stdint.h>
#include "doubleeye_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

void or_census(const uint8_t* img, int W, int H, int hw, int hh, uint64_t* out);
void or_rf_lut(float sigma_s, float sigma_r, uint16_t lut[256]);
void or_rf_coeffs(const uint8_t* L, int W, int H, const uint16_t lut[256], uint16_t* ax,
                  uint16_t* ay);
int or_score_tables(const de_cfg* cfg, int16_t tbl[65], int16_t adt[256]);
void or_filter_i16(int16_t* plane, const uint16_t* ax, const uint16_t* ay, int W, int H);
void or_filter_f64(double* plane, const uint16_t* ax, const uint16_t* ay, int W, int H);
void or_score_plane(const de_cfg* cfg, const uint8_t* L, const uint8_t* R,
                    const uint64_t* cl, const uint64_t* cr, int W, int H, int k,
                    int16_t* plane);
void or_cost_top2(const de_cfg* cfg, const uint8_t* L, const uint8_t* R, int W, int H,
                  float* cs, int* cd, int* cn, int16_t* cnb, int16_t* rbest_k);
void or_solve_row(const de_cfg* cfg, int W, const float* cs, const int* cd, const int* cn,
                  const int16_t* cnb, float* disp, float* margin, float* lrc2);
void or_solve_row_debug(const de_cfg* cfg, int W, const float* cs, const int* cd,
                        const int* cn, const int16_t* cnb, float* disp, float* margin,
                        float* lrc2, float* best_out, int* target_out);
void or_dense(const de_cfg* cfg, const uint8_t* L, const uint8_t* R, int W, int H,
              float* disp, float* margin, float* cand6);
void or_filter_i16_rect(int16_t* C, const uint16_t* ax, const uint16_t* ay, int W, int y0,
                        int y1, int x0, int x1);
void or_prior_mask(const de_cfg* cfg, const float* prior, int band, int W, int H,
                   int16_t* mx0, int16_t* mx1, int* pylo, int* pyhi, int* pxlo, int* pxhi);
void or_cost_top2_prior(const de_cfg* cfg, const uint8_t* L, const uint8_t* R, int W, int H,
                        const float* prior, int band, float* cs, int* cd, int* cn,
                        int16_t* rbest_k);
void or_dense_prior(const de_cfg* cfg, const uint8_t* L, const uint8_t* R, int W, int H,
                    const float* prior, int band, float* disp, float* margin, float* cand6);
float or_confidence(float s1, float s2, float lambda, float lrc, float lrc_tol);

/* double precision (de_oracle_f64.c), for the error statement against exact arithmetic */
void or_cost_top2_f64(const de_cfg* cfg, const uint8_t* L, const uint8_t* R, int W, int H,
                      double* cs, int* cd, int* cn, double* nb);
void or_solve_row_f64(const de_cfg* cfg, int W, const double* cs, const int* cd,
                      const int* cn, const double* nb, double* disp, double* best_out);
void or_dense_f64(const de_cfg* cfg, const uint8_t* L, const uint8_t* R, int W, int H,
                  double* disp, double* best);
unsigned or_confidence_u8(float s1, float s2, float lambda, float lrc, float lrc_tol);

/* sparse path (de_oracle_sparse.c) */
uint64_t or_census_at(const uint8_t* img, int W, int H, int x, int y, int hw, int hh,
                      int* ok);
int or_is_fast_corner(const uint8_t* img, int W, int H, int x, int y, int thr);
float or_shi_tomasi_at(const uint8_t* img, int W, int H, int x, int y, int gw);
float or_local_std_at(const uint8_t* img, int W, int H, int x, int y, int window);
int or_detect_fast(const uint8_t* img, int W, int H, const de_det_cfg* c, de_keypoint* out,
                   int cap);
float or_pair_score(const de_keypoint* l, const de_keypoint* r, uint64_t dl, uint64_t dr,
                    const de_match_cfg* c);
int or_match_masda(const de_keypoint* kl, const uint64_t* dl, int nl, const de_keypoint* kr,
                   const uint64_t* dr, int nr, const de_match_cfg* c, de_match* out, int cap,
                   de_match_stats* st);
int or_match_edges(const de_keypoint* kl, const uint64_t* dl, int nl, const de_keypoint* kr,
                   const uint64_t* dr, int nr, const de_match_cfg* c, int* ei, int* ej,
                   float* s, int cap);
int or_masda_edges(const int64_t* ei, const int64_t* ej, const double* se, int64_t E,
                   int64_t m, int64_t n, double lam, double gam, int iters, double damping,
                   double eps, int64_t* assign, double* hist);

#ifdef __cplusplus
}
#endif
#endif
