/*
 * doubleeye_b200 -- C ABI of the B200 (sm_100a) stereo hot path:
 * Census -> graded Census/AD cost -> 4-pass recursive edge-aware filter ->
 * per-pixel top-2 -> MASDA row solve (dense), and keypoint MASDA (sparse).
 *
 * Conventions (every entry point):
 *   - returns an int status: DE_OK (0) or a negative DE_ERR_*; never exits;
 *     de_last_error() gives a one-line reason for the calling thread.
 *   - buffers are caller-owned.  Functions named *_dev take DEVICE pointers and
 *     enqueue on the given cudaStream_t (passed as void*, NULL = legacy default
 *     stream) without allocating; their scratch is a caller-provided workspace
 *     sized by the matching *_workspace_bytes() call.  Functions on a de_ctx take
 *     HOST pointers, copy through pinned staging, and block until done.
 *   - a de_ctx is safe to use from one thread at a time; distinct contexts are
 *     independent (one CUDA stream each).
 *   - only plain C types cross the boundary; no torch or CUDA types appear here.
 *
 * Reference interfaces replaced (paths within mayio/doubleeye):
 *   core/include/doubleeye/dense_solve.hpp:19-97     Cfg            -> de_cfg
 *   core/tools/de_dense.cpp:94-129,186-227           census_image   -> de_census_dev
 *   core/tools/de_dense.cpp:531-561                  rf_coeffs      -> de_census_dev (ax/ay)
 *   core/tools/de_dense.cpp:1198-1297                score/filter/top-2 -> de_cost_top2_dev
 *   core/tools/de_dense_cuda.cu:159-392              k_score_hfwd..k_vert_bwd_top2 -> de_cost_top2_dev
 *   core/include/doubleeye/dense_solve.hpp:213-452   solve_row_sparse -> de_solve_dev
 *   core/tools/de_dense.cpp:738-1608                 run_dense      -> de_dense_dev / de_ctx_dense
 *   core/include/doubleeye/dense_solve.hpp:158-171   confidence(_u8) -> de_confidence
 *   core/include/doubleeye/preproc.hpp:96-97         census_at      -> de_census_at_dev
 *   core/include/doubleeye/preproc.hpp:202-204       detect_keypoints_fast -> de_detect_fast_dev
 *   core/include/doubleeye/match.hpp:221-226         match_masda    -> de_match_masda_dev
 *   article/masda_stereo.py:392-492                  masda_sparse/decide -> de_masda_edges_dev,
 *                                                    de_masda_decide_dev
 *   article/dense_masda.py:39-79                     dense_problem  -> de_dense_problem_dev
 */
#ifndef DOUBLEEYE_B200_H
#define DOUBLEEYE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DE_API __attribute__((visibility("default")))

enum {
  DE_OK = 0,
  DE_ERR_ARG = -1,         /* bad argument or size beyond a documented limit */
  DE_ERR_CUDA = -2,        /* a CUDA runtime call failed */
  DE_ERR_OOM = -3,         /* device or pinned allocation failed */
  DE_ERR_TIMEOUT = -4,     /* a bounded device wait ran out */
  DE_ERR_UNSUPPORTED = -5, /* configuration outside this build's arithmetic */
  DE_ERR_BUSY = -6,        /* admission refused: HBM budget or queue full */
  DE_ERR_CLOSED = -7       /* the server was stopped */
};

/* Dense matcher configuration.  Field meaning and defaults follow
 * core/include/doubleeye/dense_solve.hpp:19-97 (Cfg) for the fields this path
 * reads; de_cfg_default() writes those defaults. */
typedef struct de_cfg {
  int dmin, dmax;          /* disparities searched, dmin..dmax (default 1..60) */
  int iters;               /* MASDA message-passing iterations (default 0 = WTA) */
  float sigma_s, sigma_r;  /* recursive-filter reach and edge sensitivity (8, 0.2) */
  float ad;                /* weight of the truncated absolute difference (0.15) */
  int ad_trunc;            /* AD saturation, 8-bit levels (10) */
  float lambda, gamma;     /* clutter / misdetection costs (-0.1, -0.1) */
  float damping;           /* message damping (0.4) */
  float min_margin;        /* best-minus-second gate, 0 = off */
  float min_ratio;         /* peak-ratio gate, 0 = off */
  int subpixel;            /* sub-pixel fit on (1) */
  int fit_eq;              /* equiangular fit (1) or parabola (0) */
  int lrc;                 /* exact reverse match over every disparity (0) */
  int census_hw, census_hh;/* census half-window; 3,3 (7x7) is the reference's */
} de_cfg;

DE_API void de_cfg_default(de_cfg* cfg);

/* Limits of this build: D = dmax - dmin + 1 <= 256 (8-bit k in the packed top-2
 * key), 8 <= W <= 8192, 8 <= H <= 8192, dmin >= 1. */
#define DE_MAX_D 256
#define DE_MAX_DIM 8192

DE_API const char* de_last_error(void);
DE_API const char* de_version(void);

/* ---- dense, device pointers, caller workspace, asynchronous ------------------ */

/* One stereo pair.  L/R are W*H u8 rows of pitch W (device).  Outputs (device,
 * W*H each, any may be NULL): disp f32 (NaN = declined), margin f32, conf u8
 * (confidence_u8, 0 where declined), cand f32 planes in the reference's
 * --out-conf order s1,s2,d1,d2,lrc,lrc2 (6*W*H).  dmax 0 = the cfg's. */
typedef struct de_pair {
  const uint8_t* L;
  const uint8_t* R;
  int W, H, dmax;
  float* disp;
  float* margin;
  uint8_t* conf;
  float* cand;
} de_pair;

/* Workspace for de_dense_dev on n pairs (sum over pairs, 256-byte aligned, plus a
 * 256-byte status head). */
DE_API int de_dense_workspace_bytes(const de_cfg* cfg, const de_pair* pairs, int n,
                                    size_t* bytes);
/* Census -> cost -> filter -> top-2 -> row solve for n pairs in one set of
 * launches (pairs may differ in W, H and dmax).  Replaces run_dense
 * (core/tools/de_dense.cpp:738) and the de_dense_cuda pipeline
 * (core/tools/de_dense_cuda.cu:556-663). */
DE_API int de_dense_dev(const de_cfg* cfg, const de_pair* pairs, int n,
                        void* workspace, size_t ws_bytes, void* stream);

/* The same dense pipeline for one pair with NO allocation anywhere: for callers
 * that cannot call cudaMalloc (real-time threads that may not take the driver's
 * allocation locks, hosts that own the device heap, integrations whose memory budget
 * is fixed up front).  No counterpart in the reference.  The workspace is a 16 MiB
 * file-scope device array that every GPU loading this library holds until exit; a
 * pair whose de_dense_workspace_bytes exceeds it is refused with DE_ERR_ARG (the
 * default 7x7 census fits 320x240 at D <= 64).  The first call on a device resolves
 * the array's device address with that device current and keeps it, so a device
 * reset while the library is loaded is not supported.  Calls share the array and
 * each leaves its contents behind: calls whose work overlaps on the GPU (concurrent
 * streams) race and must be serialised by the caller.  The status of the last call
 * is read with de_workspace_status(NULL, stream, &status). */
DE_API int de_dense_noalloc_dev(const de_cfg* cfg, const de_pair* pair, void* stream);

/* Status of the last launch set that used this workspace: waits for the stream,
 * then writes 0, or non-zero if a bounded device wait ran out (the results of that
 * launch set are then invalid).  The host-pointer context checks it itself.
 * workspace NULL reads the status of the last de_dense_noalloc_dev call on the
 * current device. */
DE_API int de_workspace_status(const void* workspace, void* stream, int* status);

/* Stage entry points, for stage-level parity and for callers that keep their
 * own pipeline.  Census planes: cl/cr u64 (0 on the border), ax/ay u16 Q15
 * filter coefficients of the LEFT image (core/tools/de_dense.cpp:531-561). */
DE_API int de_census_dev(const de_cfg* cfg, const uint8_t* L, const uint8_t* R, int W,
                         int H, uint64_t* cl, uint64_t* cr, uint16_t* ax, uint16_t* ay,
                         void* stream);
/* Candidates in the reference layout (core/tools/de_dense_cuda.cu:286-392):
 * cs f32[2WH] (Q14/16384), cd i32[2WH] (k = d - dmin), cn i32[WH],
 * cnb i16[2WH] (filtered cost at k*-1, k*+1 in Q14; -32768 = none, may be NULL).
 * cs/cd slots j >= cn are unspecified. */
DE_API size_t de_cost_workspace_bytes(int W, int H, int D);
DE_API int de_cost_top2_dev(const de_cfg* cfg, const uint8_t* L, const uint8_t* R,
                            int W, int H, float* cs, int* cd, int* cn, int16_t* cnb,
                            void* workspace, size_t ws_bytes, void* stream);
/* Row solve over reference-layout candidates (dense_solve.hpp:213-452 with K=2,
 * vol = NULL): disp, margin, lrc2 f32[WH] (lrc2 may be NULL). */
DE_API int de_solve_dev(const de_cfg* cfg, int W, int H, const float* cs, const int* cd,
                        const int* cn, const int16_t* cnb, float* disp, float* margin,
                        float* lrc2, void* stream);

/* Stage timing (a profiling aid; the reference prints the same breakdown from
 * cudaEvents, core/tools/de_dense_cuda.cu:552-604,847-852).  While enabled, every
 * de_dense_dev launch set records events on its stream between census, row, column
 * and solve kernels.  de_stage_times() waits for them, writes the summed ms per
 * stage into ms[0..n) (n <= 4: census, rows, cols, solve), the number of launch
 * sets into *launches, and clears them. */
DE_API int de_stage_timing(int enable);
DE_API int de_stage_times(float* ms, int n, int* launches);

/* Launch-shape knobs (process-wide; results never depend on them, only speed).
 * No counterpart in the reference, whose launch shapes are fixed.
 *   "rows_ctas_per_sm"  cap on row-kernel CTAs resident per SM (default 32, i.e.
 *                       as many as fit): fewer rows in flight keep each row's
 *                       forward pass in L2 for its backward pass
 *   "cols_kt"           disparities per lane in the column kernel: 4, 8, 16, or 0
 *                       to choose by batch size (default 0: 4 for batches too small
 *                       to fill the GPU with columns, else 8)
 *   "cols_pf"           image rows the column kernel's lanes load ahead of use:
 *                       4, 8, 16 (4 disparities per lane only), or 0 to choose by
 *                       shape (default 0: 16 at 4 disparities per lane, else 8; 16
 *                       disparities per lane always use 4)
 *   "cols_cta"          column-kernel threads per CTA: 128, 256, or 0 to choose by
 *                       batch size (default 0: 128 for batches of a few 848x480
 *                       pairs or less, else 256)
 *   "solve_threads"     threads per image row in the row solve: 128, 256, 512, or
 *                       0 to choose by row width (default 0: 512 for rows wider
 *                       than 1024 pixels, else 256)
 *   "cols_async"        1 (default) or 0: at 8 disparities per lane the column
 *                       kernel's 8-row prefetch goes through shared memory by
 *                       asynchronous copies (fewer registers, so more warps and more
 *                       room for a concurrent launch set) instead of a register ring;
 *                       the host context's chunked batches keep the register ring
 *   "batch_streams"     1..4 (default 2): de_dense_dev runs a batch of several
 *                       pairs as that many parts, pairs taken in turn, each part's
 *                       launch set on its own stream forked from and joined back to
 *                       the caller's (also under graph capture), so one part's kernel
 *                       tails overlap the other's work.  The host context's chunked
 *                       batches and the server's lanes, which already overlap, run
 *                       each batch as one launch set; stage timing does too
 * and one test hook that does change results:
 *   "expire_wait_polls" 0 (default) or a poll count: every row-kernel launch then
 *                       ends, after all its real waits have completed, with a
 *                       bounded wait of that many polls on a barrier nothing
 *                       arrives at, so the launch set reports a device wait that ran
 *                       out (DE_ERR_TIMEOUT / a non-zero workspace status) without any
 *                       fault; for testing callers' handling of that status */
DE_API int de_set_param(const char* name, int value);
DE_API int de_get_param(const char* name, int* value);

/* confidence() / confidence_u8() of dense_solve.hpp:158-171, host side. */
DE_API float de_confidence(float s1, float s2, float lambda, float lrc, float lrc_tol);

/* ---- sparse (keypoint) MASDA ------------------------------------------------- */

/* Keypoint of core/include/doubleeye/preproc.hpp:125-130. */
typedef struct de_keypoint { float x, y, response, local_std; } de_keypoint;

/* DetectorConfig of core/include/doubleeye/preproc.hpp:132-145, same defaults. */
typedef struct de_det_cfg {
  int grad_window, cell, per_cell;
  float min_response, min_local_std;
  int border, subpixel, fast_threshold, nms_radius;
} de_det_cfg;
DE_API void de_det_cfg_default(de_det_cfg* cfg);

/* MatchConfig of core/include/doubleeye/match.hpp:135-176 (priors excluded), same
 * defaults.  census_bits is the descriptor length the score is scaled by; the
 * reference hard-codes 48 (core/src/match.cpp:339) and so does the default. */
typedef struct de_match_cfg {
  float max_dy, min_disparity, max_disparity;
  int max_candidates;
  float sigma_y, w_y;
  int iterations;
  float damping, lambda, gamma, converge_eps;
  int census_bits;
} de_match_cfg;
DE_API void de_match_cfg_default(de_match_cfg* cfg);

/* Match / MatchStats of core/include/doubleeye/match.hpp:44-66,178-186. */
typedef struct de_match {
  int left, right;
  float score, belief, disparity, dy, margin;
} de_match;
typedef struct de_match_stats {
  int left, right, candidates, iterations_run, converged;
  float final_max_delta;
  int oscillating;
} de_match_stats;

/* census_at (core/src/preproc.cpp:142-162) at n keypoints, each at
 * (int(x + 0.5), int(y + 0.5)) as core/tools/de_match.cpp:228-232 rounds them.
 * desc[k] = 0 and ok[k] = 0 where the window leaves the image; ok may be NULL.
 * n_dev, if not NULL, is a device count that limits n (a detector's output). */
DE_API int de_census_at_dev(const uint8_t* img, int W, int H, const de_keypoint* kp, int n,
                            const int* n_dev, int hw, int hh, uint64_t* desc, uint8_t* ok,
                            void* stream);

/* detect_keypoints_fast (core/src/preproc.cpp:442-545).  Writes at most cap keypoints
 * to out in the reference's order (grid cells row-major, each cell's strongest
 * per_cell first) and the full count to the device int *n_out (-1 if resolving the
 * strongest-first suppression exceeded its work bound, which takes a monotone
 * response ramp thousands of points long).
 * Images 16..4096 x 16..8192, cell <= 128. */
DE_API int de_detect_workspace_bytes(int W, int H, const de_det_cfg* cfg, size_t* bytes);
DE_API int de_detect_fast_dev(const uint8_t* img, int W, int H, const de_det_cfg* cfg,
                              de_keypoint* out, int cap, int* n_out, void* workspace,
                              size_t bytes, void* stream);

/* The sparse feature set read out of a dense map (core/tools/de_dense_cuda.cu:866-899):
 * for each keypoint, the disparity and margin at (int(x + 0.5), int(y + 0.5)) clamped
 * to the image; keypoints whose disparity is not > 0 are dropped, order kept.
 * Device pointers; n_dev (optional) limits n; margin may be NULL (reads 0). */
typedef struct de_kp_disparity { float x, y, disparity, margin; } de_kp_disparity;
DE_API int de_keypoint_readout_dev(const de_keypoint* kp, int n, const int* n_dev,
                                   const float* disp, const float* margin, int W, int H,
                                   de_kp_disparity* out, int cap, int* n_out, void* stream);

/* match_masda (core/include/doubleeye/match.hpp:221-226, core/src/match.cpp:334-417)
 * on device keypoints and descriptors.  nl/nr are the array sizes; nl_dev/nr_dev,
 * if not NULL, are device counts that limit them (so a detector's output feeds
 * this call without a host round trip).  Matches go to out (at most cap) in the
 * reference's emission order; the count to the device int *n_out; stats (device,
 * may be NULL) as MatchStats.  One CTA solves the problem; nr <= 16384. */
DE_API int de_match_workspace_bytes(int nl, int nr, const de_match_cfg* cfg, size_t* bytes);
DE_API int de_match_masda_dev(const de_keypoint* kl, const uint64_t* dl, int nl,
                              const int* nl_dev, const de_keypoint* kr, const uint64_t* dr,
                              int nr, const int* nr_dev, const de_match_cfg* cfg, de_match* out,
                              int cap, int* n_out, de_match_stats* stats, void* workspace,
                              size_t bytes, void* stream);

/* The soft disparity priors of MatchConfig (core/include/doubleeye/match.hpp:157-163:
 * the coarse DisparityPrior and the per-keypoint SmoothPrior), applied in pair_score
 * (core/src/match.cpp:298-332), resolved by the caller to one (disparity, sigma) per
 * LEFT keypoint: s(i,j) -= w * (((xl - xr) - d[i]) / sd[i])^2 where sd[i] > 0, no
 * term where sd[i] <= 0 (the reference's "no prior here").  Device arrays of nl
 * floats; a NULL sigma array turns that prior off. */
typedef struct de_match_prior {
  const float* coarse_d;
  const float* coarse_sd;
  float w_coarse;
  const float* smooth_d;
  const float* smooth_sd;
  float w_smooth;
} de_match_prior;
/* de_match_masda_dev with soft disparity priors (prior may be NULL). */
DE_API int de_match_masda_prior_dev(const de_keypoint* kl, const uint64_t* dl, int nl,
                                    const int* nl_dev, const de_keypoint* kr,
                                    const uint64_t* dr, int nr, const int* nr_dev,
                                    const de_match_cfg* cfg, const de_match_prior* prior,
                                    de_match* out, int cap, int* n_out, de_match_stats* stats,
                                    void* workspace, size_t bytes, void* stream);

/* ---- the disparity prior as a per-plane mask (--prior) ------------------------
 * core/tools/de_dense.cpp:797-853,438-483,1166-1297 (run_dense with a prior, the
 * --prior path of :1756-1813).  prior: W x H float32 disparities on the device (a
 * previous frame, a coarse pass), no holes; plane d is computed only over the bounding
 * box (padded by 8) of the pixels whose [round(prior) - band, round(prior) + band]
 * contains d, and offered as a candidate only inside those pixels' row intervals.
 * Sub-pixel refinement is off, as the reference's tool sets it.  One pair; 7x7 census. */
DE_API int de_dense_prior_workspace_bytes(const de_cfg* cfg, const de_pair* pair,
                                          size_t* bytes);
DE_API int de_dense_prior_dev(const de_cfg* cfg, const de_pair* pair, const float* prior,
                              int band, void* workspace, size_t bytes, void* stream);

/* Hole filling of a disparity map so it can serve as a prior (a prior with holes is
 * refused): the reference's fill (article/coarse_to_fine.py:58-76), iterated
 * 4-neighbour averaging.  Up to 128 sweeps; in each, every non-finite pixel with a
 * finite 4-neighbour (neighbours wrap around the edges) becomes the float32 mean of
 * those neighbours, summed left, right, up, down; sweeps stop when one changes
 * nothing, and what is left non-finite becomes 0.  src and dst are W x H float32 on
 * the device (src is not modified); workspace >= de_prior_fill_workspace_bytes. */
DE_API size_t de_prior_fill_workspace_bytes(int W, int H);
DE_API int de_prior_fill_dev(const float* src, float* dst, int W, int H, void* workspace,
                             size_t bytes, void* stream);

/* ---- a batch captured as a CUDA graph ---------------------------------------- */
/* Captures de_dense_dev(cfg, pairs, n, workspace) once; each de_graph_launch replays
 * the whole batch (status reset + four kernels) as one launch on the given stream,
 * reading the captured input buffers as they are at replay time.  The buffers and
 * the workspace must outlive the graph.  Knobs set with de_set_param are those in
 * force at capture. */
typedef struct de_graph de_graph;
DE_API int de_graph_create(const de_cfg* cfg, const de_pair* pairs, int n, void* workspace,
                           size_t bytes, de_graph** out);
DE_API int de_graph_launch(de_graph* g, void* stream);
DE_API int de_graph_destroy(de_graph* g);

/* ---- the Python entry points: edge-list MASDA in double precision ------------ */

/* masda_sparse (article/masda_stereo.py:453-492) on device edge lists: ei/ej int64
 * left/right node of each of E edges, se float64 scores; m left and n right nodes.
 * float64 throughout, as NumPy.  assign[m] (device) = matched right node or -1;
 * hist (device, >= iters doubles) gets the per-iteration largest message change and
 * *n_hist (device) their count; belief (device, E doubles, may be NULL) the final
 * beliefs.  Exact belief ties go to the lower edge index.  Blocks the calling
 * thread while the greedy decision runs (it checks the remaining edge count between
 * rounds).  E < 2^31. */
DE_API int de_masda_edges_workspace_bytes(long long E, long long m, long long n,
                                          size_t* bytes);
DE_API int de_masda_edges_dev(const int64_t* ei, const int64_t* ej, const double* se,
                              long long E, long long m, long long n, double lam, double gam,
                              int iters, double damping, double eps, int64_t* assign,
                              double* hist, int* n_hist, double* belief, void* workspace,
                              size_t bytes, void* stream);
/* decide (article/masda_stereo.py:392-414): greedy one-to-one in belief order over
 * edges with finite belief and score > lam.  Same workspace as de_masda_edges_dev. */
DE_API int de_masda_decide_dev(const int64_t* ei, const int64_t* ej, const double* se,
                               const double* belief, long long E, long long m, long long n,
                               double lam, int64_t* assign, void* workspace, size_t bytes,
                               void* stream);
/* _seg_max_excluding (article/masda_stereo.py:417-442); workspace >= 20*n + 1024 bytes. */
DE_API int de_seg_max_excluding_dev(const double* vals, const int64_t* idx, long long E,
                                    long long n, double* out, void* workspace, size_t bytes,
                                    void* stream);
/* hamming (article/masda_stereo.py:290-295): popcount(a ^ b) per element. */
DE_API int de_hamming_dev(const uint64_t* a, const uint64_t* b, long long n, int32_t* out,
                          void* stream);
/* census (article/masda_stereo.py:264-284) at integer points xy[2k], xy[2k+1];
 * 0 (and ok = 0) where the window leaves the image. */
DE_API int de_census_pts_dev(const uint8_t* img, int W, int H, const int32_t* xy, long long n,
                             int hw, int hh, uint64_t* out, uint8_t* ok, void* stream);
/* build_problem (article/masda_stereo.py:305-326): the m x n float32 score matrix,
 * -inf outside the epipolar band / disparity range; pl, pr are (x, y) float32 pairs;
 * bits is the descriptor length the score is scaled by (48 in the reference). */
DE_API int de_build_problem_dev(const float* pl, const uint64_t* dl, long long m,
                                const float* pr, const uint64_t* dr, long long n, float max_dy,
                                float dmin, float dmax, float sigma_y, float w_y, int bits,
                                float* S, void* stream);
/* to_edges (article/masda_stereo.py:445-450): finite entries of S in row-major order;
 * *n_out (device int64) = their count, at most cap written; workspace >= 8*m + 256. */
DE_API int de_edges_from_matrix_dev(const float* S, long long m, long long n, int64_t* ei,
                                    int64_t* ej, double* se, long long cap, int64_t* n_out,
                                    void* workspace, size_t bytes, void* stream);
/* dense_problem (article/dense_masda.py:39-79): every interior pixel against every
 * disparity dmin..dmax (0 <= dmin, at most 512 values) on its row, in the reference's
 * order (disparity, then row, then column); se = (24 - Hamming)/24 as float32.
 * de_dense_problem_edges gives the edge count; workspace >= 16*W*H + 512 bytes. */
DE_API long long de_dense_problem_edges(int W, int H, int dmin, int dmax, int hw, int hh);
DE_API int de_dense_problem_dev(const uint8_t* L, const uint8_t* R, int W, int H, int dmin,
                                int dmax, int hw, int hh, int64_t* ei, int64_t* ej, float* se,
                                long long cap, void* workspace, size_t bytes, void* stream);

/* ---- serving: many camera streams, continuous batching ------------------------
 * Replaces the reference's one-frame-at-a-time live loop
 * (core/tools/de_dense_cuda.cu:670-770).  A server owns a device: any thread submits
 * a pair (host buffers, copied at submit) tagged with its camera stream and gets a
 * ticket; a worker admits waiting pairs first come first served into lanes (a CUDA
 * stream with a device arena of hbm_budget / lanes bytes, allocated once), as many
 * as fit the arena and max_batch, and runs each lane's batch through the dense
 * pipeline while the next lane fills.  Results equal the plain pipeline's bit for
 * bit.  Each camera stream keeps its latest disparity maps on the device. */
typedef struct de_server de_server;
typedef struct de_server_cfg {
  int device;
  size_t hbm_budget;     /* device bytes for all lanes' arenas */
  int max_batch;         /* pairs per launch */
  int lanes;             /* batches in flight (CUDA streams) */
} de_server_cfg;
typedef struct de_server_stats {
  unsigned long long completed, failed, batches;
  double mean_batch;     /* pairs per launch */
  double p50_ms, p99_ms, max_ms;   /* submit-to-result latency of completed requests */
  size_t max_pending;
} de_server_report;
DE_API void de_server_cfg_default(de_server_cfg* cfg);
DE_API int de_server_create(const de_cfg* cfg, const de_server_cfg* scfg, de_server** out);
/* Output planes a request will be asked for (the server copies only these). */
#define DE_PLANE_DISP 1u
#define DE_PLANE_MARGIN 2u
#define DE_PLANE_CONF 4u
#define DE_PLANE_Q4 8u
#define DE_PLANE_QCONF 16u
#define DE_PLANE_ALL 31u
/* dmax 0 = cfg's; planes 0 = all.  Copies L and R, returns at once with a ticket. */
DE_API int de_server_submit(de_server* sv, int stream, const uint8_t* L, const uint8_t* R,
                            int W, int H, int dmax, unsigned planes,
                            unsigned long long* ticket);
/* Blocks up to timeout_ms (DE_ERR_TIMEOUT leaves the request waitable), then copies
 * the outputs (any may be NULL): disp/margin f32, conf u8, and the DEDD planes q4
 * (int16 sixteenths of a pixel, -32768 where declined) and qconf; frees the ticket. */
DE_API int de_server_wait(de_server* sv, unsigned long long ticket, int timeout_ms,
                          float* disp, float* margin, uint8_t* conf, int16_t* q4,
                          uint8_t* qconf, double* latency_ms);
DE_API int de_server_stats(de_server* sv, de_server_report* out);
DE_API int de_server_reset_stats(de_server* sv);
/* Temporal prior for one camera stream (band > 0; 0 turns it off): each of its frames
 * after the first of a size is matched through the prior path (de_dense_prior_dev)
 * with the stream's previous disparity map, hole-filled by de_prior_fill_dev, as the
 * prior; both maps stay on the device.  The frames of such a stream run in submission
 * order, each after the one before it.  Needs the 7x7 census.  Applies to frames
 * admitted after the call. */
DE_API int de_server_stream_prior(de_server* sv, int stream, int band);
/* The newest disparity map a stream has on the device (waits for it), W x H f32. */
DE_API int de_server_last_disparity(de_server* sv, int stream, float* host, int W, int H);
DE_API int de_server_destroy(de_server* sv);
/* DEDD planes from a disparity (and optional confidence) plane on the device:
 * core/tools/de_dense_cuda.cu:729-746. */
DE_API int de_dedd_encode_dev(const float* disp, const uint8_t* conf, int W, int H,
                              int16_t* q4, uint8_t* qconf, void* stream);

/* ---- dense, host pointers, context-owned memory, synchronous ----------------- */
/* A context owns device buffers, a page-locked mirror and its streams; one thread
 * uses it at a time (give each thread its own).  Host buffers may be pageable or
 * page-locked: page-locked ones move by DMA directly, pageable ones through the
 * mirror.  A batch with enough output runs as up to five chunks, each on its own
 * compute stream (priority falling with the chunk's order) and workspace slice,
 * whose uploads and downloads overlap the other chunks' compute; every call has
 * finished its copies when it returns. */

typedef struct de_ctx de_ctx;
DE_API int de_ctx_create(const de_cfg* cfg, int device, de_ctx** out);
DE_API int de_ctx_destroy(de_ctx* ctx);
DE_API int de_ctx_set_cfg(de_ctx* ctx, const de_cfg* cfg);
/* Host-buffer single pair: uploads L/R, runs de_dense_dev, downloads outputs. */
DE_API int de_ctx_dense(de_ctx* ctx, const uint8_t* L, const uint8_t* R, int W, int H,
                        float* disp, float* margin, uint8_t* conf, float* cand);
/* The prior path on host buffers; a prior with non-finite values is refused, as the
 * reference refuses one with holes (core/tools/de_dense.cpp:1798-1805). */
DE_API int de_ctx_dense_prior(de_ctx* ctx, const uint8_t* L, const uint8_t* R, int W, int H,
                              const float* prior, int band, float* disp, float* margin,
                              uint8_t* conf, float* cand);
/* Keypoint read-out on host buffers (the --keypoints output of
 * core/tools/de_dense_cuda.cu:866-899): detect keypoints in L (at most 65536), read
 * the disparity and margin maps at them; *n_detected = keypoints found, *n_out = those
 * with a disparity (at most cap written, in detection order). */
DE_API int de_ctx_keypoints(de_ctx* ctx, const uint8_t* L, int W, int H, const de_det_cfg* det,
                            const float* disp, const float* margin, de_kp_disparity* out,
                            int cap, int* n_out, int* n_detected);
/* The same for n host pairs in one batched launch. */
DE_API int de_ctx_dense_batch(de_ctx* ctx, const de_pair* host_pairs, int n);

/* Host-pointer forms of the stage and sparse entry points, for callers without device
 * memory of their own (the C++ surface in include/doubleeye/ is built on these).
 * Sizes and limits are those of the device forms above.
 *   de_ctx_census:      census_transform (core/src/preproc.cpp:110-138) of one image,
 *                       bits[W*H] (0 outside the (hw, hh) border)
 *   de_ctx_census_at:   census_at at n keypoints (de_census_at_dev)
 *   de_ctx_detect_fast: detect_keypoints_fast, *n = keypoints found (at most cap
 *                       written)
 *   de_ctx_match_masda: match_masda with optional priors (HOST arrays in prior);
 *                       *n_out matches (at most cap written), stats may be NULL
 *   de_ctx_solve:       the row solve over reference-layout candidates (de_solve_dev) */
DE_API int de_ctx_census(de_ctx* ctx, const uint8_t* img, int W, int H, int hw, int hh,
                         uint64_t* bits);
DE_API int de_ctx_census_at(de_ctx* ctx, const uint8_t* img, int W, int H,
                            const de_keypoint* kp, int n, int hw, int hh, uint64_t* desc,
                            uint8_t* ok);
DE_API int de_ctx_detect_fast(de_ctx* ctx, const uint8_t* img, int W, int H,
                              const de_det_cfg* cfg, de_keypoint* out, int cap, int* n);
DE_API int de_ctx_match_masda(de_ctx* ctx, const de_keypoint* kl, const uint64_t* dl, int nl,
                              const de_keypoint* kr, const uint64_t* dr, int nr,
                              const de_match_cfg* cfg, const de_match_prior* prior,
                              de_match* out, int cap, int* n_out, de_match_stats* stats);
DE_API int de_ctx_solve(de_ctx* ctx, const de_cfg* cfg, int W, int H, const float* cs,
                        const int* cd, const int* cn, const int16_t* cnb, float* disp,
                        float* margin, float* lrc2);

#ifdef __cplusplus
}
#endif
#endif /* DOUBLEEYE_B200_H */
