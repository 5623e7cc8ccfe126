// Internal interfaces between the C ABI (de_capi.cu) and the kernels
// (de_dense.cu).  Not installed; include/doubleeye_b200.h is the public surface.
#pragma once

#include <cstddef>
#include <cstdint>

#include <vector>

#include <cuda_runtime.h>

#include "../../include/doubleeye_b200.h"

namespace de {

// Largest batch one launch set carries; the descriptor table travels as a kernel
// parameter (no host-to-device copy, so launches are graph-capturable and need no
// allocation).  Bigger batches are split by the host.
constexpr int kMaxBatch = 64;
constexpr int kMaxW = 4096;    // row kernel keeps two census rows of W in shared memory
constexpr int kMaxH = 8192;

// Per-pair device layout.  Every pointer is device memory.
struct DevPair {
  const uint8_t* L;
  const uint8_t* R;
  uint64_t* cwL;       // census word | pixel << 56 (7x7) or census only (wider windows);
  uint64_t* cwR;       //   element (y, x) at [y*cpitch + lpad + x] (left), [y*cpitch + x]
  uint16_t* ax;        // Q15 filter coefficients of L, x direction, [y*apitch + lpad + x]
  uint16_t* ay;        // ... y direction, [y*W + x]
  int16_t* vol;        // [H][W][Dpad] filtered cost, int16 (Q14)
  uint32_t* key0;      // packed top-2 keys, (v + 32768) << 8 | (255 - k); 0 = empty
  uint32_t* key1;
  uint32_t* nb;        // winner's neighbour costs, lo16 = k*-1, hi16 = k*+1 (-32768 none)
  uint32_t* rkey;      // exact reverse match per right pixel (cfg.lrc), may be null
  float* disp;         // outputs, any may be null
  float* margin;
  uint8_t* conf;
  float* cand;         // 6 planes s1,s2,d1,d2,lrc,lrc2
  float* lrc2;         // the lrc2 plane alone (stage entry point), may be null
  // reference-layout candidates for the stage entry points (null otherwise)
  float* ref_cs;
  int* ref_cd;
  int* ref_cn;
  int16_t* ref_cnb;
  int W, H, D, Dpad;
  int cpitch;          // census row pitch in words (even: rows start 16-byte aligned)
  int apitch;          // ax row pitch in elements (multiple of 8)
  int lpad;            // left-row front pad (dmin & 1) so paired loads stay aligned
};

// Arithmetic configuration, precomputed on the host from de_cfg.
struct DevCfg {
  int dmin, iters, hw, hh;
  int wq;              // AD weight in 1/1024
  int trunc;           // AD truncation
  int packed;          // census words carry the pixel byte (window <= 48 bits)
  int subpixel, fit_eq, lrc;
  float lambda, gamma, damping, keep, min_margin, min_ratio;
  int expire_polls;    // test hook (knob "expire_wait_polls"), 0 = off
  int cols_async;      // column kernel's prefetch ring in shared memory (knob "cols_async")
  int16_t tbl[66];     // Q14 census score per Hamming distance
  int16_t adt[256];    // Q14 truncated-absolute-difference score
  uint16_t rf[256];    // Q15 filter coefficient per byte difference
};

struct Batch {
  int n;
  int maxDpad;
  int* err;            // device status word (bounded waits that ran out set it)
  int rows_prefix[kMaxBatch + 1];   // row-kernel work items (rows in [hh, H-hh))
  int cols_prefix[kMaxBatch + 1];   // column-kernel work items (cols with candidates)
  int solve_prefix[kMaxBatch + 1];  // solve work items (all rows)
  int pix_prefix[kMaxBatch + 1];    // census tiles
  DevPair p[kMaxBatch];
};

// de_dense_dev with a bound on the parts a batch runs as on concurrent streams (1: one
// launch set on `stream`); callers that already overlap batches of their own pass 1.
// `reg_ring` keeps the column kernel's prefetch ring in registers (de_capi.cu).
int dense_dev(const de_cfg* cfg, const de_pair* pairs, int n, void* workspace,
              size_t ws_bytes, cudaStream_t stream, int max_parts, bool reg_ring = false);

// Device address of the no-allocation entry point's status word on the current device
// (de_noalloc.cu); DE_OK or an error code already recorded for de_last_error().
int noalloc_status_word(void** out);

// Records a one-line reason for de_last_error() and returns code (de_capi.cu).
int set_error(int code, const char* fmt, ...);

// Host-side preparation (de_capi.cu).
void make_dev_cfg(const de_cfg& c, DevCfg* out);
size_t pair_workspace_bytes(int W, int H, int D, bool lrc);
void carve_pair(DevPair* p, void* ws, int W, int H, int D, int dmin, bool lrc);
constexpr size_t kStatusBytes = 256;   // head of every dense workspace

// Host-to-host copies (pageable <-> pinned), split over a few threads when there is
// enough to move (de_capi.cu).
struct HostCopy { void* dst; const void* src; size_t n; };
void parallel_copy(const std::vector<HostCopy>& jobs);

// Launchers (de_dense.cu).  All enqueue on `stream` and return the launch status.
cudaError_t launch_census(const DevCfg& cfg, const Batch& b, cudaStream_t s);
cudaError_t launch_rows(const DevCfg& cfg, const Batch& b, cudaStream_t s);
cudaError_t launch_cols(const DevCfg& cfg, const Batch& b, cudaStream_t s);
cudaError_t launch_solve(const DevCfg& cfg, const Batch& b, bool from_ref_layout,
                         cudaStream_t s);
void set_rows_ctas_per_sm(int v);
int get_rows_ctas_per_sm();
void set_cols_kt(int v);
void set_solve_threads(int v);
int get_solve_threads();
int get_cols_kt();
void set_cols_async(int v);
int get_cols_async();
void set_cols_pf(int v);
int get_cols_pf();
void set_cols_cta(int v);
int get_cols_cta();
void set_expire_polls(int v);
int get_expire_polls();
cudaError_t launch_export_candidates(const DevCfg& cfg, const Batch& b, cudaStream_t s);
// The prior-masked cost stage (de_prior.cu): one pair (b.p[0]) after its census.
size_t prior_ws_bytes(int W, int H, int D);
cudaError_t launch_prior(const DevCfg& cfg, const Batch& b, const float* prior, int band,
                         void* ws, cudaStream_t s);
// Hole filling of a disparity map for use as a prior (de_fill.cu).
size_t fill_ws_bytes(int W, int H);
int fill_holes_dev(const float* src, float* dst, int W, int H, void* ws, size_t ws_bytes,
                   cudaStream_t s);
// Sparse path (de_sparse.cu), for the host-pointer context.
size_t detect_ws_bytes(int W, int H, const de_det_cfg* c);
int detect_fast_dev(const uint8_t* img, int W, int H, const de_det_cfg* c, de_keypoint* out,
                    int cap, int* n_out, void* ws, size_t bytes, cudaStream_t s);
int kp_readout_dev(const de_keypoint* kp, int n, const int* n_dev, const float* disp,
                   const float* margin, int W, int H, de_kp_disparity* out, int cap,
                   int* n_out, cudaStream_t s);

}  // namespace de
