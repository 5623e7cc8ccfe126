// doubleeye_b200 -- the C++14 call surface of core/include/doubleeye/match.hpp
// (mayio/doubleeye): keypoint MASDA, backed by the B200 build.
//
// Same namespace, type names, members, defaults and signatures as the reference
// header; the types are laid out member for member as the reference's.
//
// Defined by this build:
//   match_masda          on the GPU (de_ctx_match_masda): candidate graph, damped
//                        max-sum sweeps, margins and the emission order of
//                        core/src/match.cpp:334-417, with the soft coarse and
//                        smoothness priors of MatchConfig resolved per left keypoint
//                        here and applied in the device's pair score
//   pair_score           s(i,j) of one pair (core/src/match.cpp:298-332), the formula
//                        the device applies inside match_masda, for callers that reason
//                        about the score scale
//   DisparityPrior::lookup, DisparityPrior::coverage
// Declared for source compatibility only (outside the stereo hot path, not defined by
// this build): build_disparity_prior, fit_smooth_prior, match_iterated_smoothness,
// match_mutual_nn, match_coarse_to_fine, match_brute_force, refine_disparity,
// matching_objective.
//
// Exact ties in the reference's std::sort orders are broken here by input position.

#ifndef DOUBLEEYE_MATCH_HPP
#define DOUBLEEYE_MATCH_HPP

#include "doubleeye/preproc.hpp"

#include <cstdint>
#include <vector>

namespace doubleeye {

struct Match {
  int left = -1;
  int right = -1;
  float score = 0.f;      // s(i,j)
  float belief = 0.f;     // max-sum belief of the accepted edge
  float disparity = 0.f;  // xL - xR
  float dy = 0.f;         // yL - yR
  float margin = 0.f;     // best minus second-best score of the left keypoint's candidates
};

// A coarse, per-cell disparity expectation: a soft penalty in s(i,j), never a veto.
struct DisparityPrior {
  int cell = 64;              // full-resolution pixels per cell
  int cols = 0;
  int rows = 0;
  std::vector<float> disparity;
  std::vector<float> sigma;
  std::vector<uint8_t> valid;

  bool lookup(float x, float y, float* d, float* sd) const;
  float coverage() const;     // fraction of cells with a prediction
};

DisparityPrior build_disparity_prior(const std::vector<Match>& coarse,
                                     const std::vector<Keypoint>& coarse_left,
                                     int full_width, int full_height, int scale,
                                     int cell = 64, int min_count = 3,
                                     float sigma_floor = 2.0f);

// A per-left-keypoint disparity expectation from a previous pass.
struct SmoothPrior {
  std::vector<float> disparity;
  std::vector<float> sigma;
  std::vector<uint8_t> valid;
};

SmoothPrior fit_smooth_prior(const std::vector<Match>& matches,
                             const std::vector<Keypoint>& left,
                             int k_neighbours = 10,
                             float sigma_floor = 0.75f,
                             int irls_iterations = 3);

struct MatchConfig {
  // candidate generation
  float max_dy = 2.0f;
  float min_disparity = 1.0f;
  float max_disparity = 220.0f;
  int max_candidates = 24;        // per left keypoint, best by score
  // scoring
  float sigma_y = 1.0f;
  float w_y = 1.0f;
  const DisparityPrior* prior = nullptr;
  float w_prior = 1.0f;
  const SmoothPrior* smooth = nullptr;
  float w_smooth = 1.0f;
  // message passing
  int iterations = 20;
  float damping = 0.4f;
  float lambda = 0.0f;            // clutter: a left keypoint left unmatched
  float gamma = 0.0f;             // misdetection: a right keypoint left unmatched
  float converge_eps = 1e-4f;
};

struct MatchStats {
  int left = 0;
  int right = 0;
  int candidates = 0;
  int iterations_run = 0;
  bool converged = false;
  float final_max_delta = 0.f;
  int oscillating = 0;
};

float pair_score(const Keypoint& l, const Keypoint& r, uint64_t dl, uint64_t dr,
                 int census_bits, const MatchConfig& cfg, int left_index = -1);

struct SmoothResult {
  std::vector<Match> matches;
  std::vector<Match> first_pass;
  std::vector<float> base_objective;
  std::vector<int> counts;
  std::vector<float> median_abs_dy;
  std::vector<int> changed;
  std::vector<float> prior_coverage;
};

SmoothResult match_iterated_smoothness(const std::vector<Keypoint>& left,
                                       const std::vector<uint64_t>& desc_left,
                                       const std::vector<Keypoint>& right,
                                       const std::vector<uint64_t>& desc_right,
                                       const MatchConfig& cfg,
                                       int passes = 3,
                                       int k_neighbours = 10);

// MASDA over the keypoints of a rectified pair; descriptors parallel to their
// keypoint vectors.
std::vector<Match> match_masda(const std::vector<Keypoint>& left,
                               const std::vector<uint64_t>& desc_left,
                               const std::vector<Keypoint>& right,
                               const std::vector<uint64_t>& desc_right,
                               const MatchConfig& cfg,
                               MatchStats* stats = nullptr);

std::vector<Match> match_mutual_nn(const std::vector<Keypoint>& left,
                                   const std::vector<uint64_t>& desc_left,
                                   const std::vector<Keypoint>& right,
                                   const std::vector<uint64_t>& desc_right,
                                   const MatchConfig& cfg,
                                   float ratio = 0.85f,
                                   MatchStats* stats = nullptr);

struct CoarseToFineResult {
  std::vector<Match> matches;
  std::vector<Match> coarse_matches;
  DisparityPrior prior;
  MatchStats fine_stats;
  MatchStats coarse_stats;
  double coarse_ms = 0.0;
  double fine_ms = 0.0;
};

CoarseToFineResult match_coarse_to_fine(const Image8& left_img,
                                        const Image8& right_img,
                                        const DetectorConfig& det,
                                        const CensusConfig& census,
                                        const MatchConfig& cfg,
                                        int scale = 8,
                                        int prior_cell = 64);

std::vector<Match> match_brute_force(const std::vector<Keypoint>& left,
                                     const std::vector<uint64_t>& desc_left,
                                     const std::vector<Keypoint>& right,
                                     const std::vector<uint64_t>& desc_right,
                                     const MatchConfig& cfg);

void refine_disparity(const Image8& left, const Image8& right,
                      const std::vector<Keypoint>& kl,
                      const std::vector<Keypoint>& kr,
                      std::vector<Match>* matches, int half = 3);

float matching_objective(const std::vector<Match>& matches,
                         const MatchConfig& cfg, int n_left, int n_right);

}  // namespace doubleeye

#endif  // DOUBLEEYE_MATCH_HPP
