// Test infrastructure: prints the size and member offsets of the C++ surface's types.
// Compiled once against the reference's headers and once against this build's
// include/doubleeye/, the two outputs must be identical, so objects cross freely
// between code compiled against either (oracle/Makefile, target shim).
#include <cstddef>
#include <cstdio>

#include "doubleeye/dense_solve.hpp"
#include "doubleeye/match.hpp"
#include "doubleeye/preproc.hpp"

#define SHOW(T) std::printf("%s %zu\n", #T, sizeof(T))
#define AT(T, m) std::printf("%s.%s %zu\n", #T, #m, offsetof(T, m))

int main() {
  using namespace doubleeye;
  SHOW(Image8); AT(Image8, width); AT(Image8, height); AT(Image8, data);
  SHOW(CensusConfig); SHOW(CensusImage); AT(CensusImage, bits); AT(CensusImage, valid);
  AT(CensusImage, config);
  SHOW(Keypoint); AT(Keypoint, response); AT(Keypoint, local_std);
  SHOW(DetectorConfig); AT(DetectorConfig, min_response); AT(DetectorConfig, subpixel);
  AT(DetectorConfig, fast_threshold); AT(DetectorConfig, nms_radius);
  SHOW(DetectProfile); AT(DetectProfile, candidates); AT(DetectProfile, suppressed);
  SHOW(Match); AT(Match, belief); AT(Match, margin);
  SHOW(DisparityPrior); AT(DisparityPrior, disparity); AT(DisparityPrior, valid);
  SHOW(SmoothPrior); AT(SmoothPrior, valid);
  SHOW(MatchConfig); AT(MatchConfig, max_candidates); AT(MatchConfig, prior);
  AT(MatchConfig, w_prior); AT(MatchConfig, smooth); AT(MatchConfig, w_smooth);
  AT(MatchConfig, iterations); AT(MatchConfig, lambda); AT(MatchConfig, converge_eps);
  SHOW(MatchStats); AT(MatchStats, converged); AT(MatchStats, final_max_delta);
  AT(MatchStats, oscillating);
  SHOW(SmoothResult); SHOW(CoarseToFineResult); AT(CoarseToFineResult, prior);
  AT(CoarseToFineResult, fine_ms);
  SHOW(Cfg); AT(Cfg, agg); AT(Cfg, sigma_s); AT(Cfg, fit_eq); AT(Cfg, eps); AT(Cfg, topk);
  AT(Cfg, csct); AT(Cfg, ad); AT(Cfg, lambda); AT(Cfg, min_ratio); AT(Cfg, lrc);
  AT(Cfg, threads); AT(Cfg, noblock);
  SHOW(Top2);
  return 0;
}
