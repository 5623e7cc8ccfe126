// doubleeye_b200 -- the C++14 call surface of core/include/doubleeye/preproc.hpp
// (mayio/doubleeye), backed by the B200 build.
//
// Same namespace, type names, members, defaults and function signatures as the
// reference header, so code written against it compiles unchanged.  The types are
// laid out member for member as the reference's (an object built here can be handed
// to code compiled against the reference header).
//
// Defined by this build, on the GPU through the C ABI (include/doubleeye_b200.h,
// host-pointer de_ctx_* entry points; link libdoubleeye_cpp.a and
// libdoubleeye_b200.so):
//   census_transform, census_at, detect_keypoints_fast
// and, inline below, hamming.
// Declared for source compatibility only (outside the stereo hot path, not defined by
// this build): load_raw_y8, save_pgm, downsample, local_std, local_std_at,
// shi_tomasi_response, detect_keypoints, is_fast_corner, shi_tomasi_at,
// cell_occupancy.
//
// Errors from the device path (no CUDA device, sizes beyond the C ABI's limits) are
// thrown as std::runtime_error with de_last_error()'s reason.

#ifndef DOUBLEEYE_PREPROC_HPP
#define DOUBLEEYE_PREPROC_HPP

#include <cstdint>
#include <string>
#include <vector>

namespace doubleeye {

// An 8-bit single-channel image, row-major with pitch == width.
struct Image8 {
  int width = 0;
  int height = 0;
  std::vector<uint8_t> data;

  Image8() = default;
  Image8(int w, int h) : width(w), height(h), data(size_t(w) * h, 0) {}
  bool empty() const { return width <= 0 || height <= 0; }
  size_t pixels() const { return size_t(width) * size_t(height); }
  uint8_t at(int x, int y) const { return data[size_t(y) * width + x]; }
  uint8_t& at(int x, int y) { return data[size_t(y) * width + x]; }
};

bool load_raw_y8(const std::string& path, int width, int height, Image8* out);
bool save_pgm(const std::string& path, const Image8& img);
Image8 downsample(const Image8& img, int factor);

// Census window half-sizes; bits() is the descriptor length (window minus centre).
struct CensusConfig {
  int half_w = 3;
  int half_h = 3;
  int bits() const { return (2 * half_w + 1) * (2 * half_h + 1) - 1; }
};

struct CensusImage {
  int width = 0;
  int height = 0;
  std::vector<uint64_t> bits;   // descriptor per pixel
  std::vector<uint8_t> valid;   // 0 where the window leaves the image
  CensusConfig config;

  uint64_t at(int x, int y) const { return bits[size_t(y) * width + x]; }
  bool is_valid(int x, int y) const { return valid[size_t(y) * width + x] != 0; }
};

// Census of every pixel (bit b set where the b-th window neighbour, row-major with the
// centre skipped, is darker than the centre; 0 and invalid within the border).
CensusImage census_transform(const Image8& img, CensusConfig cfg);

// Census of one pixel; *ok (if given) says whether the window fits the image.
uint64_t census_at(const Image8& img, int x, int y, CensusConfig cfg,
                   bool* ok = nullptr);

inline int hamming(uint64_t a, uint64_t b) {
  return __builtin_popcountll(a ^ b);
}

std::vector<float> local_std(const Image8& img, int window);
float local_std_at(const Image8& img, int x, int y, int window);

struct Keypoint {
  float x = 0.f;          // sub-pixel
  float y = 0.f;
  float response = 0.f;   // Shi-Tomasi minimum eigenvalue
  float local_std = 0.f;  // texture energy around the point
};

struct DetectorConfig {
  int grad_window = 3;         // structure-tensor window
  int cell = 32;               // grid cell for the spatial spread
  int per_cell = 3;            // strongest kept per cell
  float min_response = 1.0f;
  float min_local_std = 2.0f;  // texture floor
  int border = 8;              // larger than the census half-window
  bool subpixel = true;
  int fast_threshold = 8;
  int nms_radius = 3;          // suppression radius of the FAST path
};

std::vector<float> shi_tomasi_response(const Image8& img, int grad_window);
std::vector<Keypoint> detect_keypoints(const Image8& img, const DetectorConfig& cfg);
bool is_fast_corner(const Image8& img, int x, int y, int threshold);
float shi_tomasi_at(const Image8& img, int x, int y, int grad_window);

// Stage timings of detect_keypoints_fast.  This build runs the detector as one
// device call and reports its whole time as fast_ms; the counts are not collected.
struct DetectProfile {
  double fast_ms = 0;
  double nms_ms = 0;
  double refine_ms = 0;
  int candidates = 0;
  int suppressed = 0;
  double total_ms() const { return fast_ms + nms_ms + refine_ms; }
};

// FAST-9 corners, Shi-Tomasi response, strongest-first suppression, texture floor,
// sub-pixel refinement and the per-cell cut, in the reference's output order.
std::vector<Keypoint> detect_keypoints_fast(const Image8& img, const DetectorConfig& cfg,
                                            DetectProfile* prof = nullptr);

float cell_occupancy(const std::vector<Keypoint>& kps, int width, int height, int cell);

}  // namespace doubleeye

#endif  // DOUBLEEYE_PREPROC_HPP
