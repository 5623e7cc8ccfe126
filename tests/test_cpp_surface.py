"""The reference's C++ call surface (include/doubleeye/*.hpp over the C ABI).

* Without a GPU: the headers compile as C++14 together with a caller of every function
  the surface defines, and the reference's own core/tests/test_confidence.cpp, built
  unchanged against them (oracle/_ref/shim/, oracle/Makefile target shim), passes.
* On the GPU: the reference's own core/tests/test_match.cpp, built unchanged against
  the surface, passes with match_masda and the rest of the surface running on the
  device (brute-force optimality on 60 problems, exact counts, priors, margins, the
  convergence report).  Its out-of-scope helpers (brute force, mutual nearest
  neighbour, the coarse prior builder, sub-pixel refinement) run the reference's own
  code, as the Makefile recipe explains.

The harness binaries are built where the reference tree is available and travel with
the tree; without them these tests are skipped.
"""
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(REPO, "oracle", "_ref", "shim")

CALLER = r"""
#include "doubleeye/dense_solve.hpp"
#include "doubleeye/match.hpp"
#include "doubleeye/preproc.hpp"
using namespace doubleeye;
int main() {
  Image8 img(64, 48);
  CensusImage ci = census_transform(img, CensusConfig{});
  bool ok = false;
  uint64_t d = census_at(img, 10, 10, CensusConfig{}, &ok);
  DetectProfile prof;
  std::vector<Keypoint> kp = detect_keypoints_fast(img, DetectorConfig{}, &prof);
  MatchConfig mc;
  MatchStats st;
  std::vector<uint64_t> desc(kp.size(), d);
  std::vector<Match> m = match_masda(kp, desc, kp, desc, mc, &st);
  float s = pair_score(Keypoint{}, Keypoint{}, 0, 0, 48, mc);
  DisparityPrior pr;
  float pd = 0, psd = 0;
  bool have = pr.lookup(1.f, 1.f, &pd, &psd);
  Cfg cfg;
  float cs[4] = {0.5f, 0.2f, 0.4f, -1e30f};
  int cd[4] = {3, 5, 2, -1}, cn[2] = {2, 1};
  float disp[2], margin[2];
  solve_row_sparse(2, 8, 2, cfg, nullptr, cs, cd, cn, nullptr, nullptr, disp, margin, 3,
                   nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
  return int(ci.bits.size() + m.size() + s + have + confidence_u8(0.9f, 0.3f, -0.1f)) & 1;
}
"""


def _run(path):
    r = subprocess.run([path], capture_output=True, text=True, timeout=600)
    return r.returncode, r.stdout + r.stderr


def test_headers_compile_with_a_caller(tmp_path):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no g++")
    src = tmp_path / "caller.cpp"
    src.write_text(CALLER)
    r = subprocess.run([gxx, "-std=c++14", "-Wall", "-fsyntax-only",
                        "-I", os.path.join(REPO, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_reference_confidence_tests_pass():
    exe = os.path.join(SHIM, "test_confidence")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/shim not built (needs the reference tree)")
    rc, out = _run(exe)
    assert rc == 0 and "ALL PASSED" in out, out[-2000:]


@pytest.mark.gpu
def test_reference_match_tests_pass_on_the_gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    exe = os.path.join(SHIM, "test_match")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/shim not built (needs the reference tree)")
    from doubleeye_b200 import build
    build.build()
    rc, out = _run(exe)
    print(out[-3000:])
    assert rc == 0, out[-3000:]
    assert "FAIL" not in out
