"""Host code under AddressSanitizer and UndefinedBehaviorSanitizer, and the command lines' --help.

The readers of user files -- the ITK transform-file parsers (synx_linear.cpp), the composite and
registration-state reader (composite_txt.h) and the NIfTI reader (nifti_io.cpp) -- are compiled with -fsanitize=address,undefined and fed seeded mutations of valid
files (truncations, byte flips, insertions, random bytes).  Each case must either parse or fail with
an error; any sanitizer report fails the test.  The reference has no sanitizer builds; its smoke tests
run every program's --help (Examples/TestSuite/CMakeLists.txt:1038-1044), mirrored at the end.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "ants_b200", "csrc")
INCLUDE = os.path.join(ROOT, "include")

DRIVER = r"""
#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>
#include "composite_txt.h"
#include "nifti_io.h"
#include "synx.h"
#include "synx_host.h"
static std::string g_msg;
namespace synx { int set_global_error(int code, const std::string& m) { g_msg = m; return code; } }
extern "C" const char* synx_last_error(const synx_ctx*) { return g_msg.c_str(); }

static std::vector<unsigned char> mutate(std::vector<unsigned char> b, std::mt19937& rng) {
  switch (rng() % 4) {
    case 0: if (!b.empty()) b.resize(rng() % b.size()); break;
    case 1: for (int k = 0; k < 1 + (int)(rng() % 8); ++k) if (!b.empty()) b[rng() % b.size()] = (unsigned char)rng(); break;
    case 2: b.resize(rng() % 400); for (auto& c : b) c = (unsigned char)rng(); break;
    default: if (!b.empty()) b.insert(b.begin() + rng() % b.size(), (unsigned char)rng()); break;
  }
  return b;
}

static void put(const std::string& p, const std::vector<unsigned char>& b) {
  FILE* f = fopen(p.c_str(), "wb"); fwrite(b.data(), 1, b.size(), f); fclose(f);
}

int main(int argc, char** argv) {
  const std::string dir = argv[1];
  const int cases = atoi(argv[2]);
  std::mt19937 rng(7);
  // seeds: a MATLAB v4 affine, an Insight text affine, a NIfTI-1 image, a composite (rigid entry and a
  // 2 x 2 displacement field, the form of a saved registration state)
  std::vector<unsigned char> mat;
  auto add = [&](const void* p, size_t n) { auto* c = (const unsigned char*)p; mat.insert(mat.end(), c, c + n); };
  auto var = [&](const char* name, int n) {
    int h[5] = {0, n, 1, 0, (int)strlen(name) + 1}; add(h, 20); add(name, strlen(name) + 1);
    for (int i = 0; i < n; ++i) { double d = 0.25 * i; add(&d, 8); }
  };
  var("AffineTransform_double_3_3", 12);
  var("fixed", 3);
  const std::string txt = "#Insight Transform File V1.0\n#Transform 0\nTransform: Euler3DTransform_double_3_3\n"
                          "Parameters: 0.1 0.2 0.3 1 2 3\nFixedParameters: 0 0 0 1\n";
  nifti::Image im; im.dim = 3; im.size[0] = 5; im.size[1] = 4; im.size[2] = 3; im.data.assign(60, 1.5f);
  nifti::write(dir + "/seed.nii", im);
  std::vector<unsigned char> nii;
  { FILE* f = fopen((dir + "/seed.nii").c_str(), "rb"); unsigned char buf[4096]; size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) nii.insert(nii.end(), buf, buf + n); fclose(f); }
  const std::vector<unsigned char> txtb(txt.begin(), txt.end());
  const std::string comp = "#Insight Transform File V1.0\n#Transform 0\nTransform: CompositeTransform_double_2_2\n"
                           "#Transform 1\nTransform: Euler2DTransform_double_2_2\nParameters: 0.1 1 2\n"
                           "FixedParameters: 3 4\n#Transform 2\nTransform: DisplacementFieldTransform_float_2_2\n"
                           "Parameters: 0.5 -0.25 0 1 2 3 4 5\nFixedParameters: 2 2 0 0 1 1 1 0 0 1\n";
  const std::vector<unsigned char> compb(comp.begin(), comp.end());
  long parsed = 0, rejected = 0, cparsed = 0, crejected = 0;
  for (int it = 0; it < cases; ++it) {
    const int which = it % 4;
    if (which == 3) {
      const std::string path = dir + "/c.txt";
      put(path, mutate(compb, rng));
      try {
        std::vector<ants_b200::composite::Item> items = ants_b200::composite::read(path);
        for (const auto& item : items)
          for (int dim = 2; dim <= 3; ++dim) {
            try {
              if (item.is_field()) ants_b200::composite::field_geom(item, dim);
              else ants_b200::composite::to_linear(item, dim);
            } catch (const std::exception&) {
            }
          }
        ants_b200::composite::write(dir + "/rt.txt", 2, items);
        if (ants_b200::composite::read(dir + "/rt.txt").size() != items.size()) return 3;
        ++cparsed;
      } catch (const std::exception&) {
        ++crejected;
      }
      continue;
    }
    const std::string path = dir + (which == 0 ? "/x.mat" : which == 1 ? "/x.txt" : "/x.nii");
    put(path, mutate(which == 0 ? mat : which == 1 ? txtb : nii, rng));
    if (which < 2) {
      for (int dim = 2; dim <= 3; ++dim) {
        synx_linear t;
        if (synx_read_linear_transform(path.c_str(), dim, 0, &t) > 0) {
          ++parsed;
          synx_geom g{}; g.dim = dim; g.size[0] = 3; g.size[1] = 3; g.size[2] = dim == 3 ? 3 : 1;
          for (int k = 0; k < 3; ++k) g.spacing[k] = 1.0;
          g.direction[0] = g.direction[4] = g.direction[8] = 1.0;
          std::vector<float> u(27 * 3);
          synx_linear_field(&t, it & 1, &g, u.data());
        } else {
          ++rejected;
        }
      }
    } else {
      try { nifti::read(path); ++parsed; } catch (const std::exception&) { ++rejected; }
    }
  }
  printf("parsed %ld rejected %ld cparsed %ld crejected %ld\n", parsed, rejected, cparsed, crejected);
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_file_readers_under_sanitizers(tmp_path):
    src = tmp_path / "driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "driver"
    build = subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
                            "-I", INCLUDE, "-I", CSRC, "-o", str(exe), str(src), os.path.join(CSRC, "synx_linear.cpp"),
                            os.path.join(CSRC, "nifti_io.cpp"), "-lz"], capture_output=True, text=True, timeout=300)
    assert build.returncode == 0, build.stderr[-2000:]
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:allocator_may_return_null=1", UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([str(exe), str(tmp_path), "4000"], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, (r.stdout + r.stderr)[-3000:]
    assert "runtime error" not in r.stderr and "AddressSanitizer" not in r.stderr, r.stderr[-3000:]
    parsed, rejected, cparsed, crejected = (int(x) for x in r.stdout.split()[1::2])
    assert parsed > 0 and rejected > 0 and cparsed > 0 and crejected > 0, r.stdout


ROUND_TRIP = r"""
#include <cstdio>
#include <random>
#include <string>
#include <vector>
#include "composite_txt.h"
#include "nifti_io.h"
static std::string g_msg;
namespace synx { int set_global_error(int code, const std::string& m) { g_msg = m; return code; } }
extern "C" const char* synx_last_error(const synx_ctx*) { return g_msg.c_str(); }
int main(int argc, char** argv) {
  // a .nii.gz large enough for several gzip members compressed on separate threads
  nifti::Image im; im.dim = 3; im.components = 3; im.size[0] = 131; im.size[1] = 97; im.size[2] = 83;
  im.data.resize(3ull * 131 * 97 * 83);
  std::mt19937 r0(5); std::normal_distribution<float> n0(0.f, 1.f);
  for (auto& x : im.data) x = n0(r0);
  nifti::write(std::string(argv[1]) + "/big.nii.gz", im);
  if (nifti::read(std::string(argv[1]) + "/big.nii.gz").data != im.data) return 4;
  // a field large enough for the threaded formatting (> 64 K numbers) and parsing (> 1 MB of text)
  synx_geom g{}; g.dim = 2; g.size[0] = 611; g.size[1] = 467; g.size[2] = 1;
  g.spacing[0] = 0.7; g.spacing[1] = 1.3; g.spacing[2] = 1.0;
  g.direction[0] = g.direction[4] = g.direction[8] = 1.0;
  std::vector<float> v(2 * 611 * 467);
  std::mt19937 rng(3); std::normal_distribution<float> nd(0.f, 3.f);
  for (auto& x : v) x = nd(rng);
  const std::string path = std::string(argv[1]) + "/big.txt";
  ants_b200::composite::write(path, 2, {ants_b200::composite::field_item(g, v, false)});
  const auto back = ants_b200::composite::read(path);
  if (back.size() != 1 || back[0].field != v) return 2;
  const synx_geom gb = ants_b200::composite::field_geom(back[0], 2);
  if (gb.size[0] != 611 || gb.size[1] != 467 || gb.spacing[0] != 0.7) return 3;
  std::printf("round trip ok\n");
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
@pytest.mark.parametrize("sanitizer", ["address,undefined", "thread"])
def test_large_composite_round_trip(tmp_path, sanitizer):
    # the threaded number formatting and parsing of a large field, and the threaded gzip members of a
    # large .nii.gz: values back bit for bit, with no sanitizer finding (memory errors, undefined
    # behaviour, data races)
    src = tmp_path / "rt.cpp"
    src.write_text(ROUND_TRIP)
    exe = tmp_path / "rt"
    build = subprocess.run(["g++", "-std=c++17", "-O1", "-g", f"-fsanitize={sanitizer}", "-fno-sanitize-recover=all",
                            "-I", INCLUDE, "-I", CSRC, "-o", str(exe), str(src), os.path.join(CSRC, "synx_linear.cpp"),
                            os.path.join(CSRC, "nifti_io.cpp"), "-lz"], capture_output=True, text=True, timeout=300)
    assert build.returncode == 0, build.stderr[-2000:]
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "round trip ok" in r.stdout, (r.stdout + r.stderr)[-3000:]
    assert "WARNING: ThreadSanitizer" not in r.stderr and "AddressSanitizer" not in r.stderr, r.stderr[-3000:]


@pytest.mark.parametrize("exe", ["antsRegistrationSyN_b200", "antsApplyTransforms_b200"])
def test_help(exe):
    from ants_b200 import build
    build.build_all()
    for flag in ("--help", "-h"):
        r = subprocess.run([os.path.join(ROOT, "ants_b200", exe), flag], capture_output=True, text=True, timeout=60)
        assert r.returncode == 0, r.stderr
        assert exe in r.stdout
