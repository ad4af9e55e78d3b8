"""The reference's C++ library entries, ants::antsRegistration and ants::antsApplyTransforms, link and
behave like the reference's.

A wrapper that binds the reference declares `int ants::antsRegistration(std::vector<std::string>,
std::ostream*)` (Examples/include/antsRegistration.h:7-9) and `int ants::antsApplyTransforms(...)` of the
same shape (Examples/include/antsApplyTransforms.h:4-10).  The callers below are compiled against those
declarations alone and linked against libantsRegistration_b200.so / libantsApplyTransforms_b200.so; the
calls they make end before any device work (help, option errors), so this runs without a GPU.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "ants_b200")

CALLER = r"""
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace ants {
extern int antsRegistration(std::vector<std::string>, std::ostream*);
}

int main(int argc, char** argv) {
  std::vector<std::string> args(argv + 1, argv + argc);
  std::ostringstream log;
  const int rc = ants::antsRegistration(args, &log);
  std::cout << "rc=" << rc << "\n" << log.str();
  return 0;
}
"""


@pytest.fixture(scope="module")
def caller(tmp_path_factory):
    from ants_b200 import build
    build.build_lib()
    build.build_reg_lib()
    d = tmp_path_factory.mktemp("entry")
    src = d / "caller.cpp"
    src.write_text(CALLER)
    exe = d / "caller"
    subprocess.run(["g++", "-std=c++17", "-o", str(exe), str(src), "-L", LIBDIR, "-lantsRegistration_b200",
                    f"-Wl,-rpath,{LIBDIR}"], check=True)
    return str(exe)


def run(exe, args):
    r = subprocess.run([exe, *args], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    first, _, rest = r.stdout.partition("\n")
    return int(first.split("=")[1]), rest, r.stderr


def test_help_returns_success_through_the_reference_symbol(caller):
    rc, out, _ = run(caller, ["--help"])
    assert rc == 0
    assert "SyN" in out


def test_errors_return_exit_failure_without_throwing(caller):
    rc, _, err = run(caller, ["-Q", "1"])
    assert rc == 1
    assert "unexpected argument '-Q'" in err
    rc, _, err = run(caller, ["-d", "3", "--float", "1", "-t", "Affine[0.1]", "-m", "CC[a.nii,b.nii,1,4]",
                              "-c", "10", "-f", "1", "-s", "0", "-o", "out"])
    assert rc == 1
    assert "only the SyN transform is supported" in err


def test_double_precision_request_warns(caller):
    base = ["-d", "3", "-t", "Affine[0.1]", "-m", "CC[a.nii,b.nii,1,4]", "-c", "10", "-f", "1", "-s", "0", "-o", "out"]
    _, _, err0 = run(caller, base + ["--float", "0"])
    _, _, err_default = run(caller, base)
    _, _, err1 = run(caller, base + ["--float", "1"])
    assert "WARNING: double precision requested" in err0
    assert "WARNING: double precision requested" in err_default
    assert "WARNING" not in err1


APPLY_CALLER = CALLER.replace("antsRegistration", "antsApplyTransforms")


@pytest.fixture(scope="module")
def apply_caller(tmp_path_factory):
    from ants_b200 import build
    build.build_lib()
    build.build_apply_lib()
    d = tmp_path_factory.mktemp("apply_entry")
    src = d / "caller.cpp"
    src.write_text(APPLY_CALLER)
    exe = d / "caller"
    subprocess.run(["g++", "-std=c++17", "-o", str(exe), str(src), "-L", LIBDIR, "-lantsApplyTransforms_b200",
                    f"-Wl,-rpath,{LIBDIR}"], check=True)
    return str(exe)


def test_apply_entry_symbol(apply_caller, tmp_path):
    rc, out, _ = run(apply_caller, ["--help"])
    assert rc == 0 and "antsApplyTransforms_b200" in out
    rc, _, err = run(apply_caller, ["-Q", "1"])
    assert rc == 1 and "unexpected argument '-Q'" in err
    # a missing input file fails inside the call, before any device work, without an exception escaping
    rc, _, err = run(apply_caller, ["-d", "3", "-i", str(tmp_path / "none.nii.gz"), "-r", str(tmp_path / "none.nii.gz"),
                                    "-t", "[" + str(tmp_path / "w.nii.gz") + ",1]", "-o", str(tmp_path / "o.nii.gz")])
    assert rc == 1 and "inverse of displacement field" in err
