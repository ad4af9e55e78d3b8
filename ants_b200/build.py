"""Build the synx CUDA library (libsynx.so) and the antsRegistration-compatible host binary.

Everything is compiled in-tree for sm_100a with nvcc; no JIT cache is involved, so the built
files travel with the source tree.

    python -m ants_b200.build            # build what is out of date
    python -m ants_b200.build --force    # rebuild everything
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall", "-Xcompiler", "-pthread",
              "--expt-relaxed-constexpr"]

LIB = os.path.join(HERE, "libsynx.so")
CLI = os.path.join(HERE, "antsRegistrationSyN_b200")
# the C++ library entry `ants::antsRegistration(std::vector<std::string>, std::ostream*)`
REG_LIB = os.path.join(HERE, "libantsRegistration_b200.so")
APPLY_CLI = os.path.join(HERE, "antsApplyTransforms_b200")
# the C++ library entry `ants::antsApplyTransforms(std::vector<std::string>, std::ostream*)`
APPLY_LIB = os.path.join(HERE, "libantsApplyTransforms_b200.so")

LIB_SOURCES = ["synx_kernels.cu", "synx_cc.cu", "synx_level.cu", "synx_ctx.cu", "synx_noalloc.cu", "synx_server.cpp",
               "synx_linear.cpp", "synx_tune.cpp"]
LIB_HEADERS = ["synx_device.cuh", "synx_kernels.cuh", "synx_phases.cuh", "synx_cc_tile.cuh", "synx_level.cuh",
               "synx_level_body.cuh", "synx_host.h", "synx_nvtx.h"]
CLI_SOURCES = ["ants_registration.cpp", "nifti_io.cpp"]
APPLY_SOURCES = ["ants_apply_transforms.cpp", "nifti_io.cpp"]
CLI_HEADERS = ["nifti_io.h", "ants_registration.h", "ants_apply_transforms.h", "cli_common.h", "composite_txt.h"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _host_cxx() -> str:
    # the system g++ (some environments point CXX at a toolchain without libgomp)
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


BUILD_DIR = os.path.join(HERE, "_build")
LEVEL_RADII = range(1, 8)  # the persistent level kernel is instantiated once per CC radius


def _objects() -> list[tuple[str, str, list[str]]]:
    """(source, object, extra flags) for every compile unit of libsynx.so."""
    units = [(os.path.join(CSRC, s), os.path.join(BUILD_DIR, os.path.splitext(s)[0] + ".o"), []) for s in LIB_SOURCES]
    inst = os.path.join(CSRC, "synx_level_inst.cu")
    units += [(inst, os.path.join(BUILD_DIR, f"synx_level_r{r}.o"), [f"-DSYNX_RCC={r}"]) for r in LEVEL_RADII]
    return units


def build_lib(force: bool = False, verbose_ptxas: bool = False) -> str:
    from concurrent.futures import ThreadPoolExecutor

    headers = [os.path.join(CSRC, h) for h in LIB_HEADERS] + [os.path.join(INCLUDE, "synx.h")]
    os.makedirs(BUILD_DIR, exist_ok=True)
    jobs = []
    for src, obj, extra in _objects():
        if force or _stale(obj, [src] + headers):
            cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, "-ccbin", _host_cxx(), *extra, "-c", "-o", obj, src]
            if verbose_ptxas:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    if jobs:
        with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
            list(ex.map(_run, jobs))
    objs = [o for _, o, _ in _objects()]
    if force or jobs or _stale(LIB, objs):
        _run([_nvcc(), *ARCH, "-ccbin", _host_cxx(), "-shared", "-o", LIB, *objs, "-lcudart", "-ldl", "-Xcompiler",
              "-pthread"])
    return LIB


def _build_exe(target: str, sources: list[str], force: bool) -> str | None:
    srcs = [os.path.join(CSRC, s) for s in sources]
    if not all(os.path.exists(s) for s in srcs):
        return None
    deps = srcs + [os.path.join(CSRC, h) for h in CLI_HEADERS] + [LIB]
    if not force and not _stale(target, deps):
        return target
    cmd = [_host_cxx(), "-O2", "-std=c++17", "-Wall", "-I", INCLUDE, "-I", "/usr/local/cuda/include", "-o", target,
           *srcs, "-L", HERE, "-lsynx", "-Wl,-rpath,$ORIGIN", "-L", "/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath,/usr/local/cuda/lib64", "-lz"]
    _run(cmd)
    return target


def _build_entry_lib(target: str, sources: list[str], force: bool) -> str:
    """A command line without its main(), as a shared library exporting its ants:: entry symbol."""
    srcs = [os.path.join(CSRC, s) for s in sources]
    deps = srcs + [os.path.join(CSRC, h) for h in CLI_HEADERS] + [LIB]
    if not force and not _stale(target, deps):
        return target
    cmd = [_host_cxx(), "-O2", "-std=c++17", "-Wall", "-fPIC", "-shared", "-DSYNX_CLI_NO_MAIN", "-I", INCLUDE,
           "-I", "/usr/local/cuda/include", "-o", target, *srcs, "-L", HERE, "-lsynx", "-Wl,-rpath,$ORIGIN",
           "-L", "/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath,/usr/local/cuda/lib64", "-lz"]
    _run(cmd)
    return target


def build_reg_lib(force: bool = False) -> str | None:
    """libantsRegistration_b200.so: the registration command line without its main(), exporting the
    reference's library symbol ants::antsRegistration for wrappers."""
    return _build_entry_lib(REG_LIB, CLI_SOURCES, force)


def build_apply_lib(force: bool = False) -> str | None:
    """libantsApplyTransforms_b200.so: the same for ants::antsApplyTransforms."""
    return _build_entry_lib(APPLY_LIB, APPLY_SOURCES, force)


def build_cli(force: bool = False) -> str | None:
    """antsRegistrationSyN_b200, antsApplyTransforms_b200 and the two entry-symbol libraries."""
    _build_exe(APPLY_CLI, APPLY_SOURCES, force)
    build_apply_lib(force)
    build_reg_lib(force)
    return _build_exe(CLI, CLI_SOURCES, force)


def build_all(force: bool = False) -> None:
    build_lib(force)
    build_cli(force)


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print ptxas register/smem usage")
    a = ap.parse_args(argv)
    build_lib(a.force or a.ptxas, verbose_ptxas=a.ptxas)
    build_cli(a.force)
    return 0


if __name__ == "__main__":
    sys.exit(main())
