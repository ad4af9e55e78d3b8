"""The serving loop's own logic, on a machine without a GPU.

The real ants_b200/csrc/synx_server.cpp is compiled into a host shared library together with the
host stand-ins of tests/cli_host/ (CUDA runtime calls; stage and batch entry points backed by the
CPU oracle's registration, one pyramid level per batch step; a stand-in footprint) and stubs for the
rest of the C ABI.  A child process loads that library through the Python binding and drives
synx.Server: admission within the budget without head-of-line blocking, the resident limit,
rejection of a request above the budget, pooled contexts reused by later requests with the same
parameters, and each request's fields equal to the oracle's registration.  What this covers is the
loop's logic; the device behaviour is the GPU server tests'.
"""
import json
import os
import re
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "ants_b200", "csrc")
HOST = os.path.join(ROOT, "tests", "cli_host")


def _stubs(sources) -> str:
    """Definitions for every function include/synx.h declares that `sources` do not define."""
    header = open(os.path.join(ROOT, "include", "synx.h")).read()
    declared = re.findall(r"^(int|const char\*)\s+(synx_\w+)\(", header, flags=re.M)
    defined = set()
    for src in sources:
        text = open(src).read()
        defined |= set(re.findall(r"\b(synx_\w+)\s*\([^;{}]*\)\s*\{", text))
    # without synx.h: the stubs only have to exist as symbols the binding can look up
    out = ['extern "C" {']
    for ret, name in declared:
        if name in defined:
            continue
        value = "-5" if ret == "int" else '""'  # SYNX_E_UNSUPPORTED
        out.append(f"{ret} {name}(...) {{ return {value}; }}")
    out.append("}")
    return "\n".join(out) + "\n"


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    out = tmp_path_factory.mktemp("server_host")
    sources = [os.path.join(CSRC, "synx_server.cpp"), os.path.join(HOST, "host_stage.cpp"),
               os.path.join(HOST, "host_steps.cpp"), os.path.join(CSRC, "synx_linear.cpp")]
    stubs = out / "stubs.cpp"
    stubs.write_text(_stubs(sources))
    so = str(out / "libsynx_host.so")
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-fopenmp", "-pthread", "-I", HOST, "-I",
           os.path.join(ROOT, "include"), "-I", CSRC, "-I", os.path.join(ROOT, "oracle"), "-o", so, *sources,
           str(stubs), os.path.join(ROOT, "oracle", "synx_oracle_capi.cpp")]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return so


DRIVER = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, ROOT)
sys.path.insert(0, ROOT + "/oracle")
from ants_b200 import phantoms, synx
lib = synx.load_library(SO)
lib.host_stage_created.restype = ctypes.c_int
import oracle as O
from ants_b200.synx import Geom, Server, SyNParams, SynxError

def params(levels, radius=2):
    return SyNParams(dim=2, cc_radius=radius, iterations=(3, 2, 2)[-levels:], shrink_factors=(4, 2, 1)[-levels:],
                     smoothing_sigmas=(1.0, 0.5, 0.0)[-levels:], convergence_threshold=1e-12)

def pair(n, seed):
    f, m = phantoms.pair_2d((n, n - 4), seed=seed)
    return f, m, Geom((n, n - 4))

res = {}
# admission within a budget that holds two of four requests (mixed sizes and level counts)
reqs = [(pair(n, 40 + k), params(lv)) for k, (n, lv) in enumerate([(40, 2), (24, 2), (36, 3), (28, 1)])]
fps = [synx.footprint(P, g, g) for (f, m, g), P in reqs]
budget = max(fps) + min(fps)
with Server(hbm_budget_bytes=budget) as srv:
    ids = [srv.submit(P, f, g, m, g) for (f, m, g), P in reqs]
    outs = [srv.wait(i, timeout=600) for i in ids]
    st = srv.stats()
res["peak_within_budget"] = st["bytes_peak"] <= budget
res["all_done"] = all(o[2]["status"] == 2 for o in outs)
res["someone_waited"] = any(o[2]["t_admit"] > o[2]["t_submit"] + 1e-4 for o in outs)
res["levels"] = [o[2]["levels_done"] for o in outs] == [len(P.iterations) for _, P in reqs]
res["resident_zero_after"] = st["bytes_resident"] == 0 and st["completed"] == 4
# each request's fields are the oracle's registration
ok = True
for ((f, m, g), P), (fwd, inv, info) in zip(reqs, outs):
    rf, ri, _, _ = O.syn_register(f, g, m, g, P)
    ok = ok and np.array_equal(np.moveaxis(fwd, -1, 0), rf) and np.array_equal(np.moveaxis(inv, -1, 0), ri)
res["fields_equal_oracle"] = bool(ok)
# a request above the budget is refused at submission
(f, m, g), P = reqs[0]
with Server(hbm_budget_bytes=fps[0] - 1) as srv:
    try:
        srv.submit(P, f, g, m, g)
        res["oversize_refused"] = False
    except SynxError as e:
        res["oversize_refused"] = "budget" in str(e)
# the resident limit, and pooled contexts reused by later requests with the same parameters
before = lib.host_stage_created()
with Server(max_active=1) as srv:
    ids = [srv.submit(P, f, g, m, g) for _ in range(3)]
    outs = [srv.wait(i, timeout=600) for i in ids]
    st = srv.stats()
res["limit_all_done"] = st["completed"] == 3 and all(o[2]["status"] == 2 for o in outs)
res["one_context_for_three"] = lib.host_stage_created() - before == 1
res["same_bits"] = bool(np.array_equal(outs[0][0], outs[2][0]))
res["pooled_after"] = st["bytes_pooled"] == fps[0]
print(json.dumps(res))
"""


def test_serving_loop_logic(host_lib, tmp_path):
    script = tmp_path / "drive.py"
    script.write_text(f"ROOT = {ROOT!r}\nSO = {host_lib!r}\n" + DRIVER)
    r = subprocess.run([sys.executable, str(script)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, (r.stdout + r.stderr)[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert all(res.values()), res
