"""The command lines' own logic, on a machine without a GPU.

The real sources of antsApplyTransforms_b200 and antsRegistrationSyN_b200 are compiled against
host stand-ins for the device (tests/cli_host/: host CUDA runtime calls, and the step and stage
entry points routed to the CPU oracle), then run through the same checks as their GPU tests:
transform chains in the reference's order, linear transforms folded into grid geometry, the
collapsed field, initial moving transforms, output file names and written transforms, and the
bit-exact agreement of the two programs' warped images.  What this covers is the programs'
plumbing; the kernels' parity is the GPU tests'.  The stand-ins are test infrastructure: the
product's command lines link libsynx.so and fail without a GPU.
"""
import os
import shutil
import subprocess

import pytest

import test_apply_transforms as A
import test_zz_stack_apply as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "ants_b200", "csrc")
HOST = os.path.join(ROOT, "tests", "cli_host")


@pytest.fixture(scope="module")
def host_cli(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    out = tmp_path_factory.mktemp("cli_host")
    common = ["g++", "-std=c++17", "-O2", "-fopenmp", "-I", HOST, "-I", os.path.join(ROOT, "include"), "-I", CSRC,
              "-I", os.path.join(ROOT, "oracle")]
    libs = [os.path.join(CSRC, "nifti_io.cpp"), os.path.join(CSRC, "synx_linear.cpp"),
            os.path.join(HOST, "host_steps.cpp"), os.path.join(ROOT, "oracle", "synx_oracle_capi.cpp"), "-lz"]
    exes = {}
    for name, src, extra in (("apply", "ants_apply_transforms.cpp", []),
                             ("reg", "ants_registration.cpp", [os.path.join(HOST, "host_stage.cpp")])):
        exe = str(out / name)
        r = subprocess.run(common + ["-o", exe, os.path.join(CSRC, src)] + extra + libs, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-3000:]
        exes[name] = exe
    return exes


@pytest.mark.parametrize("dim", [2, 3])
def test_transform_stacks(host_cli, tmp_path, dim):
    S.check_stacks_match_the_scheme(host_cli["apply"], tmp_path, dim)


def test_default_value(host_cli, tmp_path):
    A.check_default_value_outside(host_cli["apply"], tmp_path)


def test_warped_output_matches_antsapplytransforms(host_cli, tmp_path):
    A.check_reproduces_the_registration_output(host_cli["reg"], host_cli["apply"], tmp_path)


def test_initial_moving_transform(host_cli, tmp_path):
    S.check_initial_moving_transform(host_cli["reg"], host_cli["apply"], tmp_path)


def test_derived_initial_translation(host_cli, tmp_path):
    S.check_derived_initial_translation(host_cli["reg"], tmp_path)


@pytest.mark.parametrize("interp", ["NearestNeighbor", "GenericLabel", "GenericLabel[Linear]"])
@pytest.mark.parametrize("dim", [2, 3])
def test_label_interpolation(host_cli, tmp_path, dim, interp):
    S.check_label_interpolation(host_cli["apply"], tmp_path, dim, interp)


def test_multichannel(host_cli, tmp_path):
    S.check_multichannel(host_cli["apply"], tmp_path)


def test_time_series(host_cli, tmp_path):
    S.check_time_series(host_cli["apply"], tmp_path)


def test_output_types(host_cli, tmp_path):
    S.check_output_types(host_cli["apply"], tmp_path)


def test_output_precision(host_cli, tmp_path):
    S.check_output_precision(host_cli["reg"], tmp_path)


def test_histogram_matching(host_cli, tmp_path):
    import numpy as np

    import oracle as O
    import test_zz_u_histogram_match_gpu as H

    def stage_fields(f, gf, m, gm, P):
        fwd, inv, _, _ = O.syn_register(f, gf, m, gm, P)
        return np.moveaxis(fwd, 0, -1), np.moveaxis(inv, 0, -1)

    H.check_cli_histogram_matching(host_cli["reg"], tmp_path, stage_fields)


def test_masks(host_cli, tmp_path):
    import numpy as np

    import oracle as O
    import test_zz_t_masks as X

    def stage_fields(f, gf, m, gm, P, mf, mm):
        fwd, inv, _, _ = O.syn_register(f, gf, m, gm, P, fixed_mask=mf, fixed_mask_geom=gf, moving_mask=mm,
                                        moving_mask_geom=gm)
        return np.moveaxis(fwd, 0, -1), np.moveaxis(inv, 0, -1)

    X.check_cli_masks(host_cli["reg"], tmp_path, stage_fields)


def test_state_and_composite(host_cli, tmp_path):
    import oracle as O
    import test_zz_u_state as U

    def stage(f, gf, m, gm, P, init):
        kw = {}
        if init is not None:
            kw = dict(initial_half_fields=[U.planes(a) for a in init], initial_geom=gf)
        fwd, inv, _, _, half = O.syn_register(f, gf, m, gm, P, return_half_fields=True, **kw)
        return U.interleaved(fwd), U.interleaved(inv), [U.interleaved(h) for h in half]

    U.check_cli_state(host_cli["reg"], tmp_path, stage)
