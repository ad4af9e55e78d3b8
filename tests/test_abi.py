"""The C ABI library loads, exports every symbol include/synx.h declares, and its host-only
entry points (no GPU needed) agree with the oracle and reject bad input loudly."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle as O
from ants_b200 import synx
from ants_b200.synx import Geom, SyNParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "synx.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(synx_\w+)\s*\(", text, re.M)))


def test_header_declares_the_abi():
    syms = declared_symbols()
    for s in ("synx_create", "synx_set_images", "synx_run", "synx_run_level", "synx_get_fields", "synx_get_log",
              "synx_destroy", "synx_last_error", "synx_cc_metric", "synx_invert_field"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = synx.load_library()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_params_default_matches_antsregistration_defaults():
    lib = synx.load_library()
    p = synx.SynxParams()
    assert lib.synx_params_default(C.byref(p), 3) == 0
    assert (p.learning_rate, p.update_variance, p.total_variance, p.cc_radius) == (0.1, 3.0, 0.0, 4)
    assert (p.convergence_threshold, p.convergence_window) == (1e-6, 10)
    assert (p.inv_max_iter, p.inv_mean_tol, p.inv_max_tol) == (20, 0.001, 0.1)


def test_params_reject_bad_dim():
    lib = synx.load_library()
    p = synx.SynxParams()
    assert lib.synx_params_default(C.byref(p), 4) == -1
    assert b"dim" in lib.synx_last_error(None)


def test_gaussian_kernel_matches_oracle():
    for var, err, w in ((3.0, 0.001, 200), (9.0, 0.01, 32), (0.4, 0.001, 5), (0.0, 0.01, 32)):
        np.testing.assert_array_equal(synx.gaussian_kernel(var, err, w), O.gaussian_kernel(var, err, w))


def test_shrink_geom_matches_oracle():
    for g in (Geom((182, 218, 182)), Geom((100, 100, 40), (1.0, 1.0, 2.5), (5.0, -3.0, 2.0)),
              Geom((256, 256), (0.7, 0.7))):
        for f in (1, 2, 3, 4, 8):
            a, b = synx.shrink_geom(g, f), O.shrink_geom(g, f)
            assert a.size == b.size and a.spacing == b.spacing
            np.testing.assert_allclose(a.origin, b.origin, atol=1e-12)


def test_create_fails_loudly_without_gpu_or_with_bad_params():
    # bad parameters are rejected before any device is touched
    with pytest.raises(synx.SynxError):
        synx.SyNStage(SyNParams(dim=3, cc_radius=99))
    with pytest.raises(synx.SynxError):
        synx.SyNStage(SyNParams(dim=3, iterations=(1, 2), shrink_factors=(1, 1), smoothing_sigmas=(0, 0),
                                learning_rate=-1))
    with pytest.raises(ValueError):
        SyNParams(dim=3, iterations=(1, 2), shrink_factors=(1,), smoothing_sigmas=(0,)).to_c()


def test_step_calls_reject_null_pointers():
    lib = synx.load_library()
    g = Geom((8, 8)).to_c()
    v = C.c_double()
    assert lib.synx_cc_metric(None, None, C.byref(g), 2, None, None, C.byref(v), None) == -1
    assert lib.synx_invert_field(None, None, C.byref(g), 20, 0.001, 0.1, None, None) == -1
    assert lib.synx_batch_step(None, None, 0, None, None) == -1
    assert lib.synx_batch_run(None, None, 0, None) == -1


def test_footprint_without_a_gpu():
    # the device bytes a stage would hold are computed on the host
    from ants_b200.synx import Geom, SyNParams, footprint
    P = SyNParams(dim=3, cc_radius=4, iterations=(100, 70, 50, 20), shrink_factors=(8, 4, 2, 1),
                  smoothing_sigmas=(3.0, 2.0, 1.0, 0.0))
    big = footprint(P, Geom((182, 218, 182)), Geom((182, 218, 182)))
    small = footprint(P, Geom((91, 109, 91)), Geom((91, 109, 91)))
    n = 182 * 218 * 182
    # 4 half-fields + 6 work fields of 3 components, 2 warped images, 5 image buffers: 37 floats/voxel,
    # plus the inverse's two deferred-voxel lists (2 ints) and the metric-mask validity (1 byte)
    per_voxel = 37 * 4 + 2 * 4 + 1
    assert per_voxel * n <= big < per_voxel * n * 1.05
    assert small < big / 7
