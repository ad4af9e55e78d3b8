"""Whole-stage parity: the CUDA SyN stage (through the C ABI, host buffers in and out)
against the CPU oracle on seeded phantom pairs.

* One iteration from zero fields: the four half-fields must agree to 1e-4 mm.
* A multi-level schedule: the per-iteration metric log agrees to 2e-3 and the final forward
  and inverse fields agree to an RMS of 0.05 voxel (the stage-level tolerance).  Exact
  agreement is not expected over many iterations: the fixed-point inverse stops on
  `mean > 0.001` / `max > 0.1`, and a rounding-level difference can change its iteration count
  (the same holds between the reference's float and double builds).
* Graph replay and plain launches give identical bits; repeated runs are deterministic.
"""
import numpy as np
import pytest

import oracle as O
from ants_b200 import phantoms
from ants_b200.synx import (SYNX_F_INV_TWO_PASS, SYNX_F_NO_PDL, SYNX_F_NO_PERSISTENT, SYNX_F_SMOOTH_TWO_PASS,
                            SYNX_F_USE_GRAPHS, Geom, SyNParams, SyNStage)

pytestmark = pytest.mark.gpu


def planes(interleaved: np.ndarray) -> np.ndarray:
    return np.moveaxis(interleaved, -1, 0)


def rms_vox(a: np.ndarray, b: np.ndarray, spacing) -> float:
    sp = np.asarray(spacing, dtype=np.float64).reshape((-1,) + (1,) * (a.ndim - 1))
    return float(np.sqrt((((a - b) / sp) ** 2).sum(0).mean()))


def make_pair(dim, size, seed):
    return phantoms.pair_2d(size, seed=seed) if dim == 2 else phantoms.pair_3d(size, seed=seed)


@pytest.mark.parametrize("dim,size,radius,sigma", [(2, (64, 64), 2, 1.0), (3, (32, 30, 28), 4, 1.0),
                                                   (3, (31, 33, 27), 2, 0.0)])
def test_single_iteration_half_fields(cuda, dim, size, radius, sigma):
    f, m = make_pair(dim, size, seed=1)
    g = Geom(size)
    P = SyNParams(dim=dim, cc_radius=radius, iterations=(1,), shrink_factors=(1,), smoothing_sigmas=(sigma,))
    with SyNStage(P) as st:
        st.set_images(f, g, m, g)
        st.run()
        got = [planes(a) for a in st.half_fields()]
        log = st.log()
    fp, mp = O.preprocess(f), O.preprocess(m)
    Fs, Ms = O.smooth_image(fp, g, sigma), O.smooth_image(mp, g, sigma)
    z = np.zeros((dim,) + g.shape, np.float32)
    v, ref, kinv = O.syn_iteration(Fs, g, Ms, g, P, g, z, z, z, z)
    assert len(log) == 1 and abs(log[0].metric - v) < 1e-7
    assert log[0].inverse_iterations == kinv
    for a, b in zip(got, ref):
        np.testing.assert_allclose(a, b, atol=1e-4, rtol=0)


SCHEDULES = [
    (2, (96, 96), 2, (30, 15, 8), (4, 2, 1), (2.0, 1.0, 0.0)),
    (3, (40, 44, 36), 4, (12, 6), (2, 1), (1.0, 0.0)),
]


# "persistent": levels that fit run as one cooperative kernel per level (the default);
# "kernels": the same levels as one launch per phase (SYNX_F_NO_PERSISTENT)
PATHS = {"persistent": SYNX_F_USE_GRAPHS, "kernels": SYNX_F_USE_GRAPHS | SYNX_F_NO_PERSISTENT}


@pytest.mark.parametrize("path", sorted(PATHS))
@pytest.mark.parametrize("dim,size,radius,iters,shrink,sigmas", SCHEDULES)
def test_multilevel_matches_oracle(cuda, dim, size, radius, iters, shrink, sigmas, path):
    f, m = make_pair(dim, size, seed=7)
    g = Geom(size)
    P = SyNParams(dim=dim, cc_radius=radius, iterations=iters, shrink_factors=shrink, smoothing_sigmas=sigmas,
                  convergence_threshold=1e-12, flags=PATHS[path])
    with SyNStage(P) as st:
        st.set_images(f, g, m, g)
        st.run()
        fwd, inv = (planes(a) for a in st.fields())
        go = st.output_geom()
        log = st.log()
    rf, ri, rg, rlog = O.syn_register(f, g, m, g, P)
    assert go.size == rg.size
    assert [(r.level, r.iteration) for r in log] == [(r["level"], r["iteration"]) for r in rlog]
    np.testing.assert_allclose([r.metric for r in log], [r["metric"] for r in rlog], atol=2e-3)
    assert rms_vox(fwd, rf, go.spacing) <= 0.05
    assert rms_vox(inv, ri, go.spacing) <= 0.05
    # the registration did something: the final fields are well away from zero
    assert rms_vox(fwd, np.zeros_like(fwd), go.spacing) > 0.02


@pytest.mark.parametrize("dim,size,uvar,tvar", [(2, (72, 70), 0.25, 0.5), (3, (30, 32, 28), 2.0, 1.0)])
def test_total_field_smoothing_and_blend(cuda, dim, size, uvar, tvar):
    # SyN[eta, varU, varT] with varT > 0 smooths the composed total field; varU < 0.5 blends
    f, m = make_pair(dim, size, seed=9)
    g = Geom(size)
    P = SyNParams(dim=dim, cc_radius=2, learning_rate=0.2, update_variance=uvar, total_variance=tvar,
                  iterations=(6, 3), shrink_factors=(2, 1), smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12)
    with SyNStage(P) as st:
        st.set_images(f, g, m, g)
        st.run()
        fwd, inv = (planes(a) for a in st.fields())
        go = st.output_geom()
        log = st.log()
    rf, ri, rg, rlog = O.syn_register(f, g, m, g, P)
    np.testing.assert_allclose([r.metric for r in log], [r["metric"] for r in rlog], atol=2e-3)
    assert rms_vox(fwd, rf, go.spacing) <= 0.05
    assert rms_vox(inv, ri, go.spacing) <= 0.05


@pytest.mark.parametrize("persistent", [True, False])
def test_graph_replay_is_bit_identical_and_deterministic(cuda, persistent):
    # graph replay (with the fixed-point inverse loops as conditional graph nodes on the
    # per-kernel path) gives the same bits as plain launches, run after run
    f, m = make_pair(3, (36, 34, 32), seed=3)
    g = Geom((36, 34, 32))
    base = 0 if persistent else SYNX_F_NO_PERSISTENT
    outs = []
    for flags in (base, base | SYNX_F_USE_GRAPHS, base | SYNX_F_USE_GRAPHS):
        P = SyNParams(dim=3, cc_radius=3, iterations=(6, 4), shrink_factors=(2, 1), smoothing_sigmas=(1.0, 0.0),
                      flags=flags)
        with SyNStage(P) as st:
            st.set_images(f, g, m, g)
            st.run()
            outs.append((st.fields(), [(r.metric, r.inverse_iterations) for r in st.log()]))
    for o in outs[1:]:
        np.testing.assert_array_equal(o[0][0], outs[0][0][0])
        np.testing.assert_array_equal(o[0][1], outs[0][0][1])
        assert o[1] == outs[0][1]
    # the cold-started first inversions take several sub-iterations: the loops really iterate
    assert max(k for _, k in outs[0][1]) > 4


@pytest.mark.parametrize("dim,size,radius", [(2, (80, 66), 1), (2, (50, 61), 7), (3, (26, 23, 29), 5)])
def test_persistent_level_radii_and_repeatability(cuda, dim, size, radius):
    # odd sizes and the extreme CC radii through the persistent level kernel; two runs give the
    # same bits (its reductions are ordered), and both agree with the per-phase launches
    f, m = make_pair(dim, size, seed=11)
    g = Geom(size)
    outs = []
    for flags in (PATHS["persistent"], PATHS["persistent"], PATHS["kernels"]):
        P = SyNParams(dim=dim, cc_radius=radius, iterations=(8, 5), shrink_factors=(2, 1),
                      smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12, flags=flags)
        with SyNStage(P) as st:
            st.set_images(f, g, m, g)
            st.run()
            outs.append((st.fields(), [r.metric for r in st.log()], st.output_geom()))
    np.testing.assert_array_equal(outs[0][0][0], outs[1][0][0])
    np.testing.assert_array_equal(outs[0][0][1], outs[1][0][1])
    assert outs[0][1] == outs[1][1]
    np.testing.assert_allclose(outs[0][1], outs[2][1], atol=2e-3)
    sp = outs[0][2].spacing
    for a, b in zip(outs[0][0], outs[2][0]):
        assert rms_vox(planes(a), planes(b), sp) <= 0.05


@pytest.mark.parametrize("path", sorted(PATHS))
def test_convergence_stops_level_early(cuda, path):
    # a pair that is already aligned stops as soon as the window fills (slope >= 0)
    f, _ = make_pair(2, (64, 64), seed=5)
    g = Geom((64, 64))
    P = SyNParams(dim=2, cc_radius=2, iterations=(40,), shrink_factors=(1,), smoothing_sigmas=(0.0,),
                  convergence_threshold=1e-6, convergence_window=10, flags=PATHS[path])
    with SyNStage(P) as st:
        st.set_images(f, g, f, g)
        st.run()
        log = st.log()
    rf, ri, rg, rlog = O.syn_register(f, g, f, g, P)
    assert len(log) == len(rlog) < 40


def test_run_level_order_enforced(cuda):
    f, m = make_pair(2, (32, 32), seed=2)
    g = Geom((32, 32))
    P = SyNParams(dim=2, cc_radius=2, iterations=(2, 2), shrink_factors=(2, 1), smoothing_sigmas=(0.0, 0.0))
    from ants_b200.synx import SynxError
    with SyNStage(P) as st:
        st.set_images(f, g, m, g)
        with pytest.raises(SynxError):
            st.run_level(1)
        st.run_level(0)
        st.run_level(1)
        assert st.output_geom().size == (32, 32)


@pytest.mark.parametrize("rows", [8, 16])
@pytest.mark.parametrize("uvar", [3.0, 0.3, 8.0])
def test_slab_smoothing_matches_two_pass_bit_for_bit(cuda, uvar, rows):
    # the fused slab smoothing (xy and z in one kernel, a tuning-table option) and the two-kernel path
    # through a temporary (the default) do the same arithmetic in the same order: whole registrations
    # agree bit for bit
    f, m = make_pair(3, (41, 37, 33), seed=13)
    g = Geom((41, 37, 33))
    outs = []
    for tile_rows, extra in ((rows, 0), (rows, SYNX_F_SMOOTH_TWO_PASS)):
        P = SyNParams(dim=3, cc_radius=3, update_variance=uvar, iterations=(5, 3), shrink_factors=(2, 1),
                      smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12, smooth_tile_rows=tile_rows,
                      flags=SYNX_F_USE_GRAPHS | SYNX_F_NO_PERSISTENT | extra)
        with SyNStage(P) as st:
            st.set_images(f, g, m, g)
            st.run()
            outs.append((st.fields(), [r.metric for r in st.log()]))
    np.testing.assert_array_equal(outs[0][0][0], outs[1][0][0])
    np.testing.assert_array_equal(outs[0][0][1], outs[1][0][1])
    assert outs[0][1] == outs[1][1]


@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("dim,size", [(3, (38, 35, 31)), (2, (90, 77))])
def test_single_pass_inverse_matches_two_pass_bit_for_bit(cuda, dim, size, graphs):
    # the single-pass fixed-point inverse (residual, statistics and update in one pass; clamped voxels
    # deferred to a short pass over a list) performs the two-pass form's operations on the same values:
    # whole registrations agree bit for bit, including the cold-started first inversions that iterate
    f, m = make_pair(dim, size, seed=19)
    g = Geom(size)
    outs = []
    for extra in (0, SYNX_F_INV_TWO_PASS):
        P = SyNParams(dim=dim, cc_radius=3 if dim == 3 else 2, iterations=(6, 4), shrink_factors=(2, 1),
                      smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12,
                      flags=(SYNX_F_USE_GRAPHS if graphs else 0) | SYNX_F_NO_PERSISTENT | extra)
        with SyNStage(P) as st:
            st.set_images(f, g, m, g)
            st.run()
            outs.append((st.fields(), [(r.metric, r.inverse_iterations) for r in st.log()]))
    np.testing.assert_array_equal(outs[0][0][0], outs[1][0][0])
    np.testing.assert_array_equal(outs[0][0][1], outs[1][0][1])
    assert outs[0][1] == outs[1][1]
    assert max(k for _, k in outs[0][1]) > 4  # some inversions iterate more than once


@pytest.mark.parametrize("rows", [-2, -3])
@pytest.mark.parametrize("uvar", [3.0, 0.3])
def test_pipelined_xy_smoothing_matches_bit_for_bit(cuda, uvar, rows):
    # the pipelined xy kernel (double-buffered halo tiles over chunks of slices) does the xy kernel's
    # arithmetic: whole registrations agree bit for bit with the plain xy kernel
    f, m = make_pair(3, (43, 71, 29), seed=23)
    g = Geom((43, 71, 29))
    outs = []
    for tile_rows in (rows, -1):
        P = SyNParams(dim=3, cc_radius=3, update_variance=uvar, iterations=(5, 3), shrink_factors=(2, 1),
                      smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12, smooth_tile_rows=tile_rows,
                      flags=SYNX_F_USE_GRAPHS | SYNX_F_NO_PERSISTENT)
        with SyNStage(P) as st:
            st.set_images(f, g, m, g)
            st.run()
            outs.append((st.fields(), [r.metric for r in st.log()]))
    np.testing.assert_array_equal(outs[0][0][0], outs[1][0][0])
    np.testing.assert_array_equal(outs[0][0][1], outs[1][0][1])
    assert outs[0][1] == outs[1][1]


@pytest.mark.parametrize("graphs", [True, False])
def test_programmatic_dependent_launch_changes_nothing(cuda, graphs):
    # an iteration's kernels launched with programmatic dependent launch (the default) and without it
    # give the same bits, in captured graphs (inverse loops as conditional nodes) and in plain launches
    f, m = make_pair(3, (44, 39, 35), seed=29)
    g = Geom((44, 39, 35))
    outs = []
    for extra in (0, SYNX_F_NO_PDL):
        P = SyNParams(dim=3, cc_radius=3, iterations=(6, 4), shrink_factors=(2, 1), smoothing_sigmas=(1.0, 0.0),
                      convergence_threshold=1e-12,
                      flags=(SYNX_F_USE_GRAPHS if graphs else 0) | SYNX_F_NO_PERSISTENT | extra)
        with SyNStage(P) as st:
            st.set_images(f, g, m, g)
            st.run()
            outs.append((st.fields(), [(r.metric, r.inverse_iterations) for r in st.log()]))
    np.testing.assert_array_equal(outs[0][0][0], outs[1][0][0])
    np.testing.assert_array_equal(outs[0][0][1], outs[1][0][1])
    assert outs[0][1] == outs[1][1]
