"""Batched pairs (synx_batch_*): every pair of a batch gives the same bits as the same pair
registered alone, whatever else is in the batch, at whatever level the others are.

The level kernel decomposes a level into tiles that depend on the level grid only, and every
reduction runs over those tiles in a fixed order, so a pair's group of blocks can be any size.
"""
import numpy as np
import pytest

from ants_b200 import phantoms
from ants_b200.synx import Batch, Geom, SyNParams, SyNStage

pytestmark = pytest.mark.gpu


def pair(dim, size, seed):
    return phantoms.pair_2d(size, seed=seed) if dim == 2 else phantoms.pair_3d(size, seed=seed)


def params(dim, **kw):
    base = dict(dim=dim, cc_radius=2 if dim == 2 else 4, iterations=(12, 6, 3), shrink_factors=(4, 2, 1),
                smoothing_sigmas=(2.0, 1.0, 0.0), convergence_threshold=1e-12)
    base.update(kw)
    return SyNParams(**base)


CASES = [(2, (96, 80), 1), (2, (64, 70), 2), (3, (40, 36, 44), 3), (2, (128, 112), 4), (3, (33, 41, 29), 5)]


def alone(dim, size, seed, P):
    f, m = pair(dim, size, seed)
    g = Geom(size)
    with SyNStage(P) as st:
        st.set_images(f, g, m, g)
        st.run()
        fw, iv = st.fields()
        return fw.copy(), iv.copy(), [(r.level, r.iteration, r.metric, r.inverse_iterations) for r in st.log()]


def make_stage(dim, size, seed, P):
    f, m = pair(dim, size, seed)
    g = Geom(size)
    st = SyNStage(P)
    st.set_images(f, g, m, g)
    return st


def result(st):
    fw, iv = st.fields()
    return fw.copy(), iv.copy(), [(r.level, r.iteration, r.metric, r.inverse_iterations) for r in st.log()]


def assert_same(a, b):
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert a[2] == b[2]


def test_batch_equals_alone(cuda):
    refs = [alone(d, s, k, params(d)) for d, s, k in CASES]
    stages = [make_stage(d, s, k, params(d)) for d, s, k in CASES]
    with Batch() as b:
        b.run(stages)
    for st, ref in zip(stages, refs):
        assert_same(result(st), ref)
        st.close()


def test_batch_with_pairs_at_different_levels(cuda):
    # two pairs start one level ahead; a third pair joins two steps late (as a serving loop admits it)
    refs = [alone(d, s, k, params(d)) for d, s, k in CASES[:4]]
    stages = [make_stage(d, s, k, params(d)) for d, s, k in CASES[:4]]
    stages[0].run_level(0)
    stages[2].run_level(0)
    with Batch() as b:
        assert b.step(stages[:3]) == 3
        assert b.step(stages[:3]) == 3
        assert b.step(stages) == 2  # stages 0 and 2 are done; 1 runs its last level, 3 its first
        b.run(stages)
        assert b.step(stages) == 0
    for st, ref in zip(stages, refs):
        assert_same(result(st), ref)
        st.close()


def test_batch_of_many_small_pairs(cuda):
    # more pairs than SMs: groups of one or two blocks
    P = params(2, iterations=(6, 4), shrink_factors=(2, 1), smoothing_sigmas=(1.0, 0.0))
    cases = [(2, (40 + 3 * i, 36 + 5 * (i % 7)), 100 + i) for i in range(160)]
    stages = [make_stage(d, s, k, P) for d, s, k in cases]
    with Batch() as b:
        b.run(stages)
    for i in (0, 57, 159):
        assert_same(result(stages[i]), alone(*cases[i], P))
    for st in stages:
        st.close()


def test_batch_runs_large_levels_on_the_per_kernel_path(cuda):
    # a level above the level kernel's size limit runs its own kernels inside the batch step
    P = params(2, persistent_max_voxels=3000)
    refs = [alone(d, s, k, P) for d, s, k in CASES[:2]]
    stages = [make_stage(d, s, k, P) for d, s, k in CASES[:2]]
    with Batch() as b:
        b.run(stages)
    for st, ref in zip(stages, refs):
        assert_same(result(st), ref)
        st.close()


def test_batch_argument_errors(cuda):
    from ants_b200.synx import SynxError
    st = SyNStage(params(2))
    with Batch() as b:
        with pytest.raises(SynxError):
            b.step([st])  # images not set
        f, m = pair(2, (32, 32), 1)
        st.set_images(f, Geom((32, 32)), m, Geom((32, 32)))
        with pytest.raises(SynxError):
            b.step([st, st])  # listed twice
    st.close()
