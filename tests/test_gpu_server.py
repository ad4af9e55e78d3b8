"""Serving loop (synx_server_*): admission by device footprint, continuous batching, and the
same result alone and in a mix of uneven 2-D/3-D requests."""
import time

import numpy as np
import pytest

from ants_b200 import phantoms
from ants_b200.synx import Geom, Server, SyNParams, SyNStage, SynxError, footprint

pytestmark = pytest.mark.gpu


def params(dim):
    return SyNParams(dim=dim, cc_radius=2 if dim == 2 else 4, iterations=(10, 6, 3), shrink_factors=(4, 2, 1),
                     smoothing_sigmas=(2.0, 1.0, 0.0), convergence_threshold=1e-12)


MIX = [(2, (128, 112), 11), (3, (48, 40, 44), 12), (2, (96, 100), 13), (3, (36, 52, 40), 14), (2, (160, 150), 15),
       (3, (44, 44, 44), 16)]


def make(dim, size, seed):
    f, m = phantoms.pair_2d(size, seed=seed) if dim == 2 else phantoms.pair_3d(size, seed=seed)
    return f, m, Geom(size)


def alone(dim, size, seed):
    f, m, g = make(dim, size, seed)
    with SyNStage(params(dim)) as st:
        st.set_images(f, g, m, g)
        st.run()
        fw, iv = st.fields()
        return fw.copy(), iv.copy()


def test_request_same_alone_and_in_mix(cuda):
    target = MIX[1]
    ref = alone(*target)
    f, m, g = make(*target)
    with Server() as srv:
        rid = srv.submit(params(target[0]), f, g, m, g)
        fw_a, iv_a, info = srv.wait(rid, timeout=120)
        assert info["status"] == 2 and info["levels_done"] == 3
        # the same request among others that arrive around it
        ids = []
        for k, (d, s, seed) in enumerate(MIX):
            ff, mm, gg = make(d, s, seed)
            ids.append(srv.submit(params(d), ff, gg, mm, gg))
            if k == 2:
                time.sleep(0.01)
        outs = [srv.wait(i, timeout=300) for i in ids]
        st = srv.stats()
    np.testing.assert_array_equal(fw_a, ref[0])
    np.testing.assert_array_equal(iv_a, ref[1])
    np.testing.assert_array_equal(outs[1][0], ref[0])
    np.testing.assert_array_equal(outs[1][1], ref[1])
    for (d, s, seed), (fw, iv, info) in zip(MIX, outs):
        assert info["status"] == 2 and info["t_done"] >= info["t_admit"] >= info["t_submit"]
    assert st["completed"] == 1 + len(MIX) and st["failed"] == 0 and st["bytes_resident"] == 0


def test_admission_respects_the_budget(cuda):
    reqs = [make(*c) for c in MIX[:4]]
    fps = [footprint(params(c[0]), r[2], r[2]) for c, r in zip(MIX[:4], reqs)]
    budget = max(fps) + min(fps)  # never more than two of these resident at once
    with Server(hbm_budget_bytes=budget) as srv:
        ids = [srv.submit(params(c[0]), r[0], r[2], r[1], r[2]) for c, r in zip(MIX[:4], reqs)]
        infos = [srv.wait(i, timeout=300)[2] for i in ids]
        st = srv.stats()
    assert st["bytes_peak"] <= budget
    assert all(i["status"] == 2 for i in infos)
    assert any(i["t_admit"] > i["t_submit"] + 1e-4 for i in infos)  # someone waited for memory
    for c, i, fp in zip(MIX[:4], infos, fps):
        assert i["device_bytes"] == fp


def test_footprint_matches_allocation(cuda):
    for c in MIX[:2]:
        f, m, g = make(*c)
        with SyNStage(params(c[0])) as st:
            st.set_images(f, g, m, g)
            assert st.device_bytes() == footprint(params(c[0]), g, g)


def test_oversize_request_rejected_and_resident_limit(cuda):
    f, m, g = make(*MIX[0])
    with Server(hbm_budget_bytes=1 << 20) as srv:
        with pytest.raises(SynxError):
            srv.submit(params(2), f, g, m, g)
    with Server(max_active=1) as srv:
        ids = [srv.submit(params(2), f, g, m, g) for _ in range(3)]
        outs = [srv.wait(i, timeout=300) for i in ids]
        st = srv.stats()
    np.testing.assert_array_equal(outs[0][0], outs[2][0])
    assert st["completed"] == 3


def test_pooled_context_reuse_gives_the_same_bits(cuda):
    # a small 3-D request reuses the arena a larger one left in the pool; then the larger one
    # cannot reuse the smaller arena and gets a new context
    big, small = MIX[5], MIX[1]
    refs = {c: alone(*c) for c in (big, small)}
    with Server() as srv:
        for c in (big, small, big, small):
            f, m, g = make(*c)
            fw, iv, info = srv.wait(srv.submit(params(c[0]), f, g, m, g), timeout=300)
            np.testing.assert_array_equal(fw, refs[c][0])
            np.testing.assert_array_equal(iv, refs[c][1])
        st = srv.stats()
    assert st["bytes_pooled"] > 0 and st["bytes_resident"] == 0
