"""Failure detection without a GPU fault: every grid-barrier wait of the level kernel is bounded.
The injection makes the barrier wait for a block that was never launched; the wait runs out, the
kernel ends, the stage reports the timeout, and the GPU keeps working."""
import time

import numpy as np
import pytest

from ants_b200 import phantoms
from ants_b200.synx import SYNX_INJECT_BARRIER_TIMEOUT, Geom, SyNParams, SyNStage, SynxError

pytestmark = pytest.mark.gpu


def params(inject):
    return SyNParams(dim=2, cc_radius=2, iterations=(5,), shrink_factors=(1,), smoothing_sigmas=(0.0,),
                     convergence_threshold=1e-12, test_inject=inject)


def test_barrier_timeout_is_reported_and_the_gpu_stays_usable(cuda):
    f, m = phantoms.pair_2d((64, 60), seed=8)
    g = Geom((64, 60))
    with SyNStage(params(SYNX_INJECT_BARRIER_TIMEOUT)) as st:
        st.set_images(f, g, m, g)
        t0 = time.perf_counter()
        with pytest.raises(SynxError, match="barrier"):
            st.run()
        assert time.perf_counter() - t0 < 20.0
    with SyNStage(params(0)) as st:
        st.set_images(f, g, m, g)
        st.run()
        fw, _ = st.fields()
        assert len(st.log()) == 5 and np.isfinite(fw).all()


def test_unknown_injection_is_rejected():
    with pytest.raises(SynxError):
        SyNStage(params(7))
