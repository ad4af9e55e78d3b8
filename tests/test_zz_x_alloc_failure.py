"""Failure detection without a GPU fault: a device allocation that fails.  The injection makes the
context's arena allocation report failure on the host, without calling the device allocator;
synx_set_images returns SYNX_E_NOMEM, the context is destroyed normally and the next stage on the
same GPU runs.  This file is collected last, after the tests already verified on the device."""
import numpy as np
import pytest

from ants_b200 import phantoms
from ants_b200.synx import SYNX_INJECT_ALLOC_FAILURE, Geom, SyNParams, SyNStage, SynxError

pytestmark = pytest.mark.gpu


def params(inject):
    return SyNParams(dim=2, cc_radius=2, iterations=(5,), shrink_factors=(1,), smoothing_sigmas=(0.0,),
                     convergence_threshold=1e-12, test_inject=inject)


def test_allocation_failure_is_reported_and_the_gpu_stays_usable(cuda):
    f, m = phantoms.pair_2d((64, 60), seed=8)
    g = Geom((64, 60))
    with SyNStage(params(SYNX_INJECT_ALLOC_FAILURE)) as st:
        with pytest.raises(SynxError, match="out of device memory"):
            st.set_images(f, g, m, g)
        with pytest.raises(SynxError):
            st.run()  # nothing was set up
    with SyNStage(params(0)) as st:
        st.set_images(f, g, m, g)
        st.run()
        fw, _ = st.fields()
        assert len(st.log()) == 5 and np.isfinite(fw).all()
