"""Precision variants: CC window sums in double (the default) vs float, and half-precision
storage of the half-fields, each against the double-precision oracle."""
import numpy as np
import pytest
import torch

import oracle as O
from ants_b200 import phantoms
from ants_b200.synx import SYNX_F_FIELDS_FP16, SYNX_F_USE_GRAPHS, Geom, SyNParams, SyNStage, cc_metric

pytestmark = pytest.mark.gpu


def twelve_bit(a):
    a = a.astype(np.float64)
    return ((a - a.min()) / (a.max() - a.min()) * 4095.0).astype(np.float32)


def test_cc_sums_on_12bit_intensities(cuda):
    size = (48, 44, 40)
    f, m = phantoms.pair_3d(size, seed=21)
    f, m = twelve_bit(f), twelve_bit(m)
    g = Geom(size, spacing=(0.7, 0.7, 0.7))
    v64, gF64, gM64, _ = O.cc_metric(f, m, g, 5, dtype=np.float64)
    F, M = torch.from_numpy(f).cuda(), torch.from_numpy(m).cuda()
    errs = {}
    for fp32 in (False, True):
        gF = torch.empty((3,) + g.shape, device="cuda")
        gM = torch.empty_like(gF)
        v = cc_metric(F, M, g, 5, gF, gM, fp32_sums=fp32)
        rel = [float(np.sqrt(((a.cpu().numpy() - b) ** 2).mean() / (b ** 2).mean())) for a, b in ((gF, gF64), (gM, gM64))]
        errs[fp32] = (abs(v - v64), max(rel))
    # double sums: value to ~1e-9, derivative fields to float rounding
    assert errs[False][0] < 1e-7 and errs[False][1] < 1e-5
    # float sums lose digits to the cancellation in sum(F^2) - n mean^2 at this intensity range
    assert errs[True][0] > 10 * errs[False][0] or errs[True][1] > 10 * errs[False][1]


def test_fp16_field_storage(cuda):
    size = (80, 72)
    f, m = phantoms.pair_2d(size, seed=22)
    g = Geom(size)
    outs = {}
    for flags in (SYNX_F_USE_GRAPHS, SYNX_F_USE_GRAPHS | SYNX_F_FIELDS_FP16):
        P = SyNParams(dim=2, cc_radius=2, iterations=(10, 5), shrink_factors=(2, 1), smoothing_sigmas=(1.0, 0.0),
                      convergence_threshold=1e-12, flags=flags)
        with SyNStage(P) as st:
            st.set_images(f, g, m, g)
            st.run()
            outs[flags] = (st.fields()[0].copy(), [h.copy() for h in st.half_fields()])
    # every stored half-field value is a half-precision number
    for h in outs[SYNX_F_USE_GRAPHS | SYNX_F_FIELDS_FP16][1]:
        np.testing.assert_array_equal(h.astype(np.float16).astype(np.float32), h)
    d = outs[SYNX_F_USE_GRAPHS][0] - outs[SYNX_F_USE_GRAPHS | SYNX_F_FIELDS_FP16][0]
    rms = float(np.sqrt((d ** 2).sum(-1).mean()))
    assert 0.0 < rms < 0.05
