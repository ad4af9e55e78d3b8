"""Properties at the full 182x218x182 size of the single-pair workload (the whole-stage comparison
with the oracle at this size is in test_zz_v_parity_configs.py): the CC value and both update
directions are invariant to an affine intensity change of the fixed image, update smoothing is
linear and matches the oracle, a registration repeats bit for bit, and its forward and inverse
fields compose to (nearly) the identity."""
import numpy as np
import pytest
import torch

from ants_b200 import phantoms, synx
from ants_b200.synx import SYNX_F_USE_GRAPHS, Geom, SyNParams, SyNStage

pytestmark = pytest.mark.gpu

SIZE = (182, 218, 182)


@pytest.fixture(scope="module")
def pair():
    return phantoms.pair_3d(SIZE, seed=phantoms.SEED_BASE)


def test_cc_invariant_to_affine_intensity_change(cuda, pair):
    f, m = pair
    g = Geom(SIZE)
    F, M = torch.from_numpy(f).cuda(), torch.from_numpy(m).cuda()
    F2 = 2.5 * F + 3.0
    out = []
    for a in (F, F2):
        gF = torch.empty((3,) + g.shape, device="cuda")
        gM = torch.empty_like(gF)
        v = synx.cc_metric(a, M, g, 4, gF, gM)
        out.append((v, gF.cpu().numpy(), gM.cpu().numpy()))
    assert abs(out[0][0] - out[1][0]) < 1e-7
    # 2.5 F + 3 is itself rounded to float, which moves the central differences of the warped
    # images (and so the derivative fields) by about 1e-4 relative; the window sums are double
    for k in (1, 2):
        ref, got = out[0][k], out[1][k]
        assert np.sqrt(((got - ref) ** 2).mean() / (ref ** 2).mean()) < 1e-3


def test_update_smoothing_is_linear(cuda):
    g = Geom(SIZE)
    rng = np.random.default_rng(5)
    u = torch.from_numpy(rng.standard_normal((3,) + g.shape).astype(np.float32)).cuda()
    v = torch.from_numpy(rng.standard_normal((3,) + g.shape).astype(np.float32)).cuda()
    su, sv, sw = (torch.empty_like(u) for _ in range(3))
    synx.smooth_field(u, su, g, 3.0)
    synx.smooth_field(v, sv, g, 3.0)
    synx.smooth_field(2.0 * u - 0.5 * v, sw, g, 3.0)
    err = (sw - (2.0 * su - 0.5 * sv)).abs().max().item()
    assert err < 1e-5 * max(1.0, sw.abs().max().item())


def test_update_smoothing_matches_oracle_at_full_size(cuda):
    # the xy and z smoothing kernels at full size (the z kernel walks columns in chunks): the oracle
    import oracle as O
    g = Geom(SIZE)
    u = np.random.default_rng(6).standard_normal((3,) + g.shape).astype(np.float32)
    ref = O.smooth_field(u, g, 3.0)
    out = torch.empty((3,) + g.shape, device="cuda")
    synx.smooth_field(torch.from_numpy(u).cuda(), out, g, 3.0)
    np.testing.assert_allclose(out.cpu().numpy(), ref, atol=2e-6, rtol=0)


def test_registration_repeats_and_fields_are_inverse(cuda, pair):
    f, m = pair
    g = Geom(SIZE)
    P = SyNParams(dim=3, cc_radius=4, iterations=(100, 70, 50, 20), shrink_factors=(8, 4, 2, 1),
                  smoothing_sigmas=(3.0, 2.0, 1.0, 0.0), convergence_threshold=1e-12, flags=SYNX_F_USE_GRAPHS)
    runs = []
    with SyNStage(P) as st:
        for _ in range(2):
            st.set_images(f, g, m, g)
            st.run()
            fw, iv = st.fields()
            runs.append((fw.copy(), iv.copy(), [(r.level, r.metric, r.inverse_iterations) for r in st.log()]))
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    np.testing.assert_array_equal(runs[0][1], runs[1][1])
    assert runs[0][2] == runs[1][2]
    # the metric improved over the full-resolution level (metrics of different levels differ in scale)
    last = [mv for lv, mv, _ in runs[0][2] if lv == 3]
    assert len(last) == 20 and last[-1] < last[0]
    # inverse(x + forward(x)) + forward(x) ~ 0: compose the two fields on the device
    fw = torch.from_numpy(np.ascontiguousarray(np.moveaxis(runs[0][0], -1, 0))).cuda()
    iv = torch.from_numpy(np.ascontiguousarray(np.moveaxis(runs[0][1], -1, 0))).cuda()
    r = torch.empty_like(fw)
    synx.compose(iv, fw, g, r)
    res = r.norm(dim=0).cpu().numpy()  # mm (1 mm voxels)
    inner = res[4:-4, 4:-4, 4:-4]
    assert float(np.abs(fw.cpu().numpy()).max()) > 1.0  # a real deformation
    mean, p99 = float(inner.mean()), float(np.percentile(inner, 99))
    assert mean < 0.05 and p99 < 0.5, (mean, p99)
