"""Per-step parity of the CUDA kernels (through the C ABI) against the CPU oracle.

Inputs are seeded; the oracle runs in float32 storage with FP64 window sums, as the GPU
does.  Tolerances are stated per test: differences come only from operation order and
fused multiply-adds, so they are at the level of a few float32 ulps of the values involved.
"""
import numpy as np
import pytest

import oracle as O
from ants_b200 import phantoms, synx
from ants_b200.synx import Geom

pytestmark = pytest.mark.gpu


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(cuda)


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def empty(shape, cuda):
    import torch
    return torch.empty(shape, dtype=torch.float32, device=cuda)


def field(shape, sigma, max_norm, seed):
    u = phantoms.smooth_field(shape, sigma, max_norm, np.random.default_rng(seed))
    return np.moveaxis(u, -1, 0).astype(np.float32).copy()  # component planes


GEOMS = [
    Geom((37, 29, 23), (1.0, 1.0, 1.0)),
    Geom((33, 30, 21), (1.2, 0.9, 1.5), (4.0, -3.0, 2.5)),
    Geom((61, 47), (1.0, 1.0)),
    Geom((5, 6, 7)),
]


@pytest.mark.parametrize("gi", range(len(GEOMS)))
@pytest.mark.parametrize("sigma,mm", [(1.5, False), (2.0, True), (0.0, False)])
def test_smooth_image(cuda, gi, sigma, mm):
    g = GEOMS[gi]
    img = np.random.default_rng(gi).uniform(0, 1, g.shape).astype(np.float32)
    ref = O.smooth_image(img, g, sigma, mm)
    out = empty(g.shape, cuda)
    synx.smooth_image(dev(img, cuda), out, g, sigma, mm)
    np.testing.assert_allclose(host(out), ref, atol=2e-6, rtol=0)


@pytest.mark.parametrize("gi", range(3))
def test_warp_image(cuda, gi):
    gv = GEOMS[gi]
    # the image lives on a different grid (spacing/origin) than the virtual grid
    gimg = Geom(tuple(int(s * 1.3) for s in gv.size), tuple(s * 0.8 for s in gv.spacing),
                tuple(o - 1.0 for o in gv.origin))
    img = np.random.default_rng(10 + gi).uniform(0, 1, gimg.shape).astype(np.float32)
    u = field(gv.shape, 3.0, 4.0, 20 + gi)
    ref = O.warp_image(img, gimg, u, gv)
    out = empty(gv.shape, cuda)
    synx.warp_image(dev(img, cuda), gimg, dev(u, cuda), gv, out)
    got = host(out)
    # points on the buffer rim may fall either side in float vs double coordinates
    bad = np.abs(got - ref) > 1e-5
    assert bad.mean() < 1e-3, bad.sum()


@pytest.mark.parametrize("gi", range(len(GEOMS)))
@pytest.mark.parametrize("radius", [1, 2, 4, 5])
def test_cc_metric(cuda, gi, radius):
    g = GEOMS[gi]
    rng = np.random.default_rng(100 + gi)
    if g.dim == 2:
        F = rng.uniform(0, 1, g.shape).astype(np.float32)
        M = np.roll(F, 2, axis=1) + 0.05 * rng.standard_normal(g.shape).astype(np.float32)
    else:
        F = rng.uniform(0, 1, g.shape).astype(np.float32)
        F[:4] = 0.0  # a flat block exercises the variance guard
        M = (0.7 * np.roll(F, 1, axis=2) + 0.1 * rng.standard_normal(g.shape)).astype(np.float32)
    v_ref, gF_ref, gM_ref, _ = O.cc_metric(F, M, g, radius)
    gF = empty((g.dim,) + g.shape, cuda)
    gM = empty((g.dim,) + g.shape, cuda)
    v = synx.cc_metric(dev(F, cuda), dev(M, cuda), g, radius, gF, gM)
    assert abs(v - v_ref) < 1e-9
    for a, b in ((host(gF), gF_ref), (host(gM), gM_ref)):
        scale = max(np.abs(b).max(), 1e-20)
        np.testing.assert_allclose(a, b, atol=1e-6 * scale, rtol=1e-5)


@pytest.mark.parametrize("gi", range(len(GEOMS)))
@pytest.mark.parametrize("variance", [3.0, 0.3, 0.0])
def test_smooth_field(cuda, gi, variance):
    g = GEOMS[gi]
    u = np.random.default_rng(200 + gi).standard_normal((g.dim,) + g.shape).astype(np.float32)
    ref = O.smooth_field(u, g, variance)
    _, mx_ref = O.scale_update(ref, g, 0.1)
    out = empty(u.shape, cuda)
    mx = synx.smooth_field(dev(u, cuda), out, g, variance)
    np.testing.assert_allclose(host(out), ref, atol=2e-6, rtol=0)
    assert abs(mx - mx_ref) <= 1e-6 * mx_ref


def test_smooth_field_wide_kernel_fallback(cuda):
    # variance 300 gives a kernel too wide for the fused all-axes tile: the per-axis path runs
    g = Geom((70, 66, 64))
    u = np.random.default_rng(250).standard_normal((3,) + g.shape).astype(np.float32)
    ref = O.smooth_field(u, g, 300.0)
    out = empty(u.shape, cuda)
    synx.smooth_field(dev(u, cuda), out, g, 300.0)
    np.testing.assert_allclose(host(out), ref, atol=2e-6, rtol=0)


@pytest.mark.parametrize("gi", range(3))
def test_compose(cuda, gi):
    g = GEOMS[gi]
    d = field(g.shape, 3.0, 2.0, 300 + gi) * np.float32(min(g.spacing))
    w = field(g.shape, 4.0, 3.0, 400 + gi) * np.float32(min(g.spacing))
    ref = O.compose(d, w, g)
    out = empty(w.shape, cuda)
    synx.compose(dev(d, cuda), dev(w, cuda), g, out)
    got = host(out)
    bad = np.abs(got - ref) > 2e-5
    assert bad.mean() < 1e-3, bad.sum()
    # in place (out aliases w) gives the same result
    wd = dev(w, cuda)
    synx.compose(dev(d, cuda), wd, g, wd)
    np.testing.assert_array_equal(host(wd), got)


@pytest.mark.parametrize("gi", range(3))
@pytest.mark.parametrize("max_disp", [0.5, 2.5])
def test_invert_field(cuda, gi, max_disp):
    g = GEOMS[gi]
    phi = field(g.shape, 4.0, max_disp, 500 + gi)
    psi0 = np.zeros_like(phi)
    ref, it_ref, _, _ = O.invert(phi, psi0, g)
    psi = dev(psi0, cuda)
    it = synx.invert_field(dev(phi, cuda), psi, g)
    assert it == it_ref
    np.testing.assert_allclose(host(psi), ref, atol=5e-5, rtol=0)


def test_invert_warm_start_and_cap(cuda):
    g = GEOMS[0]
    phi = field(g.shape, 4.0, 3.0, 600)
    start = -0.5 * phi
    ref, it_ref, _, _ = O.invert(phi, start, g, max_iter=3)
    psi = dev(start, cuda)
    it = synx.invert_field(dev(phi, cuda), psi, g, max_iter=3)
    assert it == it_ref == 3
    np.testing.assert_allclose(host(psi), ref, atol=5e-5, rtol=0)


@pytest.mark.parametrize("dim", [2, 3])
def test_resample_between_levels(cuda, dim):
    fine = Geom((45, 54, 45)[:dim] if dim == 3 else (64, 60))
    coarse = synx.shrink_geom(fine, 2)
    u = field(coarse.shape, 2.0, 1.0, 700 + dim)
    ref = O.resample_field(u, coarse, fine)
    out = empty((dim,) + fine.shape, cuda)
    synx.resample_field(dev(u, cuda), coarse, out, fine)
    np.testing.assert_allclose(host(out), ref, atol=1e-6, rtol=0)
