"""Parity on oblique grids: direction cosines that are not the identity, as scanners write them.

Every other parity test places its grids axis-aligned, so the gathers run their diagonal index-map
path; here the grids are rotated (and anisotropic), so the warp, composition, resampling, inversion,
CC derivative conversion (index-axis derivatives rotated into physical axes) and a whole stage run
the general path against the oracle.  Tolerances are those of the axis-aligned tests.
"""
import numpy as np
import pytest
from scipy.spatial.transform import Rotation

import oracle as O
from ants_b200 import phantoms, synx
from ants_b200.synx import SYNX_F_NO_PERSISTENT, SYNX_F_USE_GRAPHS, Geom, SyNParams, SyNStage

pytestmark = pytest.mark.gpu


def rot2(theta):
    return np.array([[np.cos(theta), -np.sin(theta)], [np.sin(theta), np.cos(theta)]])


OBLIQUE = [
    Geom((29, 25, 21), (1.1, 0.9, 1.3), (5.0, -4.0, 2.0), Rotation.from_euler("xyz", [0.3, -0.2, 0.4]).as_matrix()),
    Geom((47, 41), (0.9, 1.2), (3.0, -2.0), rot2(0.35)),
]


def other_grid(g: Geom) -> Geom:
    """A second oblique grid, rotated differently, finer, and centred on the same physical point
    with some margin, so that most warped points land inside it."""
    if g.dim == 3:
        R = Rotation.from_euler("zyx", [-0.25, 0.15, 0.1]).as_matrix()
    else:
        R = rot2(-0.3)
    size = tuple(int(s * 1.6) for s in g.size)
    sp = np.asarray(g.spacing) * 0.85
    center = np.asarray(g.origin) + g.direction @ (np.asarray(g.spacing) * (np.asarray(g.size) - 1) / 2)
    origin = center - R @ (sp * (np.asarray(size) - 1) / 2)
    return Geom(size, tuple(sp), tuple(origin), R)


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
    return np.moveaxis(u, -1, 0).astype(np.float32).copy()


@pytest.mark.parametrize("gi", range(len(OBLIQUE)))
def test_warp_image(cuda, gi):
    gv = OBLIQUE[gi]
    gimg = other_grid(gv)
    img = np.random.default_rng(10 + gi).uniform(0, 1, gimg.shape).astype(np.float32)
    u = field(gv.shape, 3.0, 4.0, 20 + gi)
    ref = O.warp_image(img, gimg, u, gv)
    out = empty(gv.shape, cuda)
    synx.warp_image(dev(img, cuda), gimg, dev(u, cuda), gv, out)
    bad = np.abs(host(out) - ref) > 1e-5
    assert bad.mean() < 1e-3, bad.sum()


@pytest.mark.parametrize("mode", ["nearest", "label"])
@pytest.mark.parametrize("gi", range(len(OBLIQUE)))
def test_warp_image_labels(cuda, gi, mode):
    gv = OBLIQUE[gi]
    gimg = other_grid(gv)
    img = np.random.default_rng(15 + gi).integers(0, 7, gimg.shape).astype(np.float32)
    u = field(gv.shape, 3.0, 4.0, 25 + gi)
    ref = O.warp_image(img, gimg, u, gv, nearest=mode == "nearest", label=mode == "label")
    out = empty(gv.shape, cuda)
    synx.warp_image(dev(img, cuda), gimg, dev(u, cuda), gv, out, nearest=mode == "nearest", label=mode == "label")
    # float vs double coordinates may round a tie or a rim point the other way
    bad = host(out) != ref
    assert bad.mean() < 1e-3, bad.sum()


@pytest.mark.parametrize("gi", range(len(OBLIQUE)))
def test_compose(cuda, gi):
    g = OBLIQUE[gi]
    d = field(g.shape, 3.0, 2.0, 300 + gi) * np.float32(min(g.spacing))
    w = field(g.shape, 4.0, 3.0, 400 + gi) * np.float32(min(g.spacing))
    ref = O.compose(d, w, g)
    out = empty(w.shape, cuda)
    synx.compose(dev(d, cuda), dev(w, cuda), g, out)
    bad = np.abs(host(out) - ref) > 2e-5
    assert bad.mean() < 1e-3, bad.sum()


@pytest.mark.parametrize("gi", range(len(OBLIQUE)))
def test_resample_field(cuda, gi):
    fine = OBLIQUE[gi]
    coarse = synx.shrink_geom(fine, 2)
    u = field(coarse.shape, 2.0, 1.0, 700 + gi)
    ref = O.resample_field(u, coarse, fine)
    out = empty((fine.dim,) + fine.shape, cuda)
    synx.resample_field(dev(u, cuda), coarse, out, fine)
    bad = np.abs(host(out) - ref) > 1e-5
    assert bad.mean() < 1e-3, bad.sum()


@pytest.mark.parametrize("gi", range(len(OBLIQUE)))
def test_invert_field(cuda, gi):
    g = OBLIQUE[gi]
    phi = field(g.shape, 4.0, 2.0, 500 + gi)
    psi0 = np.zeros_like(phi)
    ref, it_ref, _, _ = O.invert(phi, psi0, g)
    psi = dev(psi0, cuda)
    it = synx.invert_field(dev(phi, cuda), psi, g)
    # the stopping test compares a mean against 0.001: rounding may move it by one sub-iteration
    assert abs(it - it_ref) <= 1
    np.testing.assert_allclose(host(psi), ref, atol=5e-5 if it == it_ref else 2e-3, rtol=0)


@pytest.mark.parametrize("gi", range(len(OBLIQUE)))
@pytest.mark.parametrize("radius", [2, 4])
def test_cc_metric(cuda, gi, radius):
    g = OBLIQUE[gi]
    rng = np.random.default_rng(100 + gi)
    F = rng.uniform(0, 1, g.shape).astype(np.float32)
    M = (0.7 * np.roll(F, 1, axis=-1) + 0.1 * rng.standard_normal(g.shape)).astype(np.float32)
    v_ref, gF_ref, gM_ref, _ = O.cc_metric(F, M, g, radius)
    gF = empty((g.dim,) + g.shape, cuda)
    gM = empty((g.dim,) + g.shape, cuda)
    v = synx.cc_metric(dev(F, cuda), dev(M, cuda), g, radius, gF, gM)
    assert abs(v - v_ref) < 1e-9
    for a, b in ((host(gF), gF_ref), (host(gM), gM_ref)):
        scale = max(np.abs(b).max(), 1e-20)
        np.testing.assert_allclose(a, b, atol=1e-6 * scale, rtol=1e-5)


PATHS = {"persistent": SYNX_F_USE_GRAPHS, "kernels": SYNX_F_USE_GRAPHS | SYNX_F_NO_PERSISTENT}


@pytest.mark.parametrize("path", sorted(PATHS))
@pytest.mark.parametrize("dim", [2, 3])
def test_stage_on_oblique_grids(cuda, dim, path):
    size = (72, 68) if dim == 2 else (36, 40, 32)
    f, m = phantoms.pair_2d(size, seed=9) if dim == 2 else phantoms.pair_3d(size, seed=9)
    if dim == 3:
        gf = Geom(size, (1.0, 1.1, 0.9), (4.0, -3.0, 2.0), Rotation.from_euler("xyz", [0.2, 0.1, -0.3]).as_matrix())
        gm = Geom(size, (1.0, 1.1, 0.9), (3.5, -2.5, 2.5), Rotation.from_euler("xyz", [0.25, 0.05, -0.28]).as_matrix())
    else:
        gf = Geom(size, (1.0, 0.9), (4.0, -3.0), rot2(0.3))
        gm = Geom(size, (1.0, 0.9), (3.6, -2.7), rot2(0.33))
    P = SyNParams(dim=dim, cc_radius=2 if dim == 2 else 3, iterations=(10, 5), shrink_factors=(2, 1),
                  smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12, flags=PATHS[path])
    with SyNStage(P) as st:
        st.set_images(f, gf, m, gm)
        st.run()
        fwd, inv = (np.moveaxis(a, -1, 0) for a in st.fields())
        go = st.output_geom()
        log = st.log()
    rf, ri, rg, rlog = O.syn_register(f, gf, m, gm, P)
    assert go.size == rg.size
    assert [(r.level, r.iteration) for r in log] == [(r["level"], r["iteration"]) for r in rlog]
    np.testing.assert_allclose([r.metric for r in log], [r["metric"] for r in rlog], atol=2e-3)
    sp = np.asarray(go.spacing).reshape((-1,) + (1,) * dim)
    for got, want in ((fwd, rf), (inv, ri)):
        assert float(np.sqrt((((got - want) / sp) ** 2).sum(0).mean())) <= 0.05
    assert float(np.sqrt(((fwd / sp) ** 2).sum(0).mean())) > 0.02
