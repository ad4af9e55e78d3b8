"""Histogram matching (--use-histogram-matching 1), CPU side.

antsRegistration's PreprocessImage matches the windowed moving image to the preprocessed fixed one
with ITK's HistogramMatchingImageFilter: 256 histogram levels, 12 match points, threshold at the
mean intensity (Examples/itkantsRegistrationHelper.hxx:111-122, called at :1135-1143).  ITK is not
part of the reference tree, so the oracle's restatement (ITK 5.4.6, the version
SuperBuild/External_ITKv5.cmake:155 pins) is checked here against a second, vectorised numpy
restatement and against the properties the filter's construction guarantees.  The device kernels
are checked against the oracle in test_zz_u_histogram_match_gpu.py.
"""
import numpy as np
import pytest

import oracle as O
from ants_b200 import phantoms
from ants_b200.synx import Geom, SyNParams


def np_quantile(h, lo, bw, p):
    """ITK Histogram::Quantile on equal bins, vectorised: from the bottom below p = 0.5, from the top above."""
    nb, total = len(h), h.sum()
    bmin = lambda k: lo + k * bw
    bmax = lambda k: lo + (k + 1) * bw
    if p < 0.5:
        cdf = np.cumsum(h) / total
        hit = np.nonzero(cdf >= p)[0]
        k = int(hit[0]) if hit.size else nb - 1
        prev = cdf[k - 1] if k > 0 else 0.0
        return bmin(k) + ((p - prev) / (h[k] / total)) * (bmax(k) - bmin(k))
    upper = 1.0 - np.cumsum(h[::-1])[::-1] / total  # after the bins k..nb-1 are taken
    hit = np.nonzero(upper <= p)[0]
    k = int(hit[-1]) if hit.size else 0
    prev = upper[k + 1] if k + 1 < nb else 1.0
    return bmax(k) - ((prev - p) / (h[k] / total)) * (bmax(k) - bmin(k))


def np_table(src, ref, levels, points, thr_mean, dtype):
    def stats(x):
        x = x.astype(dtype).ravel()
        mean = dtype(sum(x.astype(np.float64).tolist()) / x.size)  # voxel order, as the filter sums
        return x, float(x.min()), float(x.max()), float(mean)

    def hist(x, lo, hi, vlo):
        v = x.astype(np.float64)
        v = v[(v >= vlo) & (v <= hi)]
        bw = (hi - lo) / levels
        b = np.clip((v - lo) / bw, 0, None).astype(np.int64) if bw > 0 else np.zeros(v.size, np.int64)
        return np.bincount(np.minimum(b, levels - 1), minlength=levels).astype(np.float64), bw

    s, smin, smax, smean = stats(src)
    r, rmin, rmax, rmean = stats(ref)
    sthr, rthr = (smean, rmean) if thr_mean else (smin, rmin)
    hs, bws = hist(s, smin, smax, sthr)
    hr, bwr = hist(r, rmin, rmax, rthr)
    ts, tr = np.zeros(points + 2), np.zeros(points + 2)
    ts[0], tr[0], ts[-1], tr[-1] = sthr, rthr, smax, rmax
    for j in range(1, points + 1):
        ts[j] = np_quantile(hs, smin, bws, j / (points + 1.0))
        tr[j] = np_quantile(hr, rmin, bwr, j / (points + 1.0))
    den = np.diff(ts)
    grad = np.where(den != 0, np.diff(tr) / np.where(den != 0, den, 1), 0.0)
    lower = (tr[0] - rmin) / (ts[0] - smin) if ts[0] != smin else 0.0
    upper = (tr[-1] - rmax) / (ts[-1] - smax) if ts[-1] != smax else 0.0
    return ts, tr, grad, np.array([smin, smax, rmin, rmax, lower, upper])


def np_match(src, ref, levels=256, points=12, thr_mean=True, dtype=np.float32):
    ts, tr, grad, (smin, smax, rmin, rmax, lower, upper) = np_table(src, ref, levels, points, thr_mean, dtype)
    v = src.astype(dtype).astype(np.float64).ravel()
    below = v[:, None] < ts[None, :]
    j = np.where(below.any(1), below.argmax(1), points + 2)
    jm = np.clip(j - 1, 0, points)
    out = tr[jm] + (v - ts[jm]) * grad[jm]
    out = np.where(j == 0, rmin + (v - smin) * lower, out)
    out = np.where(j == points + 2, rmax + (v - smax) * upper, out)
    return out.astype(dtype).reshape(src.shape)


def images(case):
    """Two images with different intensity profiles: a phantom and a nonlinear remap of its partner."""
    if case == "2d":
        f, m = phantoms.pair_2d((72, 66), seed=5)
    else:
        f, m = phantoms.pair_3d((30, 28, 26), seed=6)
    m = 200.0 * np.abs(m) ** 1.7 + 30.0 + np.random.default_rng(1).normal(0, 2.0, m.shape)
    return O.preprocess(f), O.preprocess(m.astype(np.float32))


@pytest.mark.parametrize("case", ["2d", "3d"])
@pytest.mark.parametrize("levels,points,thr_mean", [(256, 12, True), (256, 12, False), (64, 5, True), (7, 1, True), (255, 64, False)])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_oracle_matches_numpy_restatement(case, levels, points, thr_mean, dtype):
    ref, src = images(case)
    ts, tr, gr, ends = O.histogram_match_table(src, ref, levels, points, thr_mean, dtype=dtype)
    ns, nr, ng, ne = np_table(src, ref, levels, points, thr_mean, dtype)
    np.testing.assert_allclose(ts, ns, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(tr, nr, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(gr, ng, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(ends, ne, rtol=1e-10, atol=1e-12)
    got = O.histogram_match(src, ref, levels, points, thr_mean, dtype=dtype)
    want = np_match(src, ref, levels, points, thr_mean, dtype)
    assert got.dtype == dtype
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-6 if dtype == np.float32 else 1e-12)


def test_table_anchors_and_monotone_map():
    ref, src = images("3d")
    ts, tr, gr, (smin, smax, rmin, rmax, lower, upper) = O.histogram_match_table(src, ref)
    # first row: the means (threshold at the mean); last row: the maxima; ends of the lower line
    assert ts[0] == np.float32(np.float64(src).mean()) and tr[0] == np.float32(np.float64(ref).mean())
    assert ts[-1] == src.max() and tr[-1] == ref.max() and smin == src.min() and rmin == ref.min()
    assert upper == 0.0  # the last point is the source maximum, so the upper line has no run
    # quantile rows increase: the map is monotone
    assert np.all(np.diff(ts[1:]) >= 0) and np.all(np.diff(tr[1:]) >= 0) and np.all(gr >= 0) and lower >= 0
    x = np.sort(src.ravel())
    y = O.histogram_match(x, ref)
    assert np.all(np.diff(y) >= 0)
    # the anchors map onto the reference's: min -> min, max -> max, and the threshold (the mean)
    # separates the voxels below the reference's mean from those at or above it
    out = O.histogram_match(src, ref)
    assert np.all(out[src == smin] == np.float32(rmin)) and np.all(out[src == smax] == np.float32(rmax))
    above = src.astype(np.float64) >= ts[0]
    assert above.any() and (~above).any()
    assert out[above].min() >= np.float32(tr[0]) and out[~above].max() <= np.float32(tr[0])


def test_matching_an_image_to_itself_is_the_identity():
    ref, src = images("2d")
    np.testing.assert_allclose(O.histogram_match(src, src), src, atol=2e-7, rtol=0)


def test_matched_quantiles_follow_the_reference():
    # above the threshold the matched image's deciles move to the reference's
    ref, src = images("3d")
    out = O.histogram_match(src, ref)
    q = np.linspace(0.1, 0.9, 9)
    def dec(x):
        return np.quantile(x[x >= np.float32(np.float64(x).mean())], q)
    assert np.abs(dec(out) - dec(ref)).max() < 0.25 * np.abs(dec(src) - dec(ref)).max()


def test_registration_applies_it_to_the_moving_image_after_the_window():
    # syn_register(histogram_match) = syn_register on the windowed images with the moving one matched
    ref_raw, _ = phantoms.pair_2d((48, 44), seed=12)
    _, m = phantoms.pair_2d((48, 44), seed=12)
    m = (150.0 * np.abs(m) ** 2 + 10.0).astype(np.float32)
    g = Geom((48, 44))
    P = SyNParams(dim=2, cc_radius=2, iterations=(4, 3), shrink_factors=(2, 1), smoothing_sigmas=(1.0, 0.0),
                  convergence_threshold=1e-12, histogram_match=True)
    a = O.syn_register(ref_raw, g, m, g, P)
    F, M = O.preprocess(ref_raw), O.preprocess(m)
    Q = SyNParams(**{**P.__dict__, "preprocess": False, "histogram_match": False})
    b = O.syn_register(F, g, O.histogram_match(M, F), g, Q)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    c = O.syn_register(ref_raw, g, m, g, SyNParams(**{**P.__dict__, "histogram_match": False}))
    assert not np.array_equal(a[0], c[0])  # the option changes the registration


def test_constant_images():
    # zero-width bins: every quantile is the constant, every slope 0, and the source maps to the
    # reference's maximum (no table point lies above it)
    src = np.full((10, 12), 0.25, np.float32)
    ref = np.linspace(0, 1, 120, dtype=np.float32).reshape(10, 12)
    ts, tr, gr, ends = O.histogram_match_table(src, ref)
    assert np.all(ts == np.float32(0.25)) and np.all(gr == 0) and ends[4] == 0 and ends[5] == 0
    out = O.histogram_match(src, ref)
    np.testing.assert_array_equal(out, np.full_like(src, ref.max()))
    np.testing.assert_array_equal(out, np_match(src, ref))
    # a constant reference: all reference points coincide, so everything at or above the source's
    # mean maps onto that constant and the lower line runs flat from the reference minimum
    out = O.histogram_match(ref, np.full_like(ref, 0.5))
    np.testing.assert_array_equal(out, np_match(ref, np.full_like(ref, 0.5)))
    assert np.all(out == np.float32(0.5))
