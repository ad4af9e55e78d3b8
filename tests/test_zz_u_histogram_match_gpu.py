"""Histogram matching (--use-histogram-matching 1) on the device, against the oracle.

synx_histogram_match against the oracle's restatement of ITK's HistogramMatchingImageFilter, the
stage with the option against the oracle's registration, and the command line's -u 1 against the
Python API.  The command-line check is shared with the host harness
(tests/test_cli_host_plumbing.py), which runs it on a machine without a GPU.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from ants_b200 import nifti, phantoms, synx
from ants_b200.synx import Geom, SyNParams, SyNStage
from test_gpu_syn import planes, rms_vox
from test_histogram_match import images

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def remapped_pair(size, seed):
    """A phantom pair whose moving image has another intensity profile (a power law, an offset)."""
    f, m = phantoms.pair_2d(size, seed=seed) if len(size) == 2 else phantoms.pair_3d(size, seed=seed)
    return f, (180.0 * np.abs(m) ** 1.8 + 25.0).astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["2d", "3d"])
@pytest.mark.parametrize("levels,points,thr_mean", [(256, 12, True), (256, 12, False), (64, 5, True), (7, 1, True), (255, 64, False)])
def test_device_matches_oracle(cuda, case, levels, points, thr_mean):
    import torch
    ref, src = images(case)
    want = O.histogram_match(src, ref, levels, points, thr_mean)
    s, r = torch.from_numpy(src).to(cuda), torch.from_numpy(ref).to(cuda)
    out = torch.empty_like(s)
    synx.histogram_match(s, r, out, levels, points, thr_mean)
    got = out.cpu().numpy()
    # the same table up to the mean's summation order (per block on the device, voxel order in
    # the oracle), which moves the float mean only at a rounding tie
    np.testing.assert_allclose(got, want, atol=1e-6, rtol=0)
    assert (got == want).mean() > 0.999


@pytest.mark.gpu
def test_device_full_size_in_place(cuda):
    # 182 x 218 x 182 voxels (one MNI-sized image pair), matched in place
    import torch
    rng = np.random.default_rng(3)
    shape = (182, 218, 182)
    ref = np.where(rng.random(shape) < 0.4, 0.0, rng.gamma(4.0, 0.1, shape)).astype(np.float32)
    src = np.where(rng.random(shape) < 0.5, 0.0, rng.gamma(2.0, 0.2, shape) ** 1.5).astype(np.float32)
    want = O.histogram_match(src, ref)
    s, r = torch.from_numpy(src).to(cuda), torch.from_numpy(ref).to(cuda)
    synx.histogram_match(s, r, s)
    got = s.cpu().numpy()
    np.testing.assert_allclose(got, want, atol=1e-6, rtol=0)
    assert (got == want).mean() > 0.999


@pytest.mark.gpu
@pytest.mark.parametrize("dim,size", [(2, (80, 76)), (3, (34, 32, 30))])
def test_stage_with_histogram_matching_matches_oracle(cuda, dim, size):
    f, m = remapped_pair(size, seed=17)
    g = Geom(size)
    P = SyNParams(dim=dim, cc_radius=2, learning_rate=0.2, iterations=(10, 5), shrink_factors=(2, 1),
                  smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12, histogram_match=True)
    with SyNStage(P) as st:
        st.set_images(f, g, m, g)
        st.run()
        fwd, inv = (planes(a) for a in st.fields())
        go = st.output_geom()
        log = st.log()
    rf, ri, rg, rlog = O.syn_register(f, g, m, g, P)
    assert [(r.level, r.iteration) for r in log] == [(r["level"], r["iteration"]) for r in rlog]
    np.testing.assert_allclose([r.metric for r in log], [r["metric"] for r in rlog], atol=2e-3)
    assert rms_vox(fwd, rf, go.spacing) <= 0.05
    assert rms_vox(inv, ri, go.spacing) <= 0.05


def check_cli_histogram_matching(reg, tmp_path, stage_fields):
    """-u 1 gives the fields of the stage run with histogram_match on; -u 0 gives other fields.
    stage_fields(f, g, m, g, P) returns the stage's (forward, inverse) fields, interleaved."""
    size = (60, 56)
    f, m = remapped_pair(size, seed=21)
    g = Geom(size, (1.0, 1.0), (2.0, -3.0))
    nifti.write(tmp_path / "f.nii.gz", f, g)
    nifti.write(tmp_path / "m.nii.gz", m, g)
    out = {}
    for u in ("1", "0"):
        prefix = str(tmp_path / f"u{u}_")
        r = subprocess.run([reg, "-d", "2", "--float", "1", "-m", f"CC[{tmp_path}/f.nii.gz,{tmp_path}/m.nii.gz,1,2]",
                            "-t", "SyN[0.2,3,0]", "-c", "[6x3,1e-12,10]", "-f", "2x1", "-s", "1x0vox", "-u", u,
                            "-o", prefix], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        out[u] = (nifti.read(prefix + "0Warp.nii.gz", 2)[0], nifti.read(prefix + "0InverseWarp.nii.gz", 2)[0])
    P = SyNParams(dim=2, learning_rate=0.2, cc_radius=2, iterations=(6, 3), shrink_factors=(2, 1),
                  smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12, histogram_match=True)
    a, b = stage_fields(f, g, m, g, P)
    np.testing.assert_array_equal(out["1"][0], a)
    np.testing.assert_array_equal(out["1"][1], b)
    assert not np.array_equal(out["0"][0], out["1"][0])


@pytest.mark.gpu
def test_cli_histogram_matching(cuda, tmp_path):
    from ants_b200 import build
    build.build_all()

    def stage_fields(f, gf, m, gm, P):
        with SyNStage(P) as st:
            st.set_images(f, gf, m, gm)
            st.run()
            return st.fields()

    check_cli_histogram_matching(build.CLI, tmp_path, stage_fields)


@pytest.mark.gpu
def test_device_edge_cases(cuda):
    import torch
    from ants_b200.synx import SynxError
    # a constant source (zero-width bins) and a constant reference, as in the oracle's own tests
    src = np.full((10, 12), 0.25, np.float32)
    ref = np.linspace(0, 1, 120, dtype=np.float32).reshape(10, 12)
    for a, b in ((src, ref), (ref, np.full_like(ref, 0.5))):
        s, r = torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda)
        out = torch.empty_like(s)
        synx.histogram_match(s, r, out)
        np.testing.assert_array_equal(out.cpu().numpy(), O.histogram_match(a, b))
    # an empty source is refused by the library, not launched
    e = torch.empty(0, device=cuda)
    with pytest.raises(SynxError):
        synx.histogram_match(e, torch.from_numpy(ref).to(cuda), e)
