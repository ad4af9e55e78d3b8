"""Metric masks in the SyN + CC stage (antsRegistration -x [fixedMask,movingMask]).

The reference sets the masks on the metric (Examples/itkantsRegistrationHelper.hxx:863-890,
:1159-1166); SyN resamples each mask into the virtual domain through its image's inverse half-field
(nearest neighbour, 0 outside), and the neighbourhood CC then sums, counts and evaluates only the
voxels inside both.  Checks: the masked CC kernel against the oracle (itself checked against a
brute-force restatement on the CPU, tests/test_oracle_steps.py); whole masked stages against the
oracle's masked registration; the command line's -x against the Python API (on the GPU) and against
the oracle (through the host harness, on the CPU).
"""
import subprocess

import numpy as np
import pytest

import oracle as O
from ants_b200 import nifti, phantoms
from ants_b200.synx import SYNX_F_USE_GRAPHS, Geom, SyNParams, SyNStage


def ellipsoid_mask(shape, centre_frac, radii_frac):
    idx = np.indices(shape, dtype=np.float64)
    r = np.zeros(shape)
    for a, n in enumerate(shape):
        r += ((idx[a] - centre_frac[a] * (n - 1)) / (radii_frac[a] * n)) ** 2
    return (r <= 1.0).astype(np.float32)


def planes(interleaved):
    return np.moveaxis(interleaved, -1, 0)


def rms_vox(a, b, spacing):
    sp = np.asarray(spacing, dtype=np.float64).reshape((-1,) + (1,) * (a.ndim - 1))
    return float(np.sqrt((((a - b) / sp) ** 2).sum(0).mean()))


@pytest.mark.gpu
@pytest.mark.parametrize("shape,r", [((23, 29, 31), 3), ((37, 41), 2), ((18, 20, 22), 5)])
def test_masked_cc_matches_oracle(cuda, shape, r):
    import torch

    from ants_b200 import synx
    rng = np.random.default_rng(31)
    F = rng.uniform(0, 1, shape).astype(np.float32)
    M = (0.6 * np.roll(F, 1, axis=-1) + 0.3 * rng.uniform(0, 1, shape)).astype(np.float32)
    valid = (rng.uniform(0, 1, shape) > 0.25) & (ellipsoid_mask(shape, [0.5] * len(shape), [0.45] * len(shape)) > 0)
    g = Geom(tuple(reversed(shape)))
    v_ref, gF_ref, gM_ref, _ = O.cc_metric(F, M, g, r, valid=valid)
    gF = torch.full((g.dim,) + g.shape, float("nan"), device=cuda)
    gM = torch.full_like(gF, float("nan"))
    v = synx.cc_metric_masked(torch.from_numpy(F).to(cuda), torch.from_numpy(M).to(cuda),
                              torch.from_numpy(valid.astype(np.uint8)).to(cuda), g, r, gF, gM)
    assert abs(v - v_ref) < 1e-6
    for a, b in ((gF, gF_ref), (gM, gM_ref)):
        a = a.cpu().numpy()
        scale = max(np.abs(b).max(), 1e-20)
        np.testing.assert_allclose(a, b, atol=1e-6 * scale, rtol=1e-5)


def masked_pair(dim, seed):
    if dim == 3:
        size = (40, 44, 36)
        f, m = phantoms.pair_3d(size, seed=seed)
        g = Geom(size, (1.0, 1.125, 0.875))  # float32-exact spacings: NIfTI stores them as float
    else:
        size = (80, 72)
        f, m = phantoms.pair_2d(size, seed=seed)
        g = Geom(size, (1.0, 0.875))
    shape = f.shape
    mf = ellipsoid_mask(shape, [0.5] * dim, [0.42] * dim)
    mm = ellipsoid_mask(shape, [0.52] * dim, [0.45] * dim)
    return f, m, g, mf, mm


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("which", ["both", "fixed", "moving"])
def test_masked_stage_matches_oracle(cuda, dim, which):
    f, m, g, mf, mm = masked_pair(dim, seed=41 + dim)
    mf = mf if which in ("both", "fixed") else None
    mm = mm if which in ("both", "moving") else None
    P = SyNParams(dim=dim, cc_radius=2 if dim == 2 else 3, iterations=(10, 6), shrink_factors=(2, 1),
                  smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12, flags=SYNX_F_USE_GRAPHS)
    with SyNStage(P) as st:
        st.set_masks(mf, g if mf is not None else None, mm, g if mm is not None else None)
        st.set_images(f, g, m, g)
        st.run()
        fwd, inv = (planes(a) for a in st.fields())
        go = st.output_geom()
        log = st.log()
    rf, ri, _, rlog = O.syn_register(f, g, m, g, P, fixed_mask=mf, fixed_mask_geom=g, moving_mask=mm,
                                     moving_mask_geom=g)
    unmasked, _, _, ulog = O.syn_register(f, g, m, g, P)
    assert [(r.level, r.iteration) for r in log] == [(r["level"], r["iteration"]) for r in rlog]
    np.testing.assert_allclose([r.metric for r in log], [r["metric"] for r in rlog], atol=2e-3)
    assert rms_vox(fwd, rf, go.spacing) <= 0.05
    assert rms_vox(inv, ri, go.spacing) <= 0.05
    # the masks change the registration: the metric values differ from the unmasked run's
    assert max(abs(a["metric"] - b["metric"]) for a, b in zip(rlog, ulog)) > 1e-3


def check_cli_masks(reg, tmp_path, stage_fields):
    """-x [fixed,moving], -x fixed and -x [NULL,moving] give the stage's fields with those masks.
    stage_fields(f, g, m, g, P, mf, mm) returns the stage's (forward, inverse) fields, interleaved."""
    f, m, g, mf, mm = masked_pair(2, seed=53)
    for name, a in (("f", f), ("m", m), ("mf", mf), ("mm", mm)):
        nifti.write(tmp_path / f"{name}.nii.gz", a, g)
    P = SyNParams(dim=2, learning_rate=0.2, cc_radius=2, iterations=(6, 3), shrink_factors=(2, 1),
                  smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12)
    cases = {"both": (f"[{tmp_path}/mf.nii.gz,{tmp_path}/mm.nii.gz]", mf, mm),
             "fixed": (f"{tmp_path}/mf.nii.gz", mf, None),
             "moving": (f"[NULL,{tmp_path}/mm.nii.gz]", None, mm)}
    for label, (xarg, a, b) in cases.items():
        prefix = str(tmp_path / f"{label}_")
        r = subprocess.run([reg, "-d", "2", "--float", "1", "-m", f"CC[{tmp_path}/f.nii.gz,{tmp_path}/m.nii.gz,1,2]",
                            "-t", "SyN[0.2,3,0]", "-c", "[6x3,1e-12,10]", "-f", "2x1", "-s", "1x0vox", "-x", xarg,
                            "-o", prefix], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        got = (nifti.read(prefix + "0Warp.nii.gz", 2)[0], nifti.read(prefix + "0InverseWarp.nii.gz", 2)[0])
        want = stage_fields(f, g, m, g, P, a, b)
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[1], want[1])


@pytest.mark.gpu
def test_cli_masks(cuda, tmp_path):
    from ants_b200 import build
    build.build_all()

    def stage_fields(f, gf, m, gm, P, mf, mm):
        with SyNStage(P) as st:
            st.set_masks(mf, gf if mf is not None else None, mm, gm if mm is not None else None)
            st.set_images(f, gf, m, gm)
            st.run()
            return st.fields()

    check_cli_masks(build.CLI, tmp_path, stage_fields)
