"""Registration state and composite transform output of the SyN + CC stage.

antsRegistration --save-state writes the state as a composite transform (the initial transforms,
then the fixed-to-middle field, its inverse, the moving-to-middle field, its inverse:
Examples/antsRegistrationTemplateHeader.h:1307-1346); --restore-state with
--initialize-transforms-per-stage 1 starts the SyN stage from those four fields
(Examples/itkantsRegistrationHelper.hxx:2093-2125, :3637-3725); --write-composite-transform 1 writes
prefixComposite and prefixInverseComposite instead of the separate files (:1394-1424).  This build
writes them in ITK's text transform form.  Checks: a stage started from a saved state's half-fields
against the oracle's (GPU), and the command line's state and composite files, their round trip and its
option rules against the Python API (GPU) or the oracle (through the host harness, CPU).
"""
import subprocess

import numpy as np
import pytest

import oracle as O
from ants_b200 import nifti, phantoms
from ants_b200.synx import SYNX_F_USE_GRAPHS, Geom, SyNParams, SyNStage


def planes(interleaved):
    return np.ascontiguousarray(np.moveaxis(interleaved, -1, 0))


def interleaved(planar):
    return np.ascontiguousarray(np.moveaxis(planar, 0, -1))


def read_composite(path):
    """[(type, parameters, fixed parameters)] of an ITK text transform file, composite entry left out."""
    items = []
    for line in open(path):
        line = line.strip()
        if not line or line.startswith("#"):
            continue
        key, _, val = line.partition(":")
        if key == "Transform":
            if not val.strip().startswith("CompositeTransform_"):
                items.append([val.strip(), None, None])
        elif key == "Parameters":
            items[-1][1] = np.array([np.float32(v) if "Displacement" in items[-1][0] else float(v)
                                     for v in val.split()])
        elif key == "FixedParameters":
            items[-1][2] = np.array([float(v) for v in val.split()])
    return items


def rms_vox(a, b, spacing):
    sp = np.asarray(spacing, dtype=np.float64).reshape((-1,) + (1,) * (a.ndim - 1))
    return float(np.sqrt((((a - b) / sp) ** 2).sum(0).mean()))


def saved_state(f, g, m, P):
    """The half-fields (component planes) a short registration of the pair ends with: what a saved
    registration state holds.  Each inverse field is the inverse of its forward one, as in a real state
    (four unrelated random fields would make the first inversions ill-conditioned)."""
    *_, half = O.syn_register(f, g, m, g, P, return_half_fields=True)
    return [np.ascontiguousarray(h) for h in half]


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_stage_from_initial_half_fields_matches_oracle(cuda, dim):
    if dim == 3:
        size = (40, 44, 36)
        f, m = phantoms.pair_3d(size, seed=61)
        g = Geom(size, (1.0, 1.125, 0.875))
    else:
        size = (80, 72)
        f, m = phantoms.pair_2d(size, seed=62)
        g = Geom(size, (1.0, 0.875))
    r = 2 if dim == 2 else 3
    P0 = SyNParams(dim=dim, learning_rate=0.25, cc_radius=r, iterations=(20, 10), shrink_factors=(2, 1),
                   smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12)
    init = saved_state(f, g, m, P0)
    P = SyNParams(dim=dim, cc_radius=r, iterations=(8, 5), shrink_factors=(2, 1),
                  smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12, flags=SYNX_F_USE_GRAPHS)
    with SyNStage(P) as st:
        st.set_images(f, g, m, g)
        st.set_initial_half_fields(*[interleaved(a) for a in init], grid=g)
        st.run()
        fwd, inv = (planes(a) for a in st.fields())
        log = st.log()
        go = st.output_geom()
    rf, ri, _, rlog = O.syn_register(f, g, m, g, P, initial_half_fields=init, initial_geom=g)
    zf, _, _, zlog = O.syn_register(f, g, m, g, P)
    assert [(r.level, r.iteration) for r in log] == [(r["level"], r["iteration"]) for r in rlog]
    np.testing.assert_allclose([r.metric for r in log], [r["metric"] for r in rlog], atol=2e-3)
    assert rms_vox(fwd, rf, go.spacing) <= 0.05
    assert rms_vox(inv, ri, go.spacing) <= 0.05
    # the starting fields change the registration, and the stage followed them: it lies far closer to the
    # oracle's seeded run than to its run from zero fields
    assert rms_vox(rf, zf, go.spacing) > 0.03
    assert rms_vox(fwd, rf, go.spacing) < 0.5 * rms_vox(fwd, zf, go.spacing)


@pytest.mark.gpu
def test_seeded_stage_repeats_bit_for_bit(cuda):
    # four unrelated smooth fields make every inversion run its full 20 sub-iterations; the uploaded
    # fields (about 760 KB each) must reach the device before the first level resamples them
    size = (40, 44, 36)
    f, m = phantoms.pair_3d(size, seed=61)
    g = Geom(size, (1.0, 1.125, 0.875))
    rng = np.random.default_rng(66)
    sp = np.asarray(g.spacing).reshape((-1, 1, 1, 1))
    init = [np.ascontiguousarray(np.moveaxis((np.moveaxis(phantoms.smooth_field(f.shape, 6.0, 1.5, rng), -1, 0) * sp)
                                             .astype(np.float32), 0, -1)) for _ in range(4)]
    P = SyNParams(dim=3, cc_radius=3, iterations=(8, 5), shrink_factors=(2, 1), smoothing_sigmas=(1.0, 0.0),
                  convergence_threshold=1e-12, flags=SYNX_F_USE_GRAPHS)
    runs = []
    for _ in range(2):
        with SyNStage(P) as st:
            st.set_images(f, g, m, g)
            st.set_initial_half_fields(*init, grid=g)
            st.run()
            runs.append(st.fields())
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    np.testing.assert_array_equal(runs[0][1], runs[1][1])


def check_cli_state(reg, tmp_path, stage):
    """--save-state, --restore-state, -a 1 and their option rules on a 2-D pair.
    stage(f, g, m, g, P, init) -> (forward, inverse, (phiF, psiF, phiM, psiM)), interleaved, where
    init is None or four interleaved half-fields on g."""
    size = (80, 72)
    f, m = phantoms.pair_2d(size, seed=71)
    g = Geom(size, (1.0, 0.875))
    for name, a in (("f", f), ("m", m)):
        nifti.write(tmp_path / f"{name}.nii.gz", a, g)
    P = SyNParams(dim=2, learning_rate=0.2, cc_radius=2, iterations=(6, 3), shrink_factors=(2, 1),
                  smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12)
    base = [reg, "-d", "2", "--float", "1", "-m", f"CC[{tmp_path}/f.nii.gz,{tmp_path}/m.nii.gz,1,2]",
            "-t", "SyN[0.2,3,0]", "-c", "[6x3,1e-12,10]", "-f", "2x1", "-s", "1x0vox"]

    def run(*extra):
        return subprocess.run(base + list(extra), capture_output=True, text=True, timeout=600)

    state = str(tmp_path / "state.txt")
    r = run("-a", "1", "-z", "0", "-i", "1", "-j", state, "-o", str(tmp_path / "A_"))
    assert r.returncode == 0, r.stderr
    want_fwd, want_inv, want_half = stage(f, g, m, g, P, None)
    items = read_composite(state)
    assert [t.split("_")[0] for t, _, _ in items] == ["DisplacementFieldTransform"] * 4
    fixed = np.array([80, 72, 0, 0, 1.0, 0.875, 1, 0, 0, 1], dtype=np.float64)
    for (t, par, fx), want in zip(items, want_half):
        assert t == "DisplacementFieldTransform_float_2_2"
        np.testing.assert_array_equal(fx, fixed)
        np.testing.assert_array_equal(par.astype(np.float32), want.reshape(-1))
    comp = read_composite(tmp_path / "A_Composite.txt")
    icomp = read_composite(tmp_path / "A_InverseComposite.txt")
    assert len(comp) == 1 and len(icomp) == 1
    np.testing.assert_array_equal(comp[0][1].astype(np.float32), want_fwd.reshape(-1))
    np.testing.assert_array_equal(icomp[0][1].astype(np.float32), want_inv.reshape(-1))
    assert not (tmp_path / "A_0Warp.nii.gz").exists()  # a composite replaces the separate files

    # restore: the stage starts from the saved half-fields
    r = run("-a", "1", "-z", "0", "-i", "1", "-k", state, "-o", str(tmp_path / "B_"))
    assert r.returncode == 0, r.stderr
    got_fwd, got_inv, _ = stage(f, g, m, g, P, list(want_half))
    comp = read_composite(tmp_path / "B_Composite.txt")
    np.testing.assert_array_equal(comp[0][1].astype(np.float32), got_fwd.reshape(-1))
    icomp = read_composite(tmp_path / "B_InverseComposite.txt")
    np.testing.assert_array_equal(icomp[0][1].astype(np.float32), got_inv.reshape(-1))
    assert np.abs(got_fwd - want_fwd).max() > 1e-3  # the restored run went on from the saved state

    # the reference's option rules
    for extra in (["-j", state, "-o", str(tmp_path / "C_")],                        # save-state needs -a 1
                  ["-a", "1", "-i", "1", "-o", str(tmp_path / "C_")],                # -i with collapsing
                  ["-i", "1", "-z", "0", "-o", str(tmp_path / "C_")],                # -i needs -a 1
                  ["-k", state, "-o", str(tmp_path / "C_")],                         # fields need -i 1
                  ["-a", "1", "-z", "0", "-i", "1", "-k", state, "-r", "identity", "-o", str(tmp_path / "C_")],
                  ["-a", "1", "-z", "0", "-i", "1", "-j", str(tmp_path / "s.h5"), "-o", str(tmp_path / "C_")]):
        r = run(*extra)
        assert r.returncode != 0, extra


@pytest.mark.gpu
def test_cli_state(cuda, tmp_path):
    from ants_b200 import build
    build.build_all()

    def stage(f, gf, m, gm, P, init):
        with SyNStage(P) as st:
            st.set_images(f, gf, m, gm)
            if init is not None:
                st.set_initial_half_fields(*init, grid=gf)
            st.run()
            fw, iv = st.fields()
            return fw, iv, st.half_fields()

    check_cli_state(build.CLI, tmp_path, stage)
