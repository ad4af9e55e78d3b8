"""The antsRegistration-compatible front end (ants_b200/antsRegistrationSyN_b200) and NIfTI IO."""
import os
import subprocess

import numpy as np
import pytest

from ants_b200 import nifti, phantoms
from ants_b200.synx import Geom, SyNParams, SyNStage

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "ants_b200", "antsRegistrationSyN_b200")


@pytest.fixture(scope="module")
def cli():
    from ants_b200 import build
    build.build_all()
    assert os.path.exists(CLI)
    return CLI


def run(cli, args):
    return subprocess.run([cli, *args], capture_output=True, text=True, timeout=600)


def test_nifti_roundtrip_scalar_and_vector(tmp_path):
    g = Geom((7, 6, 5), (1.5, 1.0, 2.0), (3.0, -2.0, 1.0))
    img = np.random.default_rng(0).standard_normal(g.shape).astype(np.float32)
    nifti.write(tmp_path / "a.nii.gz", img, g)
    back, gb = nifti.read(tmp_path / "a.nii.gz")
    np.testing.assert_array_equal(back, img)
    assert gb.size == g.size and gb.spacing == g.spacing and np.allclose(gb.origin, g.origin)
    fld = np.random.default_rng(1).standard_normal(g.shape + (3,)).astype(np.float32)
    nifti.write(tmp_path / "w.nii", fld, g, vector=True)
    back, gb = nifti.read(tmp_path / "w.nii")
    np.testing.assert_array_equal(back, fld)


@pytest.mark.parametrize("args,needle", [
    (["-d", "3", "-m", "MI[a,b,1,32]", "-t", "SyN[0.1,3,0]", "-c", "10", "-f", "1", "-s", "0", "-o", "x"],
     "only the CC metric"),
    (["-d", "3", "-m", "CC[a,b,1,4]", "-t", "Affine[0.1]", "-c", "10", "-f", "1", "-s", "0", "-o", "x"],
     "only the SyN transform"),
    (["-d", "3", "-m", "CC[a,b,1,4]", "-t", "SyN[0.1,3,0]", "-c", "[10x5,1e-6,10]", "-f", "2", "-s", "0", "-o", "x"],
     "must match the levels"),
    (["-d", "3", "-m", "CC[a,b,1,4]", "-t", "SyN[0.1,3,0]", "-f", "1", "-s", "0", "-o", "x"], "no convergence"),
    (["-d", "3", "-m", "CC[a,b,1,4]", "-t", "SyN[0.1,3,0]", "-c", "10", "-f", "1", "-s", "0", "-o", "x",
      "--restore-state", "/nonexistent/state.txt"], "cannot read"),
    (["-d", "3", "-m", "CC[a,b,1,4]", "-t", "SyN[0.1,3,0]", "-c", "10", "-f", "1", "-s", "0", "-o", "x",
      "--save-state", "state.txt"], "--save-state requires --write-composite-transform"),
    (["-d", "4", "-m", "CC[a,b,1,4]", "-t", "SyN[0.1,3,0]", "-c", "10", "-f", "1", "-s", "0", "-o", "x"],
     "dimensionality"),
    (["-d", "3", "-m", "CC[/nonexistent/f.nii.gz,/nonexistent/m.nii.gz,1,4]", "-t", "SyN[0.1,3,0]", "-c", "10",
      "-f", "1", "-s", "0", "-o", "x"], "cannot open"),
    (["-d", "3", "-m", "CC[a,b,1,4]", "-t", "SyN[0.1,3,0]", "-c", "10", "-f", "1", "-s", "0", "-o", "x",
      "-r", "[/nonexistent/f.nii.gz,/nonexistent/m.nii.gz,1]"], "cannot open"),
    (["-d", "3", "-m", "CC[a,b,1,4]", "-t", "SyN[0.1,3,0]", "-c", "10", "-f", "1", "-s", "0", "-o", "x",
      "-r", "w.nii.gz"], "only linear transform files"),
    (["-d", "3", "-m", "CC[a,b,1,4]", "-t", "SyN[0.1,3,0]", "-c", "10", "-f", "1", "-s", "0", "-o", "x",
      "-r", "/nonexistent/a.mat"], "cannot open transform file"),
    (["-d", "3", "-m", "CC[a,b,1,4]", "-t", "SyN[0.1,3,0]", "-c", "10", "-f", "1", "-s", "0", "-o", "x",
      "-i", "1"], "--initialize-transforms-per-stage requires --write-composite-transform"),
    (["-d", "3", "-m", "CC[a,b,1,4]", "-t", "SyN[0.1,3,0]", "-c", "10", "-f", "1", "-s", "0", "-o", "x",
      "-a", "1", "-i", "1"], "mutually exclusive"),
    (["-d", "3", "-m", "CC[a,b,1,4]", "-t", "SyN[0.1,3,0]", "-c", "10", "-f", "1", "-s", "0", "-o", "x",
      "-q", "a.mat"], "initial-fixed-transform"),
    (["-d", "3", "-m", "CC[a,b,1,4]", "-t", "SyN[0.1,3,0]", "-c", "10", "-f", "1", "-s", "0", "-o", "x",
      "--minc", "1"], "MINC output"),
])
def test_cli_rejects_bad_input(cli, args, needle):
    r = run(cli, args)
    assert r.returncode == 1
    assert needle in r.stderr


def test_cli_rejects_an_initial_transform_with_a_field(cli, tmp_path):
    comp = tmp_path / "c.txt"
    comp.write_text("#Insight Transform File V1.0\n#Transform 0\nTransform: CompositeTransform_double_2_2\n"
                    "#Transform 1\nTransform: DisplacementFieldTransform_float_2_2\nParameters: 0 0 0 0 0 0 0 0\n"
                    "FixedParameters: 2 2 0 0 1 1 1 0 0 1\n")
    r = run(cli, ["-d", "2", "--float", "1", "-m", "CC[a,b,1,4]", "-t", "SyN[0.1,3,0]", "-c", "10", "-f", "1", "-s", "0",
                  "-o", "x", "-r", str(comp)])
    assert r.returncode == 1 and "holds a displacement field" in r.stderr, r.stderr


def test_cli_options_it_keeps_but_does_not_implement(cli):
    # the reference's parser keeps unknown options and goes on; this one does too, and says so. Its
    # other options are accepted (-p, -l, --write-interval-volumes, --minc 0, --random-seed, --version);
    # the non-zero intervals draw a warning. The run then stops at the missing images, before device work.
    r = run(cli, ["--version"])
    assert r.returncode == 0 and "antsRegistrationSyN_b200" in r.stdout
    base = ["-d", "3", "--float", "1", "-m", "CC[/nonexistent/f.nii.gz,/nonexistent/m.nii.gz,1,4]",
            "-t", "SyN[0.1,3,0]", "-c", "10", "-f", "1", "-s", "0", "-o", "x"]
    r = run(cli, base + ["--convergance", "[5,1e-6,10]", "-p", "5", "--write-interval-volumes", "3", "-l", "1",
                         "--minc", "0", "--random-seed", "7"])
    assert r.returncode == 1 and "cannot open" in r.stderr, r.stderr
    assert "unknown option --convergance ignored" in r.stderr
    assert "--print-similarity-measure-interval 5 is not implemented" in r.stderr
    assert "--write-interval-volumes 3 is not implemented" in r.stderr
    assert "unexpected argument" not in r.stderr and "--use-estimate" not in r.stderr
    r = run(cli, base + ["-p", "0", "--write-interval-volumes", "0"])
    assert "WARNING" not in r.stderr, r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("dim,size,radius", [(2, (64, 60), 2), (3, (30, 28, 26), 4)])
def test_cli_matches_python_api(cli, tmp_path, cuda, dim, size, radius):
    f, m = (phantoms.pair_2d(size, seed=4) if dim == 2 else phantoms.pair_3d(size, seed=4))
    g = Geom(size, (1.0,) * dim, (2.0,) * dim)
    nifti.write(tmp_path / "f.nii.gz", f, g)
    nifti.write(tmp_path / "m.nii.gz", m, g)
    prefix = str(tmp_path / "out_")
    r = run(cli, ["-d", str(dim), "--float", "1", "-v", "1", "-m", f"CC[{tmp_path}/f.nii.gz,{tmp_path}/m.nii.gz,1,{radius}]",
                  "-t", "SyN[0.2,3,0]", "-c", "[8x4,1e-12,10]", "-f", "2x1", "-s", "1x0vox",
                  "-o", f"[{prefix},{prefix}warped.nii.gz,{prefix}inverse_warped.nii.gz]"])
    assert r.returncode == 0, r.stderr
    assert "1DIAGNOSTIC" in r.stdout
    fwd, gf = nifti.read(prefix + "0Warp.nii.gz", dim)
    inv, _ = nifti.read(prefix + "0InverseWarp.nii.gz", dim)
    assert gf.size == g.size and np.allclose(gf.origin, g.origin)
    P = SyNParams(dim=dim, learning_rate=0.2, cc_radius=radius, iterations=(8, 4), shrink_factors=(2, 1),
                  smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12)
    with SyNStage(P) as st:
        st.set_images(f, g, m, g)
        st.run()
        a, b = st.fields()
    np.testing.assert_array_equal(fwd, a)
    np.testing.assert_array_equal(inv, b)
    warped, _ = nifti.read(prefix + "warped.nii.gz", dim)
    assert warped.shape == f.shape and np.isfinite(warped).all()
    # the warped moving image is closer to the fixed image than the moving image was
    assert np.abs(warped - f).mean() < np.abs(m - f).mean()
