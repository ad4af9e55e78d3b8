"""The antsApplyTransforms-compatible front end (ants_b200/antsApplyTransforms_b200): argument
checks, the default value outside the input, and agreement with the registration's own warped
output.  Stacks of several transforms are tested in test_zz_stack_apply.py."""
import os
import subprocess

import numpy as np
import pytest

from ants_b200 import nifti, phantoms
from ants_b200.synx import Geom

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APPLY = os.path.join(ROOT, "ants_b200", "antsApplyTransforms_b200")
REG = os.path.join(ROOT, "ants_b200", "antsRegistrationSyN_b200")


@pytest.fixture(scope="module")
def exe():
    from ants_b200 import build
    build.build_all()
    assert os.path.exists(APPLY)
    return APPLY


def run(exe, args):
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=600)


@pytest.mark.parametrize("args,needle", [
    (["-d", "3", "-i", "a.nii.gz", "-o", "x.nii.gz", "-t", "w.nii.gz"], "reference image"),
    (["-d", "3", "-i", "a.nii.gz", "-r", "a.nii.gz", "-o", "x.nii.gz", "-t", "[w.nii.gz,1]"], "inverse warp"),
    (["-d", "3", "-i", "a.nii.gz", "-r", "a.nii.gz", "-o", "x.nii.gz", "-t", "composite.h5"], "not supported"),
    (["-d", "3", "-i", "a.nii.gz", "-r", "a.nii.gz", "-o", "x.nii.gz", "-n", "BSpline[3]"], "NearestNeighbor"),
    (["-d", "5", "-i", "a.nii.gz", "-r", "a.nii.gz", "-o", "x.nii.gz"], "dimensionality"),
    (["-d", "3", "-e", "2", "-i", "a.nii.gz", "-r", "a.nii.gz", "-o", "x.nii.gz"], "multichannel (4)"),
    (["-d", "3", "-i", "a.nii.gz", "-r", "a.nii.gz", "-o", "CompositeTransform[x.h5]"], "HDF5 (.h5) is not available"),
    (["-d", "3", "-i", "a.nii.gz", "-r", "/nonexistent/r.nii.gz", "-o", "x.nii.gz"], "cannot open"),
])
def test_rejects_bad_input(exe, args, needle):
    r = run(exe, args)
    assert r.returncode == 1
    assert needle in r.stderr


@pytest.mark.gpu
def test_default_value_outside(exe, tmp_path, cuda):
    check_default_value_outside(exe, tmp_path)


def check_default_value_outside(exe, tmp_path):
    g = Geom((40, 36))
    img = np.full(g.shape, 5.0, np.float32)
    u = np.zeros(g.shape + (2,), np.float32)
    u[..., 0] = 100.0  # every point leaves the image
    u[:, :10, 0] = 0.0  # except the first ten columns
    nifti.write(tmp_path / "in.nii.gz", img, g)
    nifti.write(tmp_path / "u.nii.gz", u, g, vector=True)
    r = run(exe, ["-d", "2", "-i", f"{tmp_path}/in.nii.gz", "-r", f"{tmp_path}/in.nii.gz", "-t", f"{tmp_path}/u.nii.gz",
                  "-f", "-7", "-o", f"{tmp_path}/o.nii.gz"])
    assert r.returncode == 0, r.stderr
    got, _ = nifti.read(tmp_path / "o.nii.gz", 2)
    np.testing.assert_allclose(got[:, :10], 5.0, atol=1e-5)
    np.testing.assert_array_equal(got[:, 10:], -7.0)


@pytest.mark.gpu
def test_reproduces_the_registration_output(exe, tmp_path, cuda):
    check_reproduces_the_registration_output(REG, exe, tmp_path)


def check_reproduces_the_registration_output(reg, exe, tmp_path):
    # resampling the moving image through prefix0Warp gives antsRegistration's warped output
    size = (64, 60)
    f, m = phantoms.pair_2d(size, seed=31)
    g = Geom(size)
    nifti.write(tmp_path / "f.nii.gz", f, g)
    nifti.write(tmp_path / "m.nii.gz", m, g)
    p = str(tmp_path / "r_")
    r = subprocess.run([reg, "-d", "2", "-m", f"CC[{tmp_path}/f.nii.gz,{tmp_path}/m.nii.gz,1,2]", "-t", "SyN[0.2,3,0]",
                        "-c", "[8x4,1e-12,10]", "-f", "2x1", "-s", "1x0vox", "-o", f"[{p},{p}warped.nii.gz]"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    r = run(exe, ["-d", "2", "-i", f"{tmp_path}/m.nii.gz", "-r", f"{tmp_path}/f.nii.gz", "-t", p + "0Warp.nii.gz",
                  "-o", f"{tmp_path}/aat.nii.gz", "-v", "1"])
    assert r.returncode == 0, r.stderr
    a, _ = nifti.read(tmp_path / "aat.nii.gz", 2)
    b, _ = nifti.read(p + "warped.nii.gz", 2)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("patch,needle", [
    ({40: [3, 3000, 3000, 3000]}, "short read"),        # dim[]: claims 2.7e10 voxels in a small file
    ({40: [7, 4, 4, 3, 1, 1, 2, 1]}, "dimensions 6 and 7"),
])
def test_corrupt_headers_fail_cleanly(exe, tmp_path, patch, needle):
    # a NIfTI-1 header is read field by field: dim (int16[8]) at byte 40
    g = Geom((5, 4, 3))
    nifti.write(tmp_path / "ok.nii", np.ones(g.shape, np.float32), g)
    raw = bytearray((tmp_path / "ok.nii").read_bytes())
    for off, vals in patch.items():
        raw[off:off + 2 * len(vals)] = np.asarray(vals, "<i2").tobytes()
    (tmp_path / "bad.nii").write_bytes(bytes(raw))
    r = run(exe, ["-d", "3", "-i", f"{tmp_path}/ok.nii", "-r", f"{tmp_path}/bad.nii", "-o", f"{tmp_path}/o.nii.gz"])
    assert r.returncode == 1
    assert needle in r.stderr



def test_collapse_linear_stack(exe, tmp_path):
    """-o Linear[out.mat,invert]: an all-linear stack (first -t acting first) written as one affine;
    the center is that of the first transform acting (CollapseLinearTransforms); the inverse is
    written with center 0, as the reference builds it.  No GPU is involved."""
    from scipy.spatial.transform import Rotation

    from ants_b200 import synx
    from ants_b200.synx import LinearTransform
    A = LinearTransform(np.array([[1.05, 0.08, -0.03], [-0.06, 0.97, 0.04], [0.02, -0.05, 1.02]]),
                        np.array([2.5, -1.25, 3.0]), np.array([10.0, -4.0, 7.5]))
    B = LinearTransform(Rotation.from_euler("xyz", [0.1, -0.2, 0.3]).as_matrix(), np.array([1.0, 2.0, -0.5]),
                        np.array([3.0, 3.0, 3.0]))
    synx.write_linear_transform(tmp_path / "A.mat", A)
    synx.write_linear_transform(tmp_path / "B.txt", B)

    def mp(t):
        return t.matrix, t.translation + t.center - t.matrix @ t.center

    (MA, bA), (MB, bB) = mp(A), mp(B)
    M, b = MB @ MA, MB @ bA + bB  # A acts first, then B
    for inv, name in (("0", "c.mat"), ("1", "ci.mat")):
        r = run(exe, ["-d", "3", "-t", f"{tmp_path}/A.mat", "-t", f"{tmp_path}/B.txt", "-o",
                      f"Linear[{tmp_path}/{name},{inv}]"])
        assert r.returncode == 0, r.stderr
        t = synx.read_linear_transform(tmp_path / name, 3)
        Mt, bt = mp(t)
        if inv == "0":
            np.testing.assert_allclose(Mt, M, atol=1e-12)
            np.testing.assert_allclose(bt, b, atol=1e-10)
            np.testing.assert_array_equal(t.center, A.center)
        else:
            np.testing.assert_allclose(Mt, np.linalg.inv(M), atol=1e-12)
            np.testing.assert_allclose(bt, -np.linalg.inv(M) @ b, atol=1e-10)
            np.testing.assert_array_equal(t.center, 0.0)
    synx.write_linear_transform(tmp_path / "u.mat", A)
    g = Geom((4, 4, 4))
    nifti.write(tmp_path / "f.nii.gz", np.zeros(g.shape + (3,), np.float32), g, vector=True)
    r = run(exe, ["-d", "3", "-t", f"{tmp_path}/f.nii.gz", "-t", f"{tmp_path}/u.mat", "-o", f"Linear[{tmp_path}/x.mat]"])
    assert r.returncode == 1 and "displacement field" in r.stderr
