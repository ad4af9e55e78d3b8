"""antsApplyTransforms_b200 with a linear transform file in its stack (ITK .mat, forward and inverse),
against the oracle's composition and warp.

The linear displacements come from synx_linear_field, the host function the command line feeds to
the composition, whose values and layout the CPU tests in test_linear_transforms.py pin.  This file
is collected last, after the allocation-free entry point's, so that a run which stops at the first
failure has already run every other test.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from ants_b200 import nifti, phantoms
from ants_b200.synx import Geom

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APPLY = os.path.join(ROOT, "ants_b200", "antsApplyTransforms_b200")


@pytest.fixture(scope="module")
def exe():
    from ants_b200 import build
    build.build_all()
    assert os.path.exists(APPLY)
    return APPLY


def run(exe, args):
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=600)


def field(g, sigma, max_norm, seed):
    u = phantoms.smooth_field(g.shape, sigma, max_norm, np.random.default_rng(seed))
    return u.astype(np.float32)  # interleaved: shape + (dim,)


def planes(u):
    return np.ascontiguousarray(np.moveaxis(u, -1, 0))


def linear_stack_case(dim, tmp_path):
    """Reference grid, input image, a field `a` and a linear transform (written as an ITK .mat file),
    with the oracle's expectations for `-t a -t aff.mat` (the affine moves a point first) and for
    `-t [aff.mat,1]`.  The linear displacements come from synx_linear_field, the host function
    antsApplyTransforms_b200 feeds to the composition."""
    from ants_b200 import synx
    from ants_b200.synx import LinearTransform
    g = Geom((60, 52) if dim == 2 else (34, 30, 28), (1.0,) * dim, (2.0,) * dim)
    gi = Geom((70, 64) if dim == 2 else (40, 36, 30), (0.9,) * dim, (-1.0,) * dim)
    img = np.random.default_rng(40 + dim).uniform(0, 1, gi.shape).astype(np.float32)
    a = field(g, 4.0, 2.0, 50 + dim)
    if dim == 3:
        A = np.array([[1.03, 0.05, -0.02], [-0.04, 0.98, 0.03], [0.01, -0.03, 1.01]])
        t = LinearTransform(A, np.array([1.5, -1.0, 0.75]), np.array([18.0, 16.0, 15.0]))
    else:
        A = np.array([[0.97, 0.06], [-0.05, 1.02]])
        t = LinearTransform(A, np.array([1.25, -0.75]), np.array([31.0, 27.0]))
    name = f"AffineTransform_double_{dim}_{dim}"
    with open(tmp_path / "aff.mat", "wb") as fh:  # MATLAB v4, little endian, double column vectors
        for var, vals in ((name, np.r_[t.matrix.ravel(), t.translation]), ("fixed", t.center)):
            nm = var.encode() + b"\0"
            fh.write(np.array([0, len(vals), 1, 0, len(nm)], "<i4").tobytes() + nm + np.asarray(vals, "<f8").tobytes())
    u_fwd = synx.linear_field(t, g)  # component planes, as the step functions take them
    u_inv = synx.linear_field(t, g, invert=True)
    w = O.compose(planes(a), u_fwd, g)  # the affine first, then a
    return g, gi, img, a, w, u_inv


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_linear_transform_in_the_stack(exe, tmp_path, cuda, dim):
    g, gi, img, a, w, u_inv = linear_stack_case(dim, tmp_path)
    nifti.write(tmp_path / "ref.nii.gz", np.zeros(g.shape, np.float32), g)
    nifti.write(tmp_path / "in.nii.gz", img, gi)
    nifti.write(tmp_path / "a.nii.gz", a, g, vector=True)
    base = ["-d", str(dim), "-r", f"{tmp_path}/ref.nii.gz"]
    # float vs double index arithmetic moves interpolation weights by a few ulps and rim points
    # may fall either side, so a small share of voxels may differ (as in the field-stack test)
    r = run(exe, base + ["-i", f"{tmp_path}/in.nii.gz", "-t", f"{tmp_path}/a.nii.gz", "-t", f"{tmp_path}/aff.mat",
                         "-o", f"{tmp_path}/o1.nii.gz", "-v", "1"])
    assert r.returncode == 0, r.stderr
    assert "(linear)" in r.stdout
    got, _ = nifti.read(tmp_path / "o1.nii.gz", dim)
    bad = np.abs(got - O.warp_image(img, gi, w, g)) > 1e-4
    assert bad.mean() < 1e-3, bad.sum()
    r = run(exe, base + ["-t", f"{tmp_path}/a.nii.gz", "-t", f"{tmp_path}/aff.mat", "-o", f"[{tmp_path}/c.nii.gz,1]"])
    assert r.returncode == 0, r.stderr
    c, _ = nifti.read(tmp_path / "c.nii.gz", dim)
    bad = np.abs(planes(c) - w) > 1e-4
    assert bad.mean() < 1e-3, bad.sum()
    # the inverse of the linear transform alone
    r = run(exe, base + ["-i", f"{tmp_path}/in.nii.gz", "-t", f"[{tmp_path}/aff.mat,1]", "-o", f"{tmp_path}/o2.nii.gz"])
    assert r.returncode == 0, r.stderr
    got, _ = nifti.read(tmp_path / "o2.nii.gz", dim)
    bad = np.abs(got - O.warp_image(img, gi, u_inv, g)) > 1e-4
    assert bad.mean() < 1e-3, bad.sum()
