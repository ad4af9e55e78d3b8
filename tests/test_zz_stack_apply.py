"""antsApplyTransforms_b200 transform stacks -- order, linear transforms folded into grid geometry,
every transform applied at the displaced point, the collapsed field -- and the command lines' other
options: label interpolation, multichannel and time-series inputs, output types, and
antsRegistrationSyN_b200's initial moving transforms.

The reference applies the FIRST -t to a reference point first (its parser stores repeated options
newest first, Utilities/antsCommandLineOption.cxx:42,64, and an ITK composite applies the transform
added last first), so `-t 1Warp -t 0GenericAffine.mat` samples the input at A(p + u(p)).

`chain_displacement` is the reference's composite applied point by point: each field sampled on its
own grid (the oracle's warp, the interpolation ITK's displacement-field transform uses), each linear
transform applied analytically.  `emulate_cli` is the command line's scheme restated with the
oracle's step functions: leading linear transforms folded into the evaluation grid, trailing ones
into the input image's geometry, the middle applied transform by transform at the displaced point.
CPU tests check the scheme against the composite on every tested stack shape; GPU tests (and, through
host stand-ins, tests/test_cli_host_plumbing.py) check the command lines against the scheme.  This
file is collected after the tests already verified on the device, so that a run which stops at the
first failure has already run them.
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


def planes(u):
    return np.ascontiguousarray(np.moveaxis(u, -1, 0))


def points(g: Geom) -> np.ndarray:
    """Physical point of every voxel as component planes, shape (dim,) + g.shape."""
    axes = np.meshgrid(*[np.arange(n) for n in reversed(g.size)], indexing="ij")
    idx = np.stack(list(reversed(axes)), -1).astype(np.float64)
    return planes(np.asarray(g.origin) + (idx * np.asarray(g.spacing)) @ g.direction.T)


class Affine:
    """p -> M p + b, with the ITK parameters it is written with: A, t, c (M = A, b = t + c - A c)."""

    def __init__(self, A, t, c):
        self.A, self.t, self.c = np.asarray(A, float), np.asarray(t, float), np.asarray(c, float)
        self.M, self.b = self.A, self.t + self.c - self.A @ self.c

    def inverse(self):
        Mi = np.linalg.inv(self.M)
        r = Affine.__new__(Affine)
        r.M, r.b = Mi, -Mi @ self.b
        return r

    def apply(self, P):  # planes
        return np.tensordot(self.M, P, axes=1) + self.b.reshape((-1,) + (1,) * (P.ndim - 1))

    def write_mat(self, path):  # ITK MATLAB v4 form: parameters (A row-major, t), then "fixed" (c)
        d = len(self.t)
        with open(path, "wb") as fh:
            for var, vals in ((f"AffineTransform_double_{d}_{d}", np.r_[self.A.ravel(), self.t]), ("fixed", self.c)):
                nm = var.encode() + b"\0"
                fh.write(np.array([0, len(vals), 1, 0, len(nm)], "<i4").tobytes() + nm +
                         np.asarray(vals, "<f8").tobytes())


def push_forward(g: Geom, L) -> Geom:
    """The grid whose voxel i sits at L(p_i)."""
    return Geom(g.size, g.spacing, tuple(L.M @ np.asarray(g.origin) + L.b), L.M @ g.direction)


def chain_displacement(chain, gr: Geom) -> np.ndarray:
    """Displacement of every reference voxel under the chain (application order), planes."""
    P = points(gr)
    D = np.zeros_like(P)
    for kind, obj in chain:
        if kind == "field":
            d, gd = obj  # planes on their own grid
            D = D + np.stack([O.warp_image(np.ascontiguousarray(d[c]), gd, D, gr, dtype=np.float64)
                              for c in range(gr.dim)])
        else:
            D = obj.apply(P + D) - P
    return D


def emulate_cli(chain, gr: Geom, img=None, gi=None):
    """The command line's scheme with the oracle's step functions.  Returns the collapsed field
    (planes) and, with an input image, the warped image."""
    fields = [k for k, (kind, _) in enumerate(chain) if kind == "field"]
    lead_end = fields[0] if fields else len(chain)
    tail_begin = fields[-1] + 1 if fields else len(chain)
    dim = gr.dim
    pre = Affine(np.eye(dim), np.zeros(dim), np.zeros(dim))
    post = Affine(np.eye(dim), np.zeros(dim), np.zeros(dim))
    for k in range(lead_end):
        L = chain[k][1]
        pre.M, pre.b = L.M @ pre.M, L.M @ pre.b + L.b
    for k in range(tail_begin, len(chain)):
        L = chain[k][1]
        post.M, post.b = L.M @ post.M, L.M @ post.b + L.b
    ge = push_forward(gr, pre)

    def same(a, b):
        return (a.size == b.size and np.array_equal(a.spacing, b.spacing) and np.array_equal(a.origin, b.origin)
                and np.array_equal(a.direction, b.direction))

    w = np.zeros((dim,) + gr.shape, np.float32)
    for k in range(lead_end, tail_begin):
        kind, obj = chain[k]
        if kind == "field":
            d, gd = obj
            if k == lead_end:  # the first field, sampled at the evaluation grid's points
                w = d.copy() if same(gd, ge) else O.resample_field(d, gd, ge)
            elif same(gd, ge):  # w + d(x + w)
                w = O.compose(d, w, ge)
            else:  # d sampled on its own grid at x + w, then added
                w = (w + np.stack([O.warp_image(np.ascontiguousarray(d[c]), gd, w, ge) for c in range(dim)])
                     ).astype(np.float32)
        else:  # T(x + w) - x = (T(x) - x) + A w
            P = points(ge)
            w = (obj.apply(P) - P + np.tensordot(obj.M, w, axes=1)).astype(np.float32)
    P = points(gr)
    collapsed = (post.apply(pre.apply(P) + w) - P).astype(np.float32)
    warped = None
    if img is not None:
        warped = O.warp_image(img, push_forward(gi, post.inverse()), w, ge)
    return collapsed, warped


def field_on(g, sigma, max_norm, seed):
    return planes(phantoms.smooth_field(g.shape, sigma, max_norm, np.random.default_rng(seed)).astype(np.float32))


def affine(dim, k):
    if dim == 3:
        A = [[1.03, 0.05, -0.02], [-0.04, 0.98, 0.03], [0.01, -0.03, 1.01]] if k == 0 else \
            [[0.97, -0.02, 0.04], [0.03, 1.02, -0.01], [-0.02, 0.05, 0.99]]
        return Affine(A, [1.5, -1.0, 0.75] if k == 0 else [-2.0, 0.5, 1.25], [18.0, 16.0, 15.0])
    A = [[0.97, 0.06], [-0.05, 1.02]] if k == 0 else [[1.04, -0.03], [0.05, 0.96]]
    return Affine(A, [1.25, -0.75] if k == 0 else [-0.5, 1.0], [31.0, 27.0])


def grids(dim):
    g = Geom((60, 52) if dim == 2 else (34, 30, 28), (1.0,) * dim, (2.0,) * dim)          # fixed grid
    gm = Geom((64, 56) if dim == 2 else (36, 32, 30), (0.9,) * dim, (-1.0,) * dim)        # moving grid
    return g, gm


def cases(dim):
    """(name, chain, reference grid, scheme exact?) with the command-line spelling of each chain."""
    g, gm = grids(dim)
    a, b = field_on(g, 4.0, 2.0, 60 + dim), field_on(g, 5.0, 2.5, 70 + dim)
    inv = field_on(g, 4.0, 2.0, 80 + dim)  # an inverse warp lives on the fixed grid too
    c = field_on(gm, 4.0, 2.0, 85 + dim)   # a field on the moving grid
    A, B = affine(dim, 0), affine(dim, 1)
    return {
        # two fields on the reference grid: a first, then b
        "fields": ([("field", (a, g)), ("field", (b, g))], g, ["a", "b"]),
        # the forward standard stack on the fixed grid: warp first, then the affine
        "forward": ([("field", (a, g)), ("linear", A)], g, ["a", "A.mat"]),
        # the inverse standard stack on the moving grid: the affine's inverse first, then the inverse warp
        "inverse": ([("linear", A.inverse()), ("field", (inv, g))], gm, ["[A.mat,1]", "inv"]),
        # linear transforms only: A first, then B
        "linear": ([("linear", A), ("linear", B)], gm, ["A.mat", "B.mat"]),
        # affine, field, affine: both ends folded
        "both_ends": ([("linear", B.inverse()), ("field", (a, g)), ("linear", A)], gm, ["[B.mat,1]", "a", "A.mat"]),
        # an affine between two fields: applied at the displaced point, T(x + w) - x = (T(x) - x) + A w
        "sandwiched": ([("field", (a, g)), ("linear", A), ("field", (b, g))], g, ["a", "A.mat", "b"]),
        # a later field on another grid than the evaluation grid: sampled on its own grid at x + w
        "other_grid": ([("field", (a, g)), ("field", (c, gm))], g, ["a", "c"]),
    }, dict(a=a, b=b, c=c, inv=inv, A=A, B=B, g=g, gm=gm)


@pytest.mark.parametrize("dim", [2, 3])
def test_scheme_is_the_composite(dim):
    cs, _ = cases(dim)
    for name, (chain, gr, _) in cs.items():
        want = chain_displacement(chain, gr)
        got, _ = emulate_cli(chain, gr)
        bad = np.abs(got - want) > 1e-4
        assert bad.mean() < 1e-3, (name, float(np.abs(got - want).max()))


def test_order_is_first_given_first_applied():
    g, _ = grids(2)
    a, b = field_on(g, 4.0, 2.0, 1), field_on(g, 5.0, 2.5, 2)
    ab = chain_displacement([("field", (a, g)), ("field", (b, g))], g)
    np.testing.assert_allclose(ab, O.compose(b, a, g), atol=1e-5)  # a + b(x + a)
    ba = chain_displacement([("field", (b, g)), ("field", (a, g))], g)
    assert np.abs(ab - ba).max() > 0.05


@pytest.fixture(scope="module")
def exe():
    from ants_b200 import build
    build.build_all()
    assert os.path.exists(APPLY)
    return APPLY


def run(exe, args):
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=600)


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_stacks_match_the_scheme(exe, tmp_path, cuda, dim):
    check_stacks_match_the_scheme(exe, tmp_path, dim)


def check_stacks_match_the_scheme(exe, tmp_path, dim):
    cs, parts = cases(dim)
    g, gm = parts["g"], parts["gm"]  # the grid objects the cases refer to
    files = {"a": (parts["a"], g), "b": (parts["b"], g), "inv": (parts["inv"], g), "c": (parts["c"], gm)}
    for name, (u, gu) in files.items():
        nifti.write(tmp_path / f"{name}.nii.gz", np.ascontiguousarray(np.moveaxis(u, 0, -1)), gu, vector=True)
    parts["A"].write_mat(tmp_path / "A.mat")
    parts["B"].write_mat(tmp_path / "B.mat")
    nifti.write(tmp_path / "fixed.nii.gz", np.zeros(g.shape, np.float32), g)
    nifti.write(tmp_path / "moving.nii.gz", np.zeros(gm.shape, np.float32), gm)
    gi = Geom((70, 64) if dim == 2 else (40, 36, 32), (0.8,) * dim, (-3.0,) * dim)  # the input's own grid
    img = np.random.default_rng(90 + dim).uniform(0, 1, gi.shape).astype(np.float32)
    nifti.write(tmp_path / "in.nii.gz", img, gi)

    def spell(tok):
        if tok.startswith("["):
            return f"[{tmp_path}/{tok[1:].split(',')[0]},1]"
        return f"{tmp_path}/{tok}" + ("" if tok.endswith(".mat") else ".nii.gz")

    for name, (chain, gr, toks) in cs.items():
        assert gr is g or gr is gm
        ref = tmp_path / ("fixed.nii.gz" if gr is g else "moving.nii.gz")
        ts = sum((["-t", spell(t)] for t in toks), [])
        want_field, want_img = emulate_cli(chain, gr, img, gi)
        r = run(exe, ["-d", str(dim), "-r", str(ref), "-i", f"{tmp_path}/in.nii.gz", *ts, "-o", f"{tmp_path}/o.nii.gz"])
        assert r.returncode == 0, (name, r.stderr)
        got, go = nifti.read(tmp_path / "o.nii.gz", dim)
        assert go.size == gr.size
        # float vs double index arithmetic moves interpolation weights by a few ulps and rim points
        # may fall either side, so a small share of voxels may differ (as in the step tests)
        bad = np.abs(got - want_img) > 1e-4
        assert bad.mean() < 2e-3, (name, int(bad.sum()))
        r = run(exe, ["-d", str(dim), "-r", str(ref), *ts, "-o", f"[{tmp_path}/collapsed.nii.gz,1]"])
        assert r.returncode == 0, (name, r.stderr)
        collapsed, _ = nifti.read(tmp_path / "collapsed.nii.gz", dim)
        bad = np.abs(planes(collapsed) - want_field) > 1e-4
        assert bad.mean() < 2e-3, (name, int(bad.sum()))


REG = os.path.join(ROOT, "ants_b200", "antsRegistrationSyN_b200")


@pytest.mark.gpu
def test_multichannel_input(exe, tmp_path, cuda):
    check_multichannel(exe, tmp_path)


@pytest.mark.gpu
def test_time_series_input(exe, tmp_path, cuda):
    check_time_series(exe, tmp_path)


@pytest.mark.gpu
def test_output_data_types(exe, tmp_path, cuda):
    check_output_types(exe, tmp_path)


def check_output_types(exe, tmp_path):
    """-u: the warped image stored as a cast of the float result (truncation toward zero for integer
    types), with the matching NIfTI datatype code."""
    import struct
    g = Geom((30, 28))
    img = (np.random.default_rng(99).uniform(-40, 300, g.shape)).astype(np.float32)
    u = np.ascontiguousarray(np.moveaxis(field_on(g, 4.0, 2.0, 99), 0, -1))
    nifti.write(tmp_path / "in.nii.gz", img, g)
    nifti.write(tmp_path / "u.nii.gz", u, g, vector=True)
    base = ["-d", "2", "-i", f"{tmp_path}/in.nii.gz", "-r", f"{tmp_path}/in.nii.gz", "-t", f"{tmp_path}/u.nii.gz"]
    r = run(exe, base + ["-o", f"{tmp_path}/f.nii"])
    assert r.returncode == 0, r.stderr
    ref, _ = nifti.read(tmp_path / "f.nii", 2)
    for name, code, cast in (("char", 256, np.int8), ("uchar", 2, np.uint8), ("short", 4, np.int16),
                             ("int", 8, np.int32), ("double", 64, np.float64), ("float", 16, np.float32),
                             ("default", 64, np.float64)):  # default: the reference's computation type, double
        r = run(exe, base + ["-u", name, "-o", f"{tmp_path}/{name}.nii"])
        assert r.returncode == 0, (name, r.stderr)
        raw = (tmp_path / f"{name}.nii").read_bytes()
        assert struct.unpack("<h", raw[70:72])[0] == code, name  # datatype
        got, _ = nifti.read(tmp_path / f"{name}.nii", 2)
        want = ref.astype(np.float64) if cast in (np.float64, np.float32) else np.trunc(ref).astype(np.int64).astype(cast)
        np.testing.assert_array_equal(got, np.asarray(want, np.float32), err_msg=name)
    # with --float 1 the default type, and the collapsed field, are float
    r = run(exe, base + ["--float", "1", "-o", f"{tmp_path}/f1.nii"])
    assert r.returncode == 0 and struct.unpack("<h", (tmp_path / "f1.nii").read_bytes()[70:72])[0] == 16
    for flt, code in (("0", 64), ("1", 16)):
        r = run(exe, ["-d", "2", "-r", f"{tmp_path}/in.nii.gz", "-t", f"{tmp_path}/u.nii.gz", "--float", flt,
                      "-o", f"[{tmp_path}/col{flt}.nii,1]"])
        assert r.returncode == 0 and struct.unpack("<h", (tmp_path / f"col{flt}.nii").read_bytes()[70:72])[0] == code
    r = run(exe, base + ["-u", "long", "-o", f"{tmp_path}/x.nii"])
    assert r.returncode == 1 and "output-data-type" in r.stderr


def check_time_series(exe, tmp_path):
    """-e 3: every volume of a 4-D series resampled through `-t field -t affine.mat`, written back as a
    4-D series on the reference grid with the input's time step."""
    import struct
    cs, parts = cases(3)
    g = parts["g"]
    nifti.write(tmp_path / "a.nii.gz", np.ascontiguousarray(np.moveaxis(parts["a"], 0, -1)), g, vector=True)
    parts["A"].write_mat(tmp_path / "A.mat")
    nifti.write(tmp_path / "fixed.nii.gz", np.zeros(g.shape, np.float32), g)
    gi = Geom((40, 36, 32), (0.8,) * 3, (-3.0,) * 3)
    vols = np.random.default_rng(98).uniform(0, 1, gi.shape + (3,)).astype(np.float32)
    nifti.write(tmp_path / "ts.nii", vols, gi, time_series=True, time_step=2.5)
    r = run(exe, ["-d", "3", "-e", "3", "-r", f"{tmp_path}/fixed.nii.gz", "-i", f"{tmp_path}/ts.nii",
                  "-t", f"{tmp_path}/a.nii.gz", "-t", f"{tmp_path}/A.mat", "-o", f"{tmp_path}/o.nii"])
    assert r.returncode == 0, r.stderr
    raw = (tmp_path / "o.nii").read_bytes()
    dims = struct.unpack("<8h", raw[40:56])
    assert dims[0] == 4 and dims[4] == 3 and dims[5] == 1
    assert struct.unpack("<f", raw[92:96])[0] == 2.5  # pixdim[4]
    got, go = nifti.read(tmp_path / "o.nii", 3)
    assert got.shape == g.shape + (3,) and go.size == g.size
    gfold = push_forward(gi, parts["A"].inverse())
    for t in range(3):
        want = O.warp_image(np.ascontiguousarray(vols[..., t]), gfold, parts["a"], g)
        bad = np.abs(got[..., t] - want) > 1e-4
        assert bad.mean() < 2e-3, (t, int(bad.sum()))
    base = ["-r", f"{tmp_path}/fixed.nii.gz", "-t", f"{tmp_path}/a.nii.gz", "-o", f"{tmp_path}/x.nii"]
    for args, needle in ((["-d", "3", "-i", f"{tmp_path}/ts.nii"], "-e 3"),
                         (["-d", "3", "-e", "4", "-i", f"{tmp_path}/ts.nii"], "use -e 3"),
                         (["-d", "2", "-e", "3", "-i", f"{tmp_path}/ts.nii"], "needs -d 3")):
        r = run(exe, args + base)
        assert r.returncode == 1 and needle in r.stderr, (args, r.stderr)


def check_time_index(exe, tmp_path):
    """--time-index t with -e 3 (antsApplyTransforms.cxx:242-249, :283-317): volume t alone, resampled into
    a 3-D image, the same values as volume t of the whole series; out of range and without -e 3 as the
    reference treats them; -z and unknown options kept (the latter named on stderr)."""
    cs, parts = cases(3)
    g = parts["g"]
    nifti.write(tmp_path / "a.nii.gz", np.ascontiguousarray(np.moveaxis(parts["a"], 0, -1)), g, vector=True)
    parts["A"].write_mat(tmp_path / "A.mat")
    nifti.write(tmp_path / "fixed.nii.gz", np.zeros(g.shape, np.float32), g)
    gi = Geom((40, 36, 32), (0.8,) * 3, (-3.0,) * 3)
    vols = np.random.default_rng(99).uniform(0, 1, gi.shape + (3,)).astype(np.float32)
    nifti.write(tmp_path / "ts.nii", vols, gi, time_series=True, time_step=2.5)
    base = ["-d", "3", "-r", f"{tmp_path}/fixed.nii.gz", "-t", f"{tmp_path}/a.nii.gz", "-t", f"{tmp_path}/A.mat"]
    r = run(exe, base + ["-e", "3", "-i", f"{tmp_path}/ts.nii", "-o", f"{tmp_path}/all.nii"])
    assert r.returncode == 0, r.stderr
    whole, _ = nifti.read(tmp_path / "all.nii", 3)
    r = run(exe, base + ["-e", "3", "--time-index", "1", "-z", "1", "--bogus-option", "7", "-i", f"{tmp_path}/ts.nii",
                         "-o", f"{tmp_path}/t1.nii"])
    assert r.returncode == 0, r.stderr
    assert "unknown option --bogus-option ignored" in r.stderr and "static-cast" not in r.stderr
    one, go = nifti.read(tmp_path / "t1.nii", 3)
    assert one.shape == g.shape and go.size == g.size
    np.testing.assert_array_equal(one, whole[..., 1])
    r = run(exe, base + ["-e", "3", "--time-index", "3", "-i", f"{tmp_path}/ts.nii", "-o", f"{tmp_path}/t3.nii"])
    assert r.returncode == 1 and "out of range [0, 2]" in r.stderr, r.stderr
    # without -e 3 the reference does not read --time-index: a scalar input is resampled as usual
    nifti.write(tmp_path / "s.nii", np.ascontiguousarray(vols[..., 0]), gi)
    r = run(exe, base + ["--time-index", "2", "-i", f"{tmp_path}/s.nii", "-o", f"{tmp_path}/s_out.nii"])
    assert r.returncode == 0, r.stderr
    np.testing.assert_array_equal(nifti.read(tmp_path / "s_out.nii", 3)[0], whole[..., 0])


def check_multichannel(exe, tmp_path, dim=3):
    """-e 4: every channel of a multichannel image resampled through `-t field -t affine.mat`, written
    back as a multichannel image on the reference grid."""
    cs, parts = cases(dim)
    g = parts["g"]
    nifti.write(tmp_path / "a.nii.gz", np.ascontiguousarray(np.moveaxis(parts["a"], 0, -1)), g, vector=True)
    parts["A"].write_mat(tmp_path / "A.mat")
    nifti.write(tmp_path / "fixed.nii.gz", np.zeros(g.shape, np.float32), g)
    gi = Geom((40, 36, 32), (0.8,) * 3, (-3.0,) * 3)
    chans = np.random.default_rng(97).uniform(0, 1, gi.shape + (3,)).astype(np.float32)
    nifti.write(tmp_path / "mc.nii.gz", chans, gi, vector=True)
    r = run(exe, ["-d", "3", "-e", "4", "-r", f"{tmp_path}/fixed.nii.gz", "-i", f"{tmp_path}/mc.nii.gz",
                  "-t", f"{tmp_path}/a.nii.gz", "-t", f"{tmp_path}/A.mat", "-o", f"{tmp_path}/o.nii.gz"])
    assert r.returncode == 0, r.stderr
    got, go = nifti.read(tmp_path / "o.nii.gz", 3)
    assert got.shape == g.shape + (3,) and go.size == g.size
    gfold = push_forward(gi, parts["A"].inverse())
    for c in range(3):
        want = O.warp_image(np.ascontiguousarray(chans[..., c]), gfold, parts["a"], g)
        bad = np.abs(got[..., c] - want) > 1e-4
        assert bad.mean() < 2e-3, (c, int(bad.sum()))
    # a multichannel image without -e 4 is refused
    r = run(exe, ["-d", "3", "-r", f"{tmp_path}/fixed.nii.gz", "-i", f"{tmp_path}/mc.nii.gz",
                  "-t", f"{tmp_path}/a.nii.gz", "-o", f"{tmp_path}/o2.nii.gz"])
    assert r.returncode == 1 and "-e 4" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("interp", ["NearestNeighbor", "GenericLabel[Linear]"])
@pytest.mark.parametrize("dim", [2, 3])
def test_label_interpolation(exe, tmp_path, cuda, dim, interp):
    check_label_interpolation(exe, tmp_path, dim, interp)


def check_label_interpolation(exe, tmp_path, dim, interp="NearestNeighbor"):
    """-n NearestNeighbor / GenericLabel[Linear] through `-t field -t affine.mat`: the label image
    sampled at A(p + u(p)); a point on a rounding tie may pick either label."""
    cs, parts = cases(dim)
    chain, gr, toks = cs["forward"]
    g = parts["g"]
    nifti.write(tmp_path / "a.nii.gz", np.ascontiguousarray(np.moveaxis(parts["a"], 0, -1)), g, vector=True)
    parts["A"].write_mat(tmp_path / "A.mat")
    nifti.write(tmp_path / "fixed.nii.gz", np.zeros(g.shape, np.float32), g)
    gi = Geom((70, 64) if dim == 2 else (40, 36, 32), (0.8,) * dim, (-3.0,) * dim)
    labels = np.random.default_rng(95 + dim).integers(0, 9, gi.shape).astype(np.float32)
    nifti.write(tmp_path / "labels.nii.gz", labels, gi)
    r = run(exe, ["-d", str(dim), "-r", f"{tmp_path}/fixed.nii.gz", "-i", f"{tmp_path}/labels.nii.gz",
                  "-t", f"{tmp_path}/a.nii.gz", "-t", f"{tmp_path}/A.mat", "-n", interp,
                  "-o", f"{tmp_path}/o.nii.gz"])
    assert r.returncode == 0, r.stderr
    got, _ = nifti.read(tmp_path / "o.nii.gz", dim)
    want = O.warp_image(labels, push_forward(gi, parts["A"].inverse()), parts["a"], g,
                        nearest=interp == "NearestNeighbor", label=interp.startswith("GenericLabel"))
    assert set(np.unique(got)) <= set(range(9))
    bad = got != want
    assert bad.mean() < 2e-3, int(bad.sum())


@pytest.mark.gpu
def test_registration_with_an_initial_moving_transform(exe, tmp_path, cuda):
    check_initial_moving_transform(REG, exe, tmp_path)


@pytest.mark.gpu
def test_registration_with_a_derived_initial_translation(exe, tmp_path, cuda):
    check_derived_initial_translation(REG, tmp_path)


def check_initial_moving_transform(reg, exe, tmp_path):
    """antsRegistration -r init.mat: the moving image is sampled at Init(x + psi_M(x)); the outputs are
    numbered as the reference numbers them (0GenericAffine.mat, 1Warp, 1InverseWarp), and the warped
    images agree with antsApplyTransforms through the standard stacks."""
    from ants_b200 import synx
    from ants_b200.synx import SyNParams
    size = (64, 60)
    f, m = phantoms.pair_2d(size, seed=33)
    g = Geom(size)
    A = Affine([[1.02, 0.03], [-0.02, 0.99]], [0.8, -0.6], [32.0, 30.0])
    A.write_mat(tmp_path / "init.mat")
    nifti.write(tmp_path / "f.nii.gz", f, g)
    nifti.write(tmp_path / "m.nii.gz", m, g)
    p = str(tmp_path / "r_")
    r = run(reg, ["-d", "2", "-m", f"CC[{tmp_path}/f.nii.gz,{tmp_path}/m.nii.gz,1,2]", "-t", "SyN[0.2,3,0]",
                  "-c", "[8x4,1e-12,10]", "-f", "2x1", "-s", "1x0vox", "-r", f"{tmp_path}/init.mat",
                  "-o", f"[{p},{p}warped.nii.gz,{p}inverse_warped.nii.gz]"])
    assert r.returncode == 0, r.stderr
    assert os.path.exists(p + "1Warp.nii.gz") and os.path.exists(p + "1InverseWarp.nii.gz")
    assert not os.path.exists(p + "0Warp.nii.gz")
    back = synx.read_linear_transform(p + "0GenericAffine.mat", 2)
    np.testing.assert_allclose(back.matrix, A.A, atol=1e-12)
    np.testing.assert_allclose(back.center, A.c, atol=1e-12)
    np.testing.assert_allclose(back.translation, A.t, atol=1e-9)
    # the stage against the oracle with the initial transform folded into the moving geometry
    P = SyNParams(dim=2, learning_rate=0.2, cc_radius=2, iterations=(8, 4), shrink_factors=(2, 1),
                  smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12)
    rf, ri, _, _ = O.syn_register(f, g, m, push_forward(g, A.inverse()), P)
    fwd, _ = nifti.read(p + "1Warp.nii.gz", 2)
    inv, _ = nifti.read(p + "1InverseWarp.nii.gz", 2)
    for got, want in ((planes(fwd), rf), (planes(inv), ri)):
        assert float(np.sqrt(((got - want) ** 2).sum(0).mean())) <= 0.05
    assert float(np.sqrt((planes(fwd) ** 2).sum(0).mean())) > 0.02  # the stage did move
    # the warped outputs through antsApplyTransforms' standard stacks
    for ref_img, inp, ts, out in (("f", "m", [f"{p}1Warp.nii.gz", f"{p}0GenericAffine.mat"], "warped"),
                                  ("m", "f", [f"[{p}0GenericAffine.mat,1]", f"{p}1InverseWarp.nii.gz"],
                                   "inverse_warped")):
        r = run(exe, ["-d", "2", "-i", f"{tmp_path}/{inp}.nii.gz", "-r", f"{tmp_path}/{ref_img}.nii.gz",
                      "-t", ts[0], "-t", ts[1], "-o", f"{tmp_path}/aat_{out}.nii.gz"])
        assert r.returncode == 0, r.stderr
        a, _ = nifti.read(tmp_path / f"aat_{out}.nii.gz", 2)
        b, _ = nifti.read(f"{p}{out}.nii.gz", 2)
        bad = np.abs(a - b) > 1e-5
        assert bad.mean() < 1e-3, (out, int(bad.sum()))


@pytest.mark.gpu
def test_registration_output_precision(tmp_path, cuda):
    check_output_precision(REG, tmp_path)


def check_output_precision(reg, tmp_path):
    """The registration's fields and warped image are written as float64 by default and as float32 with
    --float 1, as the reference writes them; the values are the same float results either way."""
    import struct
    size = (40, 36)
    f, m = phantoms.pair_2d(size, seed=37)
    g = Geom(size)
    nifti.write(tmp_path / "f.nii.gz", f, g)
    nifti.write(tmp_path / "m.nii.gz", m, g)
    vals = {}
    for flt, code in (("0", 64), ("1", 16)):
        p = str(tmp_path / f"p{flt}_")
        r = run(reg, ["-d", "2", "--float", flt, "-m", f"CC[{tmp_path}/f.nii.gz,{tmp_path}/m.nii.gz,1,2]",
                      "-t", "SyN[0.2,3,0]", "-c", "[4x2,1e-12,10]", "-f", "2x1", "-s", "1x0vox",
                      "-o", f"[{p},{p}warped.nii]"])
        assert r.returncode == 0, r.stderr
        raw = (tmp_path / f"p{flt}_warped.nii").read_bytes()
        assert struct.unpack("<h", raw[70:72])[0] == code
        vals[flt] = (nifti.read(p + "0Warp.nii.gz", 2)[0], nifti.read(p + "warped.nii", 2)[0])
    np.testing.assert_array_equal(vals["0"][0], vals["1"][0])
    np.testing.assert_array_equal(vals["0"][1], vals["1"][1])


def check_derived_initial_translation(reg, tmp_path):
    """antsRegistration -r [fixed,moving,1]: the translation between the centers of intensity mass,
    folded into the moving geometry; collapsed into 0GenericAffine.mat, or with -z 0 written as
    0DerivedInitialMovingTranslation.mat, the SyN fields numbered 1 either way."""
    from ants_b200 import synx
    from ants_b200.synx import SyNParams
    size = (64, 60)
    f, m = phantoms.pair_2d(size, seed=35)
    g, gm = Geom(size), Geom(size, (1.0, 1.0), (1.5, -2.0))  # the moving image is shifted in space
    nifti.write(tmp_path / "f.nii.gz", f, g)
    nifti.write(tmp_path / "m.nii.gz", m, gm)
    t = synx.initial_translation(f, g, m, gm, 1)
    L = Affine(np.eye(2), t.translation, t.center)
    P = SyNParams(dim=2, learning_rate=0.2, cc_radius=2, iterations=(8, 4), shrink_factors=(2, 1),
                  smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12)
    rf, _, _, _ = O.syn_register(f, g, m, push_forward(gm, L.inverse()), P)
    for z, names in (("1", ["0GenericAffine.mat"]), ("0", ["0DerivedInitialMovingTranslation.mat"])):
        p = str(tmp_path / f"z{z}_")
        r = run(reg, ["-d", "2", "-m", f"CC[{tmp_path}/f.nii.gz,{tmp_path}/m.nii.gz,1,2]", "-t", "SyN[0.2,3,0]",
                      "-c", "[8x4,1e-12,10]", "-f", "2x1", "-s", "1x0vox", "-z", z,
                      "-r", f"[{tmp_path}/f.nii.gz,{tmp_path}/m.nii.gz,1]", "-o", p])
        assert r.returncode == 0, r.stderr
        for n in names + ["1Warp.nii.gz", "1InverseWarp.nii.gz"]:
            assert os.path.exists(p + n), n
        back = synx.read_linear_transform(p + names[0], 2)
        np.testing.assert_allclose(back.translation, t.translation, atol=1e-9)
        np.testing.assert_allclose(back.center, t.center, atol=1e-9)
        fwd, _ = nifti.read(p + "1Warp.nii.gz", 2)
        assert float(np.sqrt(((planes(fwd) - rf) ** 2).sum(0).mean())) <= 0.05
