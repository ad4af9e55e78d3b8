"""Linear transforms of ITK transform files (synx_read_linear_transform) and their displacement
fields (synx_linear_field): host-only entry points of the C ABI, checked on the CPU against
numpy and scipy's rotation conventions.  The files are written here in the two forms ITK's
transform IO uses: MATLAB v4 binary (.mat) and Insight text (.txt, the layout of
Scripts/ANTSAverage3DAffine.sh:94-98)."""
import ctypes as C
import os
import struct
import subprocess

import numpy as np
import pytest
from scipy.spatial.transform import Rotation

from ants_b200 import synx
from ants_b200.synx import Geom, LinearTransform, SynxError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APPLY = os.path.join(ROOT, "ants_b200", "antsApplyTransforms_b200")


def write_mat(path, variables, big=False, single=False, rowwise=False):
    """MATLAB v4: per variable a header (type, rows, cols, imagf, namelen), the name with its NUL,
    then the values.  type = 1000 M + 100 O + 10 P (M byte order, O storage order, P precision)."""
    e = ">" if big else "<"
    with open(path, "wb") as fh:
        for name, vals in variables:
            vals = np.asarray(vals, dtype=np.float64).ravel()
            typ = (1000 if big else 0) + (100 if rowwise else 0) + (10 if single else 0)
            nm = name.encode() + b"\0"
            fh.write(struct.pack(e + "5i", typ, len(vals), 1, 0, len(nm)))
            fh.write(nm)
            fh.write(vals.astype(e + ("f4" if single else "f8")).tobytes())


def write_txt(path, transforms):
    lines = ["#Insight Transform File V1.0 "]
    for i, (name, params, fixed) in enumerate(transforms):
        lines += [f"# Transform {i} ", f"Transform: {name}  ",
                  "Parameters:  " + " ".join(repr(float(v)) for v in params) + "  ",
                  "FixedParameters: " + " ".join(repr(float(v)) for v in fixed) + " "]
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def physical_points(g: Geom) -> np.ndarray:
    """p = origin + D diag(spacing) index at every voxel, shape g.shape + (dim,)."""
    axes = np.meshgrid(*[np.arange(n) for n in reversed(g.size)], indexing="ij")
    idx = np.stack(list(reversed(axes)), -1).astype(np.float64)  # (..., dim) in x, y, z order
    return np.asarray(g.origin) + (idx * np.asarray(g.spacing)) @ g.direction.T


def apply(t: LinearTransform, p: np.ndarray, inverse=False) -> np.ndarray:
    if inverse:
        return (p - t.translation - t.center) @ np.linalg.inv(t.matrix).T + t.center
    return (p - t.center) @ t.matrix.T + t.translation + t.center


AFFINE3 = np.array([1.05, 0.08, -0.03, -0.06, 0.97, 0.04, 0.02, -0.05, 1.02])
TRANS3 = np.array([2.5, -1.25, 3.0])
CENTER3 = np.array([10.0, -4.0, 7.5])


@pytest.mark.parametrize("big,single,rowwise", [(False, False, False), (True, False, False), (False, True, False),
                                                (False, False, True)])
def test_read_affine_mat(tmp_path, big, single, rowwise):
    p = tmp_path / "a.mat"
    name = "AffineTransform_float_3_3" if single else "AffineTransform_double_3_3"
    write_mat(p, [(name, np.r_[AFFINE3, TRANS3]), ("fixed", CENTER3)], big=big, single=single, rowwise=rowwise)
    assert synx.count_linear_transforms(p, 3) == 1
    t = synx.read_linear_transform(p, 3)
    tol = 1e-7 if single else 0.0
    np.testing.assert_allclose(t.matrix, AFFINE3.reshape(3, 3), atol=tol)
    np.testing.assert_allclose(t.translation, TRANS3, atol=tol)
    np.testing.assert_allclose(t.center, CENTER3, atol=tol)


def test_read_text_form_of_the_reference_script(tmp_path):
    p = tmp_path / "avg.txt"
    write_txt(p, [("MatrixOffsetTransformBase_double_3_3", np.r_[AFFINE3, TRANS3], CENTER3)])
    t = synx.read_linear_transform(p, 3)
    np.testing.assert_array_equal(t.matrix, AFFINE3.reshape(3, 3))
    np.testing.assert_array_equal(t.translation, TRANS3)
    np.testing.assert_array_equal(t.center, CENTER3)


def test_rotation_types_follow_itk_conventions(tmp_path):
    ax, ay, az = 0.3, -0.2, 0.45
    c = [1.0, 2.0, 3.0]
    cases = [
        # Euler3DTransform: A = Rz Rx Ry (rotate about y, then x, then z, fixed axes)
        ("Euler3DTransform_double_3_3", [ax, ay, az, 1, 2, 3], c, Rotation.from_euler("yxz", [ay, ax, az]).as_matrix()),
        # with the fourth fixed parameter set: A = Rz Ry Rx
        ("Euler3DTransform_double_3_3", [ax, ay, az, 1, 2, 3], c + [1.0],
         Rotation.from_euler("xyz", [ax, ay, az]).as_matrix()),
        ("VersorRigid3DTransform_double_3_3", [0.1, -0.2, 0.15, 1, 2, 3], c,
         Rotation.from_quat([0.1, -0.2, 0.15, np.sqrt(1 - 0.1**2 - 0.2**2 - 0.15**2)]).as_matrix()),
        ("Similarity3DTransform_double_3_3", [0.1, -0.2, 0.15, 1, 2, 3, 1.3], c,
         1.3 * Rotation.from_quat([0.1, -0.2, 0.15, np.sqrt(1 - 0.1**2 - 0.2**2 - 0.15**2)]).as_matrix()),
        ("TranslationTransform_double_3_3", [1, 2, 3], [], np.eye(3)),
    ]
    for i, (name, params, fixed, A) in enumerate(cases):
        p = tmp_path / f"r{i}.txt"
        write_txt(p, [(name, params, fixed)])
        t = synx.read_linear_transform(p, 3)
        np.testing.assert_allclose(t.matrix, A, atol=1e-12, err_msg=name)
        np.testing.assert_allclose(t.translation, [1, 2, 3], err_msg=name)
        np.testing.assert_allclose(t.center, fixed[:3] if fixed else [0, 0, 0], err_msg=name)
    th = 0.4
    R = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
    for name, params, A in [("Euler2DTransform_double_2_2", [th, 5, -6], R),
                            ("Rigid2DTransform_double_2_2", [th, 5, -6], R),
                            ("Similarity2DTransform_double_2_2", [0.8, th, 5, -6], 0.8 * R)]:
        p = tmp_path / f"{name}.mat"
        write_mat(p, [(name, params), ("fixed", [3.0, 4.0])])
        t = synx.read_linear_transform(p, 2)
        np.testing.assert_allclose(t.matrix, A, atol=1e-12, err_msg=name)
        np.testing.assert_allclose(t.translation, [5, -6])
        np.testing.assert_allclose(t.center, [3, 4])
    write_txt(tmp_path / "id.txt", [("IdentityTransform_double_3_3", [], [])])
    t = synx.read_linear_transform(tmp_path / "id.txt", 3)
    np.testing.assert_array_equal(t.matrix, np.eye(3))
    np.testing.assert_array_equal(t.translation, 0)


def test_composite_file_lists_components_in_order(tmp_path):
    p = tmp_path / "comp.txt"
    write_txt(p, [("CompositeTransform_double_3_3", [], []),
                  ("TranslationTransform_double_3_3", [1, 0, 0], []),
                  ("AffineTransform_double_3_3", np.r_[AFFINE3, TRANS3], CENTER3)])
    assert synx.count_linear_transforms(p, 3) == 2
    np.testing.assert_array_equal(synx.read_linear_transform(p, 3, 0).translation, [1, 0, 0])
    np.testing.assert_array_equal(synx.read_linear_transform(p, 3, 1).matrix, AFFINE3.reshape(3, 3))


@pytest.mark.parametrize("content,needle,code", [
    ("txt:BSplineTransform_double_3_3", "not supported", -5),
    ("txt:AffineTransform_double_2_2", "not a 3-D transform", -1),
    ("txt:AffineTransform_double_3_3:short", "expected 12", -1),
    ("mat:garbage", "not a MATLAB v4 file", -1),
    ("mat:truncated", "truncated", -1),
    ("txt:noheader", "not an Insight transform text file", -1),
    ("missing", "cannot open transform file", -1),
    ("index", "out of range", -1),
])
def test_read_errors(tmp_path, content, needle, code):
    kind = content.split(":")
    if kind[0] == "txt" and kind[1] == "noheader":
        p = tmp_path / "x.txt"
        p.write_text("Transform: AffineTransform_double_3_3\nParameters: 1 0 0 0 1 0 0 0 1 0 0 0\n")
    elif kind[0] == "txt":
        p = tmp_path / "x.txt"
        n = 6 if len(kind) > 2 else 12
        write_txt(p, [(kind[1], list(range(n)), [0, 0, 0])])
    elif content == "mat:garbage":
        p = tmp_path / "x.mat"
        p.write_bytes(b"\x7f\x7f\x7f\x7f" * 10)
    elif content == "mat:truncated":
        p = tmp_path / "x.mat"
        write_mat(p, [("AffineTransform_double_3_3", np.r_[AFFINE3, TRANS3])])
        p.write_bytes(p.read_bytes()[:-9])
    elif content == "missing":
        p = tmp_path / "none.mat"
    else:
        p = tmp_path / "x.mat"
        write_mat(p, [("AffineTransform_double_3_3", np.r_[AFFINE3, TRANS3]), ("fixed", CENTER3)])
        with pytest.raises(SynxError, match=needle):
            synx.read_linear_transform(p, 3, 1)
        return
    lib = synx.load_library()
    rc = lib.synx_read_linear_transform(os.fsencode(str(p)), 3, 0, None)
    assert rc == code
    assert needle in lib.synx_last_error(None).decode()


@pytest.mark.parametrize("dim", [2, 3])
def test_linear_field_matches_numpy(dim):
    if dim == 3:
        t = LinearTransform(AFFINE3.reshape(3, 3), TRANS3, CENTER3)
        direction = Rotation.from_euler("xyz", [0.2, -0.1, 0.3]).as_matrix()
        g = Geom((17, 13, 11), (1.2, 0.9, 1.5), (-5.0, 3.0, 2.0), direction)
    else:
        t = LinearTransform(np.array([[0.95, 0.1], [-0.07, 1.04]]), np.array([1.5, -2.0]), np.array([4.0, 6.0]))
        th = 0.3
        g = Geom((23, 19), (1.1, 0.8), (2.0, -1.0), np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]]))
    P = physical_points(g)
    for inverse in (False, True):
        u = synx.linear_field(t, g, invert=inverse)
        assert u.shape == (dim,) + g.shape  # component planes
        np.testing.assert_allclose(u, np.moveaxis(apply(t, P, inverse) - P, -1, 0), atol=2e-5)
    # forward then inverse is the identity
    np.testing.assert_allclose(apply(t, apply(t, P), inverse=True), P, atol=1e-9)


@pytest.mark.parametrize("dim", [2, 3])
def test_linear_field_drives_the_step_functions(dim):
    """The field's layout is the one the step functions take: warping an image that is linear in
    physical space through it (the oracle's warp, whose layout the GPU parity tests pin) gives
    that linear function at T(p) wherever T(p) stays inside the image."""
    import oracle as O
    if dim == 3:
        t = LinearTransform(AFFINE3.reshape(3, 3), TRANS3, CENTER3)
        g = Geom((20, 18, 16), (1.0, 1.2, 0.9), (4.0, -6.0, 2.0))
        gi = Geom((40, 40, 36), (1.0, 1.0, 1.0), (-6.0, -16.0, -8.0))
    else:
        t = LinearTransform(np.array([[0.95, 0.1], [-0.07, 1.04]]), np.array([1.5, -2.0]), np.array([4.0, 6.0]))
        g = Geom((24, 20), (1.1, 0.8), (2.0, -1.0))
        gi = Geom((44, 40), (1.0, 1.0), (-8.0, -11.0))
    coef = np.array([0.7, -0.4, 0.25])[:dim]
    img = (physical_points(gi) @ coef + 3.0).astype(np.float32)
    got = O.warp_image(img, gi, synx.linear_field(t, g), g)
    Tp = apply(t, physical_points(g))
    want = Tp @ coef + 3.0
    lo = np.asarray(gi.origin)
    hi = lo + (np.asarray(gi.size) - 1) * np.asarray(gi.spacing)
    inside = np.all((Tp > lo + 1e-3) & (Tp < hi - 1e-3), axis=-1)
    assert inside.mean() > 0.9
    np.testing.assert_allclose(got[inside], want[inside], atol=2e-4)


def test_linear_field_rejects_singular_inverse_and_bad_grids():
    t = LinearTransform(np.array([[1.0, 2.0, 0.0], [2.0, 4.0, 0.0], [0.0, 0.0, 1.0]]), np.zeros(3), np.zeros(3))
    g = Geom((4, 4, 4))
    synx.linear_field(t, g)  # the forward map needs no inverse
    with pytest.raises(SynxError, match="singular"):
        synx.linear_field(t, g, invert=True)
    with pytest.raises(SynxError, match="dimensions differ"):
        synx.linear_field(t, Geom((4, 4)))


@pytest.mark.parametrize("ext", [".mat", ".txt", ".tfm"])
@pytest.mark.parametrize("dim", [2, 3])
def test_write_round_trip(tmp_path, ext, dim):
    if dim == 3:
        t = LinearTransform(AFFINE3.reshape(3, 3), TRANS3, CENTER3)
    else:
        t = LinearTransform(np.array([[0.95, 0.1], [-0.07, 1.04]]), np.array([1.5, -2.0]), np.array([4.0, 6.0]))
    p = tmp_path / f"w{ext}"
    synx.write_linear_transform(p, t)
    back = synx.read_linear_transform(p, dim)
    np.testing.assert_array_equal(back.matrix, t.matrix)
    np.testing.assert_array_equal(back.translation, t.translation)
    np.testing.assert_array_equal(back.center, t.center)
    if ext == ".mat":  # the bytes ITK's MATLAB writer lays down: this file's own writer agrees
        q = tmp_path / "ref.mat"
        write_mat(q, [(f"AffineTransform_double_{dim}_{dim}", np.r_[t.matrix.ravel(), t.translation]),
                      ("fixed", t.center)])
        assert p.read_bytes() == q.read_bytes()
    else:
        assert p.read_text().startswith("#Insight Transform File V1.0")


def test_has_center_flags(tmp_path):
    lib = synx.load_library()
    for name, params, fixed, want in [("AffineTransform_double_3_3", np.r_[AFFINE3, TRANS3], CENTER3, 1),
                                      ("Euler3DTransform_double_3_3", [0.1, 0.2, 0.3, 1, 2, 3], [0, 0, 0], 1),
                                      ("TranslationTransform_double_3_3", [1, 2, 3], [], 0),
                                      ("IdentityTransform_double_3_3", [], [], 0)]:
        p = tmp_path / f"{name}.txt"
        write_txt(p, [(name, params, fixed)])
        t = synx.SynxLinear()
        assert lib.synx_read_linear_transform(os.fsencode(str(p)), 3, 0, t) == 1
        assert t.has_center == want, name


@pytest.mark.parametrize("dim", [2, 3])
def test_initial_translation_features(dim):
    rng = np.random.default_rng(dim)
    if dim == 3:
        gf = Geom((17, 13, 11), (1.2, 0.9, 1.5), (-5.0, 3.0, 2.0), Rotation.from_euler("xyz", [0.2, -0.1, 0.3]).as_matrix())
        gm = Geom((15, 16, 12), (1.0, 1.1, 1.3), (2.0, -1.0, 4.0), Rotation.from_euler("zyx", [0.1, 0.2, -0.1]).as_matrix())
    else:
        gf = Geom((23, 19), (1.1, 0.8), (2.0, -1.0), np.array([[np.cos(0.3), -np.sin(0.3)], [np.sin(0.3), np.cos(0.3)]]))
        gm = Geom((21, 25), (0.9, 1.0), (-3.0, 4.0))
    F = rng.uniform(0, 1, gf.shape).astype(np.float32)
    M = rng.uniform(0, 2, gm.shape).astype(np.float32)

    def centers(g, img, feature):
        if feature == 2:
            return np.asarray(g.origin)
        P = physical_points(g).reshape(-1, dim)
        if feature == 0:
            return np.asarray(g.origin) + g.direction @ (np.asarray(g.spacing) * (np.asarray(g.size) - 1) / 2)
        w = img.astype(np.float64).ravel()
        return (P * w[:, None]).sum(0) / w.sum()

    for feature in (0, 1, 2):
        t = synx.initial_translation(F, gf, M, gm, feature)
        cf, cm = centers(gf, F, feature), centers(gm, M, feature)
        np.testing.assert_array_equal(t.matrix, np.eye(dim))
        np.testing.assert_allclose(t.center, cf, atol=1e-9)
        np.testing.assert_allclose(t.translation, cm - cf, atol=1e-9)
    # features 0 and 2 need no intensities
    t = synx.initial_translation(None, gf, None, gm, 0)
    np.testing.assert_allclose(t.translation, centers(gm, M, 0) - centers(gf, F, 0), atol=1e-9)


def test_initial_translation_errors():
    g = Geom((8, 8))
    with pytest.raises(SynxError, match="total mass"):
        synx.initial_translation(np.zeros(g.shape, np.float32), g, np.ones(g.shape, np.float32), g, 1)
    with pytest.raises(SynxError, match="feature must be"):
        synx.initial_translation(None, g, None, g, 3)
    with pytest.raises(SynxError, match="dimensions differ"):
        synx.initial_translation(None, g, None, Geom((8, 8, 8)), 0)


@pytest.fixture(scope="module")
def apply_exe():
    from ants_b200 import build
    build.build_all()
    assert os.path.exists(APPLY)
    return APPLY


@pytest.mark.parametrize("tname,needle", [("affine.h5", "not supported"), ("missing.mat", "cannot open transform file")])
def test_cli_rejects_unreadable_transforms(apply_exe, tmp_path, tname, needle):
    r = subprocess.run([apply_exe, "-d", "3", "-i", "a.nii.gz", "-r", "a.nii.gz", "-o", "x.nii.gz", "-t",
                        str(tmp_path / tname)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert needle in r.stderr


def test_registration_cli_rejects_a_bad_feature(tmp_path):
    from ants_b200 import build, nifti
    build.build_all()
    reg = os.path.join(ROOT, "ants_b200", "antsRegistrationSyN_b200")
    g = Geom((8, 8))
    nifti.write(tmp_path / "a.nii.gz", np.ones(g.shape, np.float32), g)
    r = subprocess.run([reg, "-d", "2", "-m", f"CC[{tmp_path}/a.nii.gz,{tmp_path}/a.nii.gz,1,2]", "-t", "SyN[0.1,3,0]",
                        "-c", "2", "-f", "1", "-s", "0", "-o", str(tmp_path / "x"),
                        "-r", f"[{tmp_path}/a.nii.gz,{tmp_path}/a.nii.gz,3]"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert "feature must be" in r.stderr


def test_fold_moving_geometry_reads_the_image_at_init():
    """Index of q in the folded geometry == index of Init(q) in the original (two transforms, first
    applied first)."""
    g = Geom((9, 8, 7), (1.1, 0.9, 1.2), (3.0, -2.0, 1.0), Rotation.from_euler("xyz", [0.1, 0.2, -0.1]).as_matrix())
    T1 = LinearTransform(AFFINE3.reshape(3, 3), TRANS3, CENTER3)
    T2 = LinearTransform(Rotation.from_euler("z", 0.3).as_matrix(), np.array([1.0, 0.5, -2.0]), np.array([4.0, 4.0, 4.0]))
    gf = synx.fold_moving_geometry(g, [T1, T2])

    def index_of(geom, q):
        return np.linalg.solve(geom.direction * np.asarray(geom.spacing), q - np.asarray(geom.origin))

    rng = np.random.default_rng(5)
    for q in rng.uniform(-10, 20, (10, 3)):
        init_q = apply(T2, apply(T1, q))
        np.testing.assert_allclose(index_of(gf, q), index_of(g, init_q), atol=1e-9)


def test_from_parameters_matches_the_file_reader(tmp_path):
    # synx_linear_from_parameters converts one (type, parameters, fixed parameters) entry exactly as
    # synx_read_linear_transform converts that entry of a file
    v = [0.1, -0.2, 0.15]
    cases = [
        (3, "AffineTransform_double_3_3", list(AFFINE3) + list(TRANS3), list(CENTER3)),
        (3, "MatrixOffsetTransformBase_float_3_3", list(AFFINE3) + list(TRANS3), list(CENTER3)),
        (3, "Euler3DTransform_double_3_3", [0.3, -0.2, 0.45, 1, 2, 3], [1.0, 2.0, 3.0]),
        (3, "Euler3DTransform_double_3_3", [0.3, -0.2, 0.45, 1, 2, 3], [1.0, 2.0, 3.0, 1.0]),
        (3, "VersorRigid3DTransform_double_3_3", v + [1, 2, 3], [1.0, 2.0, 3.0]),
        (3, "Similarity3DTransform_double_3_3", v + [1, 2, 3, 1.3], [1.0, 2.0, 3.0]),
        (3, "TranslationTransform_double_3_3", [1, 2, 3], []),
        (3, "IdentityTransform_double_3_3", [], []),
        (2, "AffineTransform_double_2_2", [1.1, 0.2, -0.1, 0.9, 4, 5], [3.0, 4.0]),
        (2, "Euler2DTransform_double_2_2", [0.4, 5, -6], [3.0, 4.0]),
        (2, "Rigid2DTransform_double_2_2", [0.4, 5, -6], [3.0, 4.0]),
        (2, "Similarity2DTransform_double_2_2", [0.8, 0.4, 5, -6], [3.0, 4.0]),
    ]
    for i, (dim, name, params, fixed) in enumerate(cases):
        p = tmp_path / f"t{i}.txt"
        write_txt(p, [(name, params, fixed)])
        want = synx.read_linear_transform(p, dim)
        got = synx.linear_from_parameters(name, params, fixed, dim)
        for a, b in ((got.matrix, want.matrix), (got.translation, want.translation), (got.center, want.center)):
            np.testing.assert_array_equal(a, b, err_msg=name)
    lib = synx.load_library()
    for name, params, fixed, dim, code, needle in [
        ("CompositeTransform_double_3_3", [], [], 3, -1, "composite is not a linear transform"),
        ("Euler3DTransform_double_3_3", [0.1, 0.2, 0.3, 1, 2], [0, 0, 0], 3, -1, "expected 6"),
        ("AffineTransform_double_2_2", [1, 0, 0, 1, 0, 0], [0, 0], 3, -1, "is not a 3-D transform"),
        ("BSplineTransform_double_3_3", [0.0] * 6, [0, 0, 0], 3, -5, "is not supported"),
        ("Affine", [1, 0, 0, 1, 0, 0], [0, 0], 2, -1, "unrecognised transform type"),
    ]:
        with pytest.raises(SynxError, match=needle):
            synx.linear_from_parameters(name, params, fixed, dim)
        t = synx.SynxLinear()
        arr = (C.c_double * max(len(params), 1))(*params)
        fx = (C.c_double * max(len(fixed), 1))(*fixed)
        assert lib.synx_linear_from_parameters(name.encode(), arr, len(params), fx, len(fixed), dim, C.byref(t)) == code
    assert lib.synx_linear_from_parameters(b"IdentityTransform_double_2_2", None, 0, None, 0, 2, None) == -1
    assert lib.synx_linear_from_parameters(b"IdentityTransform_double_2_2", None, 1, None, 0, 2,
                                           C.byref(synx.SynxLinear())) == -1
