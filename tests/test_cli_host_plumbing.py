"""The command lines' own logic, on a machine without a GPU.

The real sources of antsApplyTransforms_b200 and antsRegistrationSyN_b200 are compiled against
host stand-ins for the device (tests/cli_host/: host CUDA runtime calls, and the step and stage
entry points routed to the CPU oracle), then run through the same checks as their GPU tests:
transform chains in the reference's order, linear transforms folded into grid geometry, the
collapsed field, initial moving transforms, output file names and written transforms, and the
bit-exact agreement of the two programs' warped images.  What this covers is the programs'
plumbing; the kernels' parity is the GPU tests'.  The stand-ins are test infrastructure: the
product's command lines link libsynx.so and fail without a GPU.
"""
import os
import shutil
import subprocess

import pytest

import test_apply_transforms as A
import test_zz_stack_apply as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "ants_b200", "csrc")
HOST = os.path.join(ROOT, "tests", "cli_host")


@pytest.fixture(scope="module")
def host_cli(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    out = tmp_path_factory.mktemp("cli_host")
    common = ["g++", "-std=c++17", "-O2", "-fopenmp", "-I", HOST, "-I", os.path.join(ROOT, "include"), "-I", CSRC,
              "-I", os.path.join(ROOT, "oracle")]
    libs = [os.path.join(CSRC, "nifti_io.cpp"), os.path.join(CSRC, "synx_linear.cpp"),
            os.path.join(HOST, "host_steps.cpp"), os.path.join(ROOT, "oracle", "synx_oracle_capi.cpp"), "-lz"]
    exes = {}
    for name, src, extra in (("apply", "ants_apply_transforms.cpp", []),
                             ("reg", "ants_registration.cpp", [os.path.join(HOST, "host_stage.cpp")])):
        exe = str(out / name)
        r = subprocess.run(common + ["-o", exe, os.path.join(CSRC, src)] + extra + libs, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-3000:]
        exes[name] = exe
    return exes


@pytest.mark.parametrize("dim", [2, 3])
def test_transform_stacks(host_cli, tmp_path, dim):
    S.check_stacks_match_the_scheme(host_cli["apply"], tmp_path, dim)


def test_default_value(host_cli, tmp_path):
    A.check_default_value_outside(host_cli["apply"], tmp_path)


def test_warped_output_matches_antsapplytransforms(host_cli, tmp_path):
    A.check_reproduces_the_registration_output(host_cli["reg"], host_cli["apply"], tmp_path)


def test_initial_moving_transform(host_cli, tmp_path):
    S.check_initial_moving_transform(host_cli["reg"], host_cli["apply"], tmp_path)


def test_derived_initial_translation(host_cli, tmp_path):
    S.check_derived_initial_translation(host_cli["reg"], tmp_path)


@pytest.mark.parametrize("interp", ["NearestNeighbor", "GenericLabel", "GenericLabel[Linear]"])
@pytest.mark.parametrize("dim", [2, 3])
def test_label_interpolation(host_cli, tmp_path, dim, interp):
    S.check_label_interpolation(host_cli["apply"], tmp_path, dim, interp)


def test_multichannel(host_cli, tmp_path):
    S.check_multichannel(host_cli["apply"], tmp_path)


def test_time_series(host_cli, tmp_path):
    S.check_time_series(host_cli["apply"], tmp_path)


def test_time_index(host_cli, tmp_path):
    S.check_time_index(host_cli["apply"], tmp_path)


def test_output_types(host_cli, tmp_path):
    S.check_output_types(host_cli["apply"], tmp_path)


def test_output_precision(host_cli, tmp_path):
    S.check_output_precision(host_cli["reg"], tmp_path)


def test_histogram_matching(host_cli, tmp_path):
    import numpy as np

    import oracle as O
    import test_zz_u_histogram_match_gpu as H

    def stage_fields(f, gf, m, gm, P):
        fwd, inv, _, _ = O.syn_register(f, gf, m, gm, P)
        return np.moveaxis(fwd, 0, -1), np.moveaxis(inv, 0, -1)

    H.check_cli_histogram_matching(host_cli["reg"], tmp_path, stage_fields)


def test_masks(host_cli, tmp_path):
    import numpy as np

    import oracle as O
    import test_zz_t_masks as X

    def stage_fields(f, gf, m, gm, P, mf, mm):
        fwd, inv, _, _ = O.syn_register(f, gf, m, gm, P, fixed_mask=mf, fixed_mask_geom=gf, moving_mask=mm,
                                        moving_mask_geom=gm)
        return np.moveaxis(fwd, 0, -1), np.moveaxis(inv, 0, -1)

    X.check_cli_masks(host_cli["reg"], tmp_path, stage_fields)


def test_state_and_composite(host_cli, tmp_path):
    import oracle as O
    import test_zz_u_state as U

    def stage(f, gf, m, gm, P, init):
        kw = {}
        if init is not None:
            kw = dict(initial_half_fields=[U.planes(a) for a in init], initial_geom=gf)
        fwd, inv, _, _, half = O.syn_register(f, gf, m, gm, P, return_half_fields=True, **kw)
        return U.interleaved(fwd), U.interleaved(inv), [U.interleaved(h) for h in half]

    U.check_cli_state(host_cli["reg"], tmp_path, stage)


def test_state_with_initial_transform(host_cli, tmp_path):
    # -r init.mat with --save-state: the state and the composite list the initial transform first
    # (ITK's composite order: it acts last); --restore-state makes it the initial moving transform again
    # and starts the stage from the saved fields
    import numpy as np

    import oracle as O
    import test_zz_stack_apply as S
    import test_zz_u_state as U
    from ants_b200 import nifti, phantoms
    from ants_b200.synx import Geom, SyNParams
    size = (64, 60)
    f, m = phantoms.pair_2d(size, seed=33)
    g = Geom(size)
    A = S.Affine([[1.02, 0.03], [-0.02, 0.99]], [0.8, -0.6], [32.0, 30.0])
    A.write_mat(tmp_path / "init.mat")
    nifti.write(tmp_path / "f.nii.gz", f, g)
    nifti.write(tmp_path / "m.nii.gz", m, g)
    base = [host_cli["reg"], "-d", "2", "--float", "1", "-m", f"CC[{tmp_path}/f.nii.gz,{tmp_path}/m.nii.gz,1,2]",
            "-t", "SyN[0.2,3,0]", "-c", "[8x4,1e-12,10]", "-f", "2x1", "-s", "1x0vox", "-a", "1", "-z", "0", "-i", "1"]
    state = str(tmp_path / "state.txt")
    r = subprocess.run(base + ["-r", f"{tmp_path}/init.mat", "-j", state, "-o", str(tmp_path / "A_")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    items = U.read_composite(state)
    assert [t for t, _, _ in items] == ["AffineTransform_double_2_2"] + ["DisplacementFieldTransform_float_2_2"] * 4
    np.testing.assert_allclose(items[0][1], np.r_[A.A.ravel(), A.t], atol=1e-12)
    np.testing.assert_allclose(items[0][2], A.c, atol=1e-12)
    comp = U.read_composite(tmp_path / "A_Composite.txt")
    icomp = U.read_composite(tmp_path / "A_InverseComposite.txt")
    assert [t for t, _, _ in comp] == ["AffineTransform_double_2_2", "DisplacementFieldTransform_float_2_2"]
    assert [t for t, _, _ in icomp] == ["DisplacementFieldTransform_float_2_2", "AffineTransform_double_2_2"]
    Ai = np.linalg.inv(A.A)
    np.testing.assert_allclose(icomp[1][1][:4].reshape(2, 2), Ai, atol=1e-12)
    np.testing.assert_allclose(icomp[1][1][4:], -Ai @ A.t, atol=1e-9)  # same center, inverted map
    # restore: the initial transform comes back from the state, the stage starts from its fields
    r = subprocess.run(base + ["-k", state, "-o", str(tmp_path / "B_")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    comp_b = U.read_composite(tmp_path / "B_Composite.txt")
    np.testing.assert_allclose(comp_b[0][1], items[0][1], atol=1e-12)
    half = [np.ascontiguousarray(it[1].astype(np.float32).reshape(size[1], size[0], 2).transpose(2, 0, 1))
            for it in items[1:]]
    P = SyNParams(dim=2, learning_rate=0.2, cc_radius=2, iterations=(8, 4), shrink_factors=(2, 1),
                  smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12)
    rf, _, go, _ = O.syn_register(f, g, m, S.push_forward(g, A.inverse()), P, initial_half_fields=half,
                                  initial_geom=g)
    got = comp_b[1][1].astype(np.float32).reshape(size[1], size[0], 2).transpose(2, 0, 1)
    assert float(np.sqrt(((got - rf) ** 2).sum(0).mean())) <= 1e-3


def test_restore_rejects_malformed_state(host_cli, tmp_path):
    # a saved state edited by hand: each defect is refused with its own message before the stage runs
    from ants_b200 import nifti, phantoms
    from ants_b200.synx import Geom
    size = (40, 36)
    f, m = phantoms.pair_2d(size, seed=34)
    g = Geom(size)
    nifti.write(tmp_path / "f.nii.gz", f, g)
    nifti.write(tmp_path / "m.nii.gz", m, g)
    base = [host_cli["reg"], "-d", "2", "--float", "1", "-m", f"CC[{tmp_path}/f.nii.gz,{tmp_path}/m.nii.gz,1,2]",
            "-t", "SyN[0.2,3,0]", "-c", "[2x1,1e-12,10]", "-f", "2x1", "-s", "1x0vox", "-a", "1", "-z", "0", "-i", "1"]
    state = tmp_path / "state.txt"
    r = subprocess.run(base + ["-j", str(state), "-o", str(tmp_path / "A_")], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    lines = state.read_text().splitlines()
    par = [i for i, s in enumerate(lines) if s.startswith("Parameters:")]
    fix = [i for i, s in enumerate(lines) if s.startswith("FixedParameters:")]
    assert len(par) == len(fix) == 4

    def edited(line, fn):
        out = list(lines)
        out[line] = fn(out[line])
        return out

    def replace_token(k, value):
        def fn(s):
            key, vals = s.split(":", 1)
            t = vals.split()
            t[k] = value
            return key + ": " + " ".join(t)
        return fn

    cases = {
        "not an ITK text transform file": lines[1:],
        "bad number": edited(par[3], replace_token(0, "x1")),
        "positive integers": edited(fix[0], replace_token(0, "0")),
        "do not match its size": edited(par[0], lambda s: s.rsplit(" ", 1)[0]),
        "do not share one grid": edited(fix[3], replace_token(2, "1.5")),
        "other than a SyN state": lines[:par[3] - 2],
        "unexpected key": lines + ["Offset: 1 2"],
    }
    for k, (msg, text) in enumerate(cases.items()):
        bad = tmp_path / f"bad{k}.txt"
        bad.write_text("\n".join(text) + "\n")
        r = subprocess.run(base + ["-k", str(bad), "-o", str(tmp_path / f"B{k}_")], capture_output=True, text=True,
                           timeout=600)
        assert r.returncode != 0 and msg in r.stderr, (msg, r.stderr)
        assert not (tmp_path / f"B{k}_Composite.txt").exists()
    # the unedited state restores
    r = subprocess.run(base + ["-k", str(state), "-o", str(tmp_path / "C_")], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr


def test_collapsed_composite(host_cli, tmp_path):
    # -a 1 with collapsing (the default -z 1) and two -r transforms: the composite holds one affine
    # transform, the same one prefix0GenericAffine.mat holds without -a, then the SyN field (the same
    # values as prefix1Warp); the inverse composite lists the field's inverse, then the affine's inverse
    import numpy as np

    import test_zz_stack_apply as S
    import test_zz_u_state as U
    from ants_b200 import nifti, phantoms, synx
    from ants_b200.synx import Geom
    size = (48, 44)
    f, m = phantoms.pair_2d(size, seed=35)
    g = Geom(size)
    A = S.Affine([[1.01, 0.02], [-0.01, 0.98]], [0.5, -0.4], [24.0, 22.0])
    B = S.Affine([[0.99, -0.015], [0.01, 1.02]], [-0.3, 0.2], [20.0, 21.0])
    A.write_mat(tmp_path / "a.mat")
    B.write_mat(tmp_path / "b.mat")
    nifti.write(tmp_path / "f.nii.gz", f, g)
    nifti.write(tmp_path / "m.nii.gz", m, g)
    base = [host_cli["reg"], "-d", "2", "--float", "1", "-m", f"CC[{tmp_path}/f.nii.gz,{tmp_path}/m.nii.gz,1,2]",
            "-t", "SyN[0.2,3,0]", "-c", "[4x2,1e-12,10]", "-f", "2x1", "-s", "1x0vox",
            "-r", f"{tmp_path}/a.mat", "-r", f"{tmp_path}/b.mat"]
    for extra in (["-o", str(tmp_path / "A_")], ["-a", "1", "-o", str(tmp_path / "B_")]):
        r = subprocess.run(base + extra, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
    assert not (tmp_path / "B_0GenericAffine.mat").exists() and not (tmp_path / "B_1Warp.nii.gz").exists()
    comp = U.read_composite(tmp_path / "B_Composite.txt")
    icomp = U.read_composite(tmp_path / "B_InverseComposite.txt")
    assert [t for t, _, _ in comp] == ["AffineTransform_double_2_2", "DisplacementFieldTransform_float_2_2"]
    assert [t for t, _, _ in icomp] == ["DisplacementFieldTransform_float_2_2", "AffineTransform_double_2_2"]
    mat = synx.read_linear_transform(str(tmp_path / "A_0GenericAffine.mat"), 2)
    np.testing.assert_allclose(comp[0][1][:4].reshape(2, 2), mat.matrix, atol=1e-12)
    np.testing.assert_allclose(comp[0][1][4:], mat.translation, atol=1e-9)
    np.testing.assert_allclose(comp[0][2], mat.center, atol=1e-12)
    fwd, _ = nifti.read(tmp_path / "A_1Warp.nii.gz", 2)
    inv, _ = nifti.read(tmp_path / "A_1InverseWarp.nii.gz", 2)
    np.testing.assert_array_equal(comp[1][1].astype(np.float32), fwd.astype(np.float32).reshape(-1))
    np.testing.assert_array_equal(icomp[0][1].astype(np.float32), inv.astype(np.float32).reshape(-1))
    # the inverse composite's affine undoes the collapsed one
    Cf = S.Affine(comp[0][1][:4].reshape(2, 2), comp[0][1][4:], comp[0][2])
    Ci = S.Affine(icomp[1][1][:4].reshape(2, 2), icomp[1][1][4:], icomp[1][2])
    np.testing.assert_allclose(Ci.M @ Cf.M, np.eye(2), atol=1e-12)
    np.testing.assert_allclose(Ci.M @ Cf.b + Ci.b, 0.0, atol=1e-9)
    # and the collapsed affine is the two -r transforms composed: the reference stores repeated options
    # newest first and adds them to the composite in that order, which applies the last one added (the
    # first given) first to a point; the center is that of the transform acting first
    np.testing.assert_allclose(Cf.M, B.M @ A.M, atol=1e-12)
    np.testing.assert_allclose(Cf.b, B.M @ A.b + B.b, atol=1e-9)
    np.testing.assert_allclose(comp[0][2], A.c, atol=1e-12)
    # without --float 1 the reference's fields are double: the entries say so, and carry the same values
    r = subprocess.run([a for a in base if a not in ("--float", "1")] + ["-a", "1", "-o", str(tmp_path / "D_")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    dcomp = U.read_composite(tmp_path / "D_Composite.txt")
    assert [t for t, _, _ in dcomp] == ["AffineTransform_double_2_2", "DisplacementFieldTransform_double_2_2"]
    np.testing.assert_array_equal(dcomp[1][1].astype(np.float32), comp[1][1].astype(np.float32))


def test_restore_state_with_a_rigid_entry(host_cli, tmp_path):
    # a state whose linear part is a rigid transform (the type a rigid stage saves, here Euler2D): it
    # becomes the initial moving transform in matrix-offset form, written back as an affine entry, and
    # the stage starts from the saved fields with the moving image read through it
    import numpy as np

    import oracle as O
    import test_zz_stack_apply as S
    import test_zz_u_state as U
    from ants_b200 import nifti, phantoms, synx
    from ants_b200.synx import Geom, SyNParams
    size = (48, 44)
    f, m = phantoms.pair_2d(size, seed=36)
    g = Geom(size)
    nifti.write(tmp_path / "f.nii.gz", f, g)
    nifti.write(tmp_path / "m.nii.gz", m, g)
    base = [host_cli["reg"], "-d", "2", "--float", "1", "-m", f"CC[{tmp_path}/f.nii.gz,{tmp_path}/m.nii.gz,1,2]",
            "-t", "SyN[0.2,3,0]", "-c", "[4x2,1e-12,10]", "-f", "2x1", "-s", "1x0vox", "-a", "1", "-z", "0", "-i", "1"]
    state = tmp_path / "state.txt"
    r = subprocess.run(base + ["-j", str(state), "-o", str(tmp_path / "A_")], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    lines = state.read_text().splitlines()
    assert lines[2].startswith("Transform: CompositeTransform_")
    euler = ("Euler2DTransform_double_2_2", [0.05, 0.7, -0.4], [20.0, 18.0])
    lines[3:3] = ["#Transform 1", f"Transform: {euler[0]}", "Parameters: 0.05 0.7 -0.4", "FixedParameters: 20 18"]
    rigid = tmp_path / "rigid_state.txt"
    rigid.write_text("\n".join(lines) + "\n")
    r = subprocess.run(base + ["-k", str(rigid), "-o", str(tmp_path / "B_")], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    L = synx.linear_from_parameters(*euler, 2)
    th = 0.05
    np.testing.assert_allclose(L.matrix, [[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]], atol=1e-15)
    comp = U.read_composite(tmp_path / "B_Composite.txt")
    assert [t for t, _, _ in comp] == ["AffineTransform_double_2_2", "DisplacementFieldTransform_float_2_2"]
    np.testing.assert_allclose(comp[0][1], np.r_[L.matrix.ravel(), L.translation], atol=1e-15)
    np.testing.assert_allclose(comp[0][2], L.center, atol=1e-15)
    items = U.read_composite(state)
    half = [np.ascontiguousarray(it[1].astype(np.float32).reshape(size[1], size[0], 2).transpose(2, 0, 1))
            for it in items]
    A = S.Affine(L.matrix, L.translation, L.center)
    P = SyNParams(dim=2, learning_rate=0.2, cc_radius=2, iterations=(4, 2), shrink_factors=(2, 1),
                  smoothing_sigmas=(1.0, 0.0), convergence_threshold=1e-12)
    rf, _, _, _ = O.syn_register(f, g, m, S.push_forward(g, A.inverse()), P, initial_half_fields=half,
                                 initial_geom=g)
    got = comp[1][1].astype(np.float32).reshape(size[1], size[0], 2).transpose(2, 0, 1)
    assert float(np.sqrt(((got - rf) ** 2).sum(0).mean())) <= 1e-3


def test_apply_reads_the_composite(host_cli, tmp_path):
    # antsApplyTransforms -t prefixComposite.txt acts as the separate files of the same registration:
    # the composite's last entry (the SyN field) first, then the affine; the inverse composite as
    # -t [prefix0GenericAffine.mat,1] -t prefix1InverseWarp; and [composite,1] is refused
    import numpy as np

    import test_zz_stack_apply as S
    from ants_b200 import nifti, phantoms
    from ants_b200.synx import Geom
    size = (48, 44)
    f, m = phantoms.pair_2d(size, seed=37)
    g = Geom(size, (1.0, 0.9))
    A = S.Affine([[1.01, 0.02], [-0.01, 0.98]], [0.5, -0.4], [24.0, 20.0])
    A.write_mat(tmp_path / "a.mat")
    nifti.write(tmp_path / "f.nii.gz", f, g)
    nifti.write(tmp_path / "m.nii.gz", m, g)
    base = [host_cli["reg"], "-d", "2", "--float", "1", "-m", f"CC[{tmp_path}/f.nii.gz,{tmp_path}/m.nii.gz,1,2]",
            "-t", "SyN[0.2,3,0]", "-c", "[4x2,1e-12,10]", "-f", "2x1", "-s", "1x0vox", "-r", f"{tmp_path}/a.mat"]
    for extra in (["-o", str(tmp_path / "A_")], ["-a", "1", "-o", str(tmp_path / "B_")]):
        r = subprocess.run(base + extra, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr

    def apply(ref, inp, ts, out, collapse=False):
        o = f"[{tmp_path / out},1]" if collapse else str(tmp_path / out)
        args = [host_cli["apply"], "-d", "2", "--float", "1", "-i", f"{tmp_path}/{inp}.nii.gz",
                "-r", f"{tmp_path}/{ref}.nii.gz"] + sum((["-t", t] for t in ts), []) + ["-o", o]
        r = subprocess.run(args, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        return nifti.read(tmp_path / out, 2)[0]

    p, q = str(tmp_path / "A_"), str(tmp_path / "B_")
    want = apply("f", "m", [f"{p}1Warp.nii.gz", f"{p}0GenericAffine.mat"], "w_files.nii.gz")
    got = apply("f", "m", [f"{q}Composite.txt"], "w_comp.nii.gz")
    np.testing.assert_array_equal(got, want)
    want = apply("m", "f", [f"[{p}0GenericAffine.mat,1]", f"{p}1InverseWarp.nii.gz"], "i_files.nii.gz")
    got = apply("m", "f", [f"{q}InverseComposite.txt"], "i_comp.nii.gz")
    bad = np.abs(got - want) > 1e-5  # the inverse affine is stored re-centred: rounding-level changes
    assert bad.mean() < 1e-3, int(bad.sum())
    # the collapsed field through the composite equals the one through the files
    cf = apply("f", "m", [f"{q}Composite.txt"], "c_comp.nii.gz", collapse=True)
    ff = apply("f", "m", [f"{p}1Warp.nii.gz", f"{p}0GenericAffine.mat"], "c_files.nii.gz", collapse=True)
    np.testing.assert_array_equal(cf, ff)
    r = subprocess.run([host_cli["apply"], "-d", "2", "-i", f"{tmp_path}/m.nii.gz", "-r", f"{tmp_path}/f.nii.gz",
                        "-t", f"[{q}Composite.txt,1]", "-o", str(tmp_path / "x.nii.gz")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode != 0 and "use the inverse composite" in r.stderr, r.stderr
    # a damaged composite is reported as such, not as an unsupported linear type
    lines = (tmp_path / "B_Composite.txt").read_text().splitlines()
    par = [i for i, ln in enumerate(lines) if ln.startswith("Parameters:")][-1]
    lines[par] = lines[par].rsplit(" ", 1)[0]
    (tmp_path / "bad_comp.txt").write_text("\n".join(lines) + "\n")
    r = subprocess.run([host_cli["apply"], "-d", "2", "-i", f"{tmp_path}/m.nii.gz", "-r", f"{tmp_path}/f.nii.gz",
                        "-t", str(tmp_path / "bad_comp.txt"), "-o", str(tmp_path / "x.nii.gz")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode != 0 and "do not match its size" in r.stderr, r.stderr
    lines[par] = lines[par] + " abc"
    (tmp_path / "bad_comp2.txt").write_text("\n".join(lines) + "\n")
    r = subprocess.run([host_cli["apply"], "-d", "2", "-i", f"{tmp_path}/m.nii.gz", "-r", f"{tmp_path}/f.nii.gz",
                        "-t", str(tmp_path / "bad_comp2.txt"), "-o", str(tmp_path / "x.nii.gz")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode != 0 and "bad number" in r.stderr, r.stderr

    # -o CompositeTransform[file] writes the stack uncollapsed (no input or reference image needed): the
    # same composite antsRegistration -a 1 wrote, and it applies as the files do
    def write_composite(ts, out):
        args = [host_cli["apply"], "-d", "2", "--float", "1"] + sum((["-t", t] for t in ts), [])
        r = subprocess.run(args + ["-o", f"CompositeTransform[{tmp_path / out}]"], capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr
        return U.read_composite(tmp_path / out)

    import test_zz_u_state as U
    fw = write_composite([f"{p}1Warp.nii.gz", f"{p}0GenericAffine.mat"], "fw.txt")
    reg = U.read_composite(tmp_path / "B_Composite.txt")
    assert [t for t, _, _ in fw] == [t for t, _, _ in reg]
    for (_, a, fa), (_, b, fb) in zip(fw, reg):
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(fa, fb)
    np.testing.assert_array_equal(apply("f", "m", [str(tmp_path / "fw.txt")], "w_fw.nii.gz"),
                                  apply("f", "m", [f"{p}1Warp.nii.gz", f"{p}0GenericAffine.mat"], "w_files2.nii.gz"))
    iv = write_composite([f"[{p}0GenericAffine.mat,1]", f"{p}1InverseWarp.nii.gz"], "iv.txt")
    assert [t for t, _, _ in iv] == ["DisplacementFieldTransform_float_2_2", "AffineTransform_double_2_2"]
    got = apply("m", "f", [str(tmp_path / "iv.txt")], "i_iv.nii.gz")
    bad = np.abs(got - want) > 1e-5
    assert bad.mean() < 1e-3, int(bad.sum())
    # -o [warped,0] is the plain warped output
    np.testing.assert_array_equal(apply("f", "m", [f"{q}Composite.txt"], "w0.nii.gz"),
                                  nifti.read(tmp_path / "w_comp.nii.gz", 2)[0])
    r = subprocess.run([host_cli["apply"], "-d", "2", "--float", "1", "-i", f"{tmp_path}/m.nii.gz", "-r",
                        f"{tmp_path}/f.nii.gz", "-t", f"{q}Composite.txt", "-o", f"[{tmp_path / 'w0b.nii.gz'},0]"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    np.testing.assert_array_equal(nifti.read(tmp_path / "w0b.nii.gz", 2)[0], nifti.read(tmp_path / "w_comp.nii.gz", 2)[0])


def test_large_gzip_output(host_cli, tmp_path):
    # a collapsed field of 3 x 160 x 150 x 100 floats (29 MB) is written as several gzip members; the
    # Python reader (gzip) and the C++ reader (zlib gzread, here as a -t input) both see the bytes of the
    # uncompressed file
    import gzip

    import numpy as np

    from ants_b200 import nifti
    from ants_b200.synx import Geom
    g = Geom((160, 150, 100), (1.0, 1.1, 1.2))
    nifti.write(tmp_path / "ref.nii.gz", np.zeros(g.shape, np.float32), g)
    rng = np.random.default_rng(5)
    small = Geom((20, 19, 13), (8.0, 8.7, 9.3))
    u = rng.normal(0, 1.5, small.shape + (3,)).astype(np.float32)
    nifti.write(tmp_path / "u.nii.gz", u, small, vector=True)
    for out in ("c.nii.gz", "c.nii"):
        r = subprocess.run([host_cli["apply"], "-d", "3", "--float", "1", "-r", f"{tmp_path}/ref.nii.gz",
                            "-t", f"{tmp_path}/u.nii.gz", "-o", f"[{tmp_path / out},1]"],
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
    raw = (tmp_path / "c.nii").read_bytes()
    assert len(raw) > (8 << 20) * 3
    assert gzip.open(tmp_path / "c.nii.gz").read() == raw
    members = (tmp_path / "c.nii.gz").read_bytes().count(b"\x1f\x8b\x08")
    assert members >= 3
    a, _ = nifti.read(tmp_path / "c.nii.gz", 3)
    b, _ = nifti.read(tmp_path / "c.nii", 3)
    np.testing.assert_array_equal(a, b)
    # the C++ reader: the compressed field as a transform gives the same collapsed field as the plain one
    for src, out in (("c.nii.gz", "d1.nii"), ("c.nii", "d2.nii")):
        r = subprocess.run([host_cli["apply"], "-d", "3", "--float", "1", "-r", f"{tmp_path}/ref.nii.gz",
                            "-t", f"{tmp_path}/{src}", "-o", f"[{tmp_path / out},1]"],
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
    assert (tmp_path / "d1.nii").read_bytes() == (tmp_path / "d2.nii").read_bytes()
