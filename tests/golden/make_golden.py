"""Generate the known-answer fixtures in tests/golden/ with code independent of the oracle.

The reference ships no SyN+CC golden vectors and its arithmetic lives in ITK (absent from
the reference tree), so these fixtures restate the published definitions directly:

* gaussian_kernels.json -- Lindeberg's discrete Gaussian e^{-t} I_n(t) from scipy's
  exponentially scaled Bessel functions (scipy.special.ive), grown with the GaussianOperator
  stopping rule (two-sided mass >= 1 - max_error, or half-width > max_width), normalised.
* cc_bruteforce.npz -- neighbourhood CC value and both update directions on tiny seeded
  images, by explicit loops over each voxel's in-bounds window (the definition in
  ImageRegistration/itkCrossCorrelationRegistrationFunction.cxx:179-306, :379-504) and the
  half-voxel central difference of ITK's CentralDifferenceImageFunction.

Run: python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os

import numpy as np
from scipy import special

HERE = os.path.dirname(os.path.abspath(__file__))


def discrete_gaussian(variance: float, max_error: float, max_width: int) -> list[float]:
    if variance <= 0:
        return [1.0]
    half = [special.ive(0, variance), special.ive(1, variance)]
    total = half[0] + 2 * half[1]
    i = 2
    while total < 1.0 - max_error:
        half.append(special.ive(i, variance))
        total += 2 * half[-1]
        if len(half) > max_width:
            break
        i += 1
    half = np.array(half) / total
    return list(np.concatenate([half[:0:-1], half]))


def grad_axis(I: np.ndarray, idx: tuple, axis: int, h: float) -> float:
    n = I.shape[axis]
    pos = idx[axis]
    if n < 2 or pos == n - 1:
        return 0.0
    up = list(idx)
    up[axis] += 1
    if pos == 0:
        return 0.5 * (float(I[tuple(up)]) - float(I[idx])) / h
    dn = list(idx)
    dn[axis] -= 1
    return (float(I[tuple(up)]) - float(I[tuple(dn)])) / (2 * h)


def cc_bruteforce(F: np.ndarray, M: np.ndarray, r: int, spacing: tuple, eps: float = 1.1920928955078125e-07):
    """numpy arrays indexed [z][y][x] (or [y][x]); spacing in x, y, z order."""
    d = F.ndim
    gF = np.zeros((d,) + F.shape)
    gM = np.zeros((d,) + F.shape)
    ccs = np.zeros(F.shape)
    for idx in np.ndindex(F.shape):
        sl = tuple(slice(max(i - r, 0), min(i + r, n - 1) + 1) for i, n in zip(idx, F.shape))
        f = F[sl].astype(np.float64).ravel()
        m = M[sl].astype(np.float64).ravel()
        n = f.size
        sF, sM = f.sum(), m.sum()
        mF, mM = sF / n, sM / n
        sFF = (f * f).sum() - 2 * mF * sF + n * mF * mF
        sMM = (m * m).sum() - 2 * mM * sM + n * mM * mM
        sFM = (f * m).sum() - mM * sF - mF * sM + n * mM * mF
        fh = float(F[idx]) - mF
        mh = float(M[idx]) - mM
        cc, aF, aM = 1.0, 0.0, 0.0
        if sFF > eps and sMM > eps:
            cc = sFM * sFM / (sFF * sMM)
            coef = 2 * sFM / (sFF * sMM)
            aF = coef * (fh - sFM / sMM * mh)
            aM = coef * (mh - sFM / sFF * fh)
        ccs[idx] = cc
        # numpy axis a corresponds to ITK axis d-1-a
        for comp in range(d):
            ax = d - 1 - comp
            gF[comp][idx] = aF * grad_axis(M, idx, ax, spacing[comp])
            gM[comp][idx] = aM * grad_axis(F, idx, ax, spacing[comp])
    return -ccs.mean(), gF, gM, ccs


def cc_bruteforce_masked(F: np.ndarray, M: np.ndarray, valid: np.ndarray, r: int, spacing: tuple,
                         eps: float = 1.1920928955078125e-07):
    """The same over the valid voxels only: invalid voxels are left out of every window sum and of the
    count n, and an invalid centre has no cc and no derivative; value = -mean cc over valid centres."""
    d = F.ndim
    gF = np.zeros((d,) + F.shape)
    gM = np.zeros((d,) + F.shape)
    ccs = np.zeros(F.shape)
    total, count = 0.0, 0
    for idx in np.ndindex(F.shape):
        if not valid[idx]:
            continue
        sl = tuple(slice(max(i - r, 0), min(i + r, n - 1) + 1) for i, n in zip(idx, F.shape))
        keep = valid[sl].ravel().astype(bool)
        f = F[sl].astype(np.float64).ravel()[keep]
        m = M[sl].astype(np.float64).ravel()[keep]
        n = f.size
        sF, sM = f.sum(), m.sum()
        mF, mM = sF / n, sM / n
        sFF = (f * f).sum() - 2 * mF * sF + n * mF * mF
        sMM = (m * m).sum() - 2 * mM * sM + n * mM * mM
        sFM = (f * m).sum() - mM * sF - mF * sM + n * mM * mF
        fh = float(F[idx]) - mF
        mh = float(M[idx]) - mM
        cc, aF, aM = 1.0, 0.0, 0.0
        if sFF > eps and sMM > eps:
            cc = sFM * sFM / (sFF * sMM)
            coef = 2 * sFM / (sFF * sMM)
            aF = coef * (fh - sFM / sMM * mh)
            aM = coef * (mh - sFM / sFF * fh)
        ccs[idx] = cc
        total += cc
        count += 1
        for comp in range(d):
            ax = d - 1 - comp
            gF[comp][idx] = aF * grad_axis(M, idx, ax, spacing[comp])
            gM[comp][idx] = aM * grad_axis(F, idx, ax, spacing[comp])
    return (-total / count if count else 0.0), gF, gM, ccs


def main() -> None:
    kernels = []
    for var in (0.25, 0.5, 1.0, 2.0, 3.0, 4.5, 9.0):
        for err, width in ((0.001, 1000), (0.01, 32), (0.001, 3)):
            kernels.append({"variance": var, "max_error": err, "max_width": width,
                            "coefficients": discrete_gaussian(var, err, width)})
    with open(os.path.join(HERE, "gaussian_kernels.json"), "w") as fh:
        json.dump(kernels, fh, indent=1)

    rng = np.random.default_rng(20240607)
    cases = {}
    shapes = {"2d": ((7, 9), (1.0, 1.3)), "3d": ((4, 5, 6), (1.0, 0.8, 1.5))}
    for name, (shape, sp) in shapes.items():
        base = rng.uniform(0.0, 1.0, shape)
        F = (base + 0.05 * rng.standard_normal(shape)).astype(np.float32)
        M = (np.roll(base, 1, axis=-1) + 0.05 * rng.standard_normal(shape)).astype(np.float32)
        for r in (1, 2):
            v, gF, gM, cc = cc_bruteforce(F, M, r, sp)
            cases[f"{name}_r{r}_F"] = F
            cases[f"{name}_r{r}_M"] = M
            cases[f"{name}_r{r}_spacing"] = np.array(sp)
            cases[f"{name}_r{r}_value"] = np.array(v)
            cases[f"{name}_r{r}_gF"] = gF
            cases[f"{name}_r{r}_gM"] = gM
            cases[f"{name}_r{r}_cc"] = cc
    np.savez_compressed(os.path.join(HERE, "cc_bruteforce.npz"), **cases)


if __name__ == "__main__":
    main()
