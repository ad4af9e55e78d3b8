"""ctypes binding of the CPU oracle (liboracle.so).  TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker;
never by the product path.  Parity unpinned: the reference arithmetic lives in ITK, which is
absent from the reference tree, and no SyN+CC golden vectors exist (see synx_oracle.hpp).

Fields are component planes: array shape (dim,) + grid.shape (component c = x, y, z).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def _geom_struct():
    import sys
    root = os.path.dirname(HERE)
    if root not in sys.path:
        sys.path.insert(0, root)
    from ants_b200.synx import SynxGeom, SynxParams  # structure layouts only (no library load)
    return SynxGeom, SynxParams


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    G, Pm = _geom_struct()
    P, V, D, I = C.POINTER, C.c_void_p, C.c_double, C.c_int
    sigs = {
        "oracle_num_threads": (I, []),
        "oracle_set_threads": (None, [I]),
        "oracle_gaussian_kernel": (I, [D, D, I, V, I]),
        "oracle_shrink_geom": (None, [P(G), C.c_uint, P(G)]),
        "oracle_run_create_f32": (V, [V, P(G), V, P(G), P(Pm)]),
        "oracle_run_advance_f32": (C.c_int64, [V, C.c_int64]),
        "oracle_run_done_f32": (I, [V]),
        "oracle_run_levels_f32": (I, [V, V, V, V, I]),
        "oracle_run_destroy_f32": (None, [V]),
    }
    for suf in ("f32", "f64"):
        sigs.update({
            f"oracle_preprocess_{suf}": (None, [V, V, C.c_int64, C.c_float, C.c_float]),
            f"oracle_histogram_match_{suf}": (None, [V, C.c_int64, V, C.c_int64, I, I, I, V]),
            f"oracle_histogram_match_table_{suf}": (None, [V, C.c_int64, V, C.c_int64, I, I, I, V, V, V, V]),
            f"oracle_smooth_image_{suf}": (None, [V, V, P(G), D, I]),
            f"oracle_warp_image_{suf}": (None, [V, P(G), V, P(G), V]),
            f"oracle_warp_image_nearest_{suf}": (None, [V, P(G), V, P(G), V]),
            f"oracle_warp_image_label_{suf}": (None, [V, P(G), V, P(G), V]),
            f"oracle_cc_{suf}": (D, [V, V, P(G), I, V, V, V]),
            f"oracle_cc_masked_{suf}": (D, [V, V, P(G), I, V, V, V, V]),
            f"oracle_syn_register_masked_{suf}": (I, [V, P(G), V, P(G), P(Pm), V, P(G), V, P(G), V, V, P(G), V, V,
                                                        V, V, V, I]),
            f"oracle_smooth_field_{suf}": (None, [V, V, P(G), D]),
            f"oracle_scale_update_{suf}": (D, [V, P(G), D]),
            f"oracle_compose_{suf}": (None, [V, V, P(G), V, D]),
            f"oracle_invert_{suf}": (I, [V, V, P(G), I, D, D, P(D), P(D)]),
            f"oracle_resample_field_{suf}": (None, [V, P(G), V, P(G)]),
            f"oracle_syn_iteration_{suf}": (D, [V, P(G), V, P(G), P(Pm), P(G), V, V, V, V, P(I)]),
            f"oracle_syn_register_{suf}": (I, [V, P(G), V, P(G), P(Pm), V, V, P(G), V, V, V, V, V, I]),
            f"oracle_syn_register_full_{suf}": (I, [V, P(G), V, P(G), P(Pm), V, P(G), V, P(G), V, V, V, V, P(G), V,
                                                      V, V, P(G), V, V, V, V, V, I]),
        })
    for n, (r, a) in sigs.items():
        f = getattr(lib, n)
        f.restype = r
        f.argtypes = a
    _lib = lib
    return lib


def _suf(dtype) -> str:
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _p(a):
    return a.ctypes.data


def set_threads(n: int) -> None:
    load().oracle_set_threads(n)


def num_threads() -> int:
    return load().oracle_num_threads()


def gaussian_kernel(variance, max_error, max_width) -> np.ndarray:
    lib = load()
    out = np.zeros(4096)
    n = lib.oracle_gaussian_kernel(variance, max_error, max_width, _p(out), 4096)
    return out[:n].copy()


def shrink_geom(g, factor):
    from ants_b200.synx import Geom, SynxGeom
    o = SynxGeom()
    gi = g.to_c()
    load().oracle_shrink_geom(C.byref(gi), factor, C.byref(o))
    return Geom.from_c(o)


def preprocess(img, qlo=0.0, qhi=1.0, dtype=np.float32):
    a = _c(img, dtype)
    out = np.empty_like(a)
    getattr(load(), f"oracle_preprocess_{_suf(dtype)}")(_p(a), _p(out), a.size, qlo, qhi)
    return out


def histogram_match(src, ref, levels=256, points=12, threshold_at_mean=True, dtype=np.float32):
    """src with its histogram matched to ref's (ITK's HistogramMatchingImageFilter restated)."""
    a, b = _c(src, dtype), _c(ref, dtype)
    out = np.empty_like(a)
    getattr(load(), f"oracle_histogram_match_{_suf(dtype)}")(_p(a), a.size, _p(b), b.size, levels, points,
                                                             int(threshold_at_mean), _p(out))
    return out


def histogram_match_table(src, ref, levels=256, points=12, threshold_at_mean=True, dtype=np.float32):
    """The match-point table: (source points, reference points, slopes, ends) with ends = (source
    min, source max, reference min, reference max, lower slope, upper slope)."""
    a, b = _c(src, dtype), _c(ref, dtype)
    ts, tr, gr, ends = np.zeros(points + 2), np.zeros(points + 2), np.zeros(points + 1), np.zeros(6)
    getattr(load(), f"oracle_histogram_match_table_{_suf(dtype)}")(_p(a), a.size, _p(b), b.size, levels, points,
                                                                   int(threshold_at_mean), _p(ts), _p(tr), _p(gr),
                                                                   _p(ends))
    return ts, tr, gr, ends


def smooth_image(img, g, sigma, mm=False, dtype=np.float32):
    a = _c(img, dtype)
    out = np.empty_like(a)
    gc = g.to_c()
    getattr(load(), f"oracle_smooth_image_{_suf(dtype)}")(_p(a), _p(out), C.byref(gc), sigma, int(mm))
    return out


def warp_image(img, gi, u, gv, dtype=np.float32, nearest=False, label=False):
    a, uu = _c(img, dtype), _c(u, dtype)
    out = np.empty(gv.shape, dtype)
    ga, gb = gi.to_c(), gv.to_c()
    name = "oracle_warp_image_label_" if label else "oracle_warp_image_nearest_" if nearest else "oracle_warp_image_"
    getattr(load(), name + _suf(dtype))(_p(a), C.byref(ga), _p(uu), C.byref(gb), _p(out))
    return out


def cc_metric(F, M, g, radius, dtype=np.float32, valid=None):
    """Returns (value, grad_fixed_update, grad_moving_update, local_cc).  `valid` (bool per voxel):
    the metric masks' validity; invalid voxels are left out of the window sums and get no value."""
    f, m = _c(F, dtype), _c(M, dtype)
    gF = np.empty((g.dim,) + g.shape, dtype)
    gM = np.empty_like(gF)
    cc = np.empty(g.shape, dtype)
    gc = g.to_c()
    if valid is None:
        v = getattr(load(), f"oracle_cc_{_suf(dtype)}")(_p(f), _p(m), C.byref(gc), radius, _p(gF), _p(gM), _p(cc))
    else:
        vb = np.ascontiguousarray(valid, dtype=np.uint8)
        v = getattr(load(), f"oracle_cc_masked_{_suf(dtype)}")(_p(f), _p(m), C.byref(gc), radius, _p(vb), _p(gF),
                                                               _p(gM), _p(cc))
    return v, gF, gM, cc


def smooth_field(u, g, variance, dtype=np.float32):
    a = _c(u, dtype)
    out = np.empty_like(a)
    gc = g.to_c()
    getattr(load(), f"oracle_smooth_field_{_suf(dtype)}")(_p(a), _p(out), C.byref(gc), variance)
    return out


def scale_update(u, g, eta, dtype=np.float32):
    a = _c(u, dtype).copy()
    gc = g.to_c()
    mx = getattr(load(), f"oracle_scale_update_{_suf(dtype)}")(_p(a), C.byref(gc), eta)
    return a, mx


def compose(d, w, g, scale=1.0, dtype=np.float32):
    dd, ww = _c(d, dtype), _c(w, dtype)
    out = np.empty_like(ww)
    gc = g.to_c()
    getattr(load(), f"oracle_compose_{_suf(dtype)}")(_p(dd), _p(ww), C.byref(gc), _p(out), scale)
    return out


def invert(phi, psi0, g, max_iter=20, mean_tol=0.001, max_tol=0.1, dtype=np.float32):
    p, q = _c(phi, dtype), _c(psi0, dtype).copy()
    gc = g.to_c()
    mean, mx = C.c_double(), C.c_double()
    it = getattr(load(), f"oracle_invert_{_suf(dtype)}")(_p(p), _p(q), C.byref(gc), max_iter, mean_tol, max_tol,
                                                          C.byref(mean), C.byref(mx))
    return q, it, mean.value, mx.value


def resample_field(u, gi, go, dtype=np.float32):
    a = _c(u, dtype)
    out = np.empty((go.dim,) + go.shape, dtype)
    ga, gb = gi.to_c(), go.to_c()
    getattr(load(), f"oracle_resample_field_{_suf(dtype)}")(_p(a), C.byref(ga), _p(out), C.byref(gb))
    return out


def syn_iteration(Fs, gF, Ms, gM, params, g, phiF, psiF, phiM, psiM, dtype=np.float32):
    """One SyN iteration on the four half-fields (returned updated) from pre-smoothed images."""
    f, m = _c(Fs, dtype), _c(Ms, dtype)
    flds = [_c(a, dtype).copy() for a in (phiF, psiF, phiM, psiM)]
    pc = params.to_c()
    ga, gb, gg = gF.to_c(), gM.to_c(), g.to_c()
    k = C.c_int()
    v = getattr(load(), f"oracle_syn_iteration_{_suf(dtype)}")(_p(f), C.byref(ga), _p(m), C.byref(gb), C.byref(pc),
                                                               C.byref(gg), *[_p(a) for a in flds], C.byref(k))
    return v, flds, k.value


def syn_register(F, gF, M, gM, params, dtype=np.float32, fixed_mask=None, fixed_mask_geom=None, moving_mask=None,
                 moving_mask_geom=None, initial_half_fields=None, initial_geom=None, return_half_fields=False):
    """Full stage: returns (forward, inverse, out_geom, log) with fields as component planes.  Metric
    masks (nonzero = inside) on their own grids (default: the image's grid) are optional.
    initial_half_fields: (phiF, psiF, phiM, psiM) as component planes on initial_geom, the stage's
    starting half-fields (resampled to the first level's grid), or None for zero fields.  With
    return_half_fields the final half-fields are returned as a fifth item."""
    from ants_b200.synx import Geom, SynxGeom
    f, m = _c(F, dtype), _c(M, dtype)
    g_last = gF
    for s in params.shrink_factors[-1:]:
        g_last = shrink_geom(gF, s)
    fwd = np.empty((g_last.dim,) + g_last.shape, dtype)
    inv = np.empty_like(fwd)
    half = np.empty((4, g_last.dim) + g_last.shape, dtype) if return_half_fields else None
    cap = int(sum(params.iterations)) + 1
    lv = np.zeros(cap, np.int32)
    it = np.zeros(cap, np.int32)
    me = np.zeros(cap)
    cv = np.zeros(cap)
    ki = np.zeros(cap, np.int32)
    go = SynxGeom()
    pc = params.to_c()
    ga, gb = gF.to_c(), gM.to_c()
    mf = _c(fixed_mask, dtype) if fixed_mask is not None else None
    mm = _c(moving_mask, dtype) if moving_mask is not None else None
    gmf = (fixed_mask_geom or gF).to_c() if mf is not None else None
    gmm = (moving_mask_geom or gM).to_c() if mm is not None else None
    ini = [None] * 4
    gi = None
    if initial_half_fields is not None:
        ini = [_c(a, dtype) for a in initial_half_fields]
        gi = (initial_geom or gF).to_c()
    n = getattr(load(), f"oracle_syn_register_full_{_suf(dtype)}")(
        _p(f), C.byref(ga), _p(m), C.byref(gb), C.byref(pc), _p(mf) if mf is not None else None,
        C.byref(gmf) if gmf is not None else None, _p(mm) if mm is not None else None,
        C.byref(gmm) if gmm is not None else None, *[(_p(a) if a is not None else None) for a in ini],
        C.byref(gi) if gi is not None else None, _p(fwd), _p(inv), _p(half) if half is not None else None,
        C.byref(go), _p(lv), _p(it), _p(me), _p(cv), _p(ki), cap)
    log = [dict(level=int(lv[i]), iteration=int(it[i]), metric=float(me[i]), convergence=float(cv[i]),
                inverse_iterations=int(ki[i])) for i in range(min(n, cap))]
    if return_half_fields:
        return fwd, inv, Geom.from_c(go), log, half
    return fwd, inv, Geom.from_c(go), log


class SynRun:
    """A float32 stage run that is advanced a bounded number of SyN iterations at a time (level
    set-ups and the final composition included), so that one complete registration can be split
    over several timed steps.  Running it to the end computes what syn_register computes."""

    def __init__(self, F, gF, M, gM, params):
        self._keep = (_c(F, np.float32), _c(M, np.float32), gF.to_c(), gM.to_c(), params.to_c())
        f, m, ga, gb, pc = self._keep
        self.n_levels = int(params.n_levels) if hasattr(params, "n_levels") else len(params.iterations)
        self.h = load().oracle_run_create_f32(_p(f), C.byref(ga), _p(m), C.byref(gb), C.byref(pc))

    def advance(self, n: int) -> int:
        return int(load().oracle_run_advance_f32(self.h, n))

    @property
    def done(self) -> bool:
        return bool(load().oracle_run_done_f32(self.h))

    def levels(self):
        """[(voxel-iterations, seconds in iterations, iterations run)] per level."""
        L = self.n_levels
        vi = np.zeros(L, np.int64)
        sec = np.zeros(L)
        it = np.zeros(L, np.int32)
        load().oracle_run_levels_f32(self.h, _p(vi), _p(sec), _p(it), L)
        return [(int(a), float(b), int(c)) for a, b, c in zip(vi, sec, it)]

    def close(self):
        if self.h:
            load().oracle_run_destroy_f32(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
