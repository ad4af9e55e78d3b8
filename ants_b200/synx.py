"""ctypes binding of the synx C ABI (include/synx.h).

This is the Python mirror of the reference's stage interface: a `SyNStage` is configured
with the values antsRegistration parses from `-t SyN[...] -m CC[...] -c ... -f ... -s ...`
(Examples/antsRegistrationTemplateHeader.h:545-651, :801-815, :1081-1087) and run on one
fixed/moving pair; it returns the forward (prefix0Warp) and inverse (prefix0InverseWarp)
displacement fields.  Every call goes through libsynx.so; there is no CPU path.  Loading the
library fails loudly if it has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsynx.so")

SYNX_MAX_LEVELS = 8
SYNX_F_PROFILE_EVENTS = 0x1
SYNX_F_USE_GRAPHS = 0x2
SYNX_F_NO_PERSISTENT = 0x4
SYNX_F_CC_FP32_SUMS = 0x8
SYNX_F_FIELDS_FP16 = 0x10
SYNX_F_SMOOTH_TWO_PASS = 0x20
SYNX_F_INV_TWO_PASS = 0x40
SYNX_F_NO_PDL = 0x80
SYNX_INJECT_BARRIER_TIMEOUT = 1
SYNX_INJECT_ALLOC_FAILURE = 2

ERRORS = {-1: "invalid argument", -2: "bad state", -3: "CUDA error", -4: "out of device memory", -5: "unsupported"}


class SynxGeom(C.Structure):
    _fields_ = [
        ("dim", C.c_int32),
        ("reserved0", C.c_int32),
        ("size", C.c_int64 * 3),
        ("spacing", C.c_double * 3),
        ("origin", C.c_double * 3),
        ("direction", C.c_double * 9),
    ]


class SynxLinear(C.Structure):
    """synx_linear: T(p) = A (p - c) + t + c on physical (LPS) points."""
    _fields_ = [
        ("dim", C.c_int32),
        ("has_center", C.c_int32),
        ("matrix", C.c_double * 9),
        ("translation", C.c_double * 3),
        ("center", C.c_double * 3),
    ]


class SynxParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int32),
        ("n_levels", C.c_int32),
        ("learning_rate", C.c_double),
        ("update_variance", C.c_double),
        ("total_variance", C.c_double),
        ("cc_radius", C.c_int32),
        ("sigmas_in_mm", C.c_int32),
        ("iterations", C.c_int32 * SYNX_MAX_LEVELS),
        ("shrink_factors", C.c_int32 * SYNX_MAX_LEVELS),
        ("smoothing_sigmas", C.c_double * SYNX_MAX_LEVELS),
        ("convergence_threshold", C.c_double),
        ("convergence_window", C.c_int32),
        ("preprocess", C.c_int32),
        ("winsor_lower", C.c_float),
        ("winsor_upper", C.c_float),
        ("inv_max_iter", C.c_int32),
        ("flags", C.c_int32),
        ("inv_mean_tol", C.c_double),
        ("inv_max_tol", C.c_double),
        ("persistent_blocks", C.c_int32),
        ("persistent_max_voxels", C.c_int32),
        ("test_inject", C.c_int32),
        ("histogram_match", C.c_int32),
        ("smooth_tile_rows", C.c_int32),
        ("cc_z_chunks", C.c_int32),
        ("tuning", C.c_int32),
        ("reserved", C.c_int32 * 1),
    ]


class SynxServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_active", C.c_int32), ("hbm_budget_bytes", C.c_int64),
                ("reserved", C.c_int32 * 8)]


class SynxRequestInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("levels_done", C.c_int32), ("device_bytes", C.c_int64),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double), ("error", C.c_char * 256)]


class SynxServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64), ("queued", C.c_int64),
                ("resident", C.c_int64), ("bytes_resident", C.c_int64), ("bytes_peak", C.c_int64),
                ("budget", C.c_int64), ("bytes_pooled", C.c_int64), ("steps", C.c_int64), ("step_seconds", C.c_double),
                ("resident_byte_seconds", C.c_double), ("elapsed", C.c_double)]


# ---- geometry --------------------------------------------------------------------------------
@dataclass
class Geom:
    """ITK image information: p = origin + direction @ diag(spacing) @ index (index x-fastest)."""

    size: tuple  # (nx, ny) or (nx, ny, nz)
    spacing: tuple = None
    origin: tuple = None
    direction: np.ndarray = None

    def __post_init__(self):
        d = len(self.size)
        if d not in (2, 3):
            raise ValueError("size must have 2 or 3 entries")
        self.size = tuple(int(s) for s in self.size)
        self.spacing = tuple(float(s) for s in (self.spacing or (1.0,) * d))
        self.origin = tuple(float(s) for s in (self.origin or (0.0,) * d))
        if self.direction is None:
            self.direction = np.eye(d)
        self.direction = np.asarray(self.direction, dtype=np.float64).reshape(d, d)

    @property
    def dim(self) -> int:
        return len(self.size)

    @property
    def count(self) -> int:
        return int(np.prod(self.size))

    @property
    def shape(self) -> tuple:
        """numpy shape of an image on this grid (z, y, x) / (y, x)."""
        return tuple(reversed(self.size))

    def to_c(self) -> SynxGeom:
        g = SynxGeom()
        d = self.dim
        g.dim = d
        for k in range(3):
            g.size[k] = self.size[k] if k < d else 1
            g.spacing[k] = self.spacing[k] if k < d else 1.0
            g.origin[k] = self.origin[k] if k < d else 0.0
        m = np.eye(3)
        m[:d, :d] = self.direction
        for k in range(9):
            g.direction[k] = float(m.flat[k])
        return g

    @staticmethod
    def from_c(g: SynxGeom) -> "Geom":
        d = g.dim
        m = np.array(list(g.direction), dtype=np.float64).reshape(3, 3)[:d, :d]
        return Geom(tuple(g.size[k] for k in range(d)), tuple(g.spacing[k] for k in range(d)),
                    tuple(g.origin[k] for k in range(d)), m)


# ---- library loading -------------------------------------------------------------------------
_lib = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load libsynx.so; raises if it is missing (build it with `python -m ants_b200.build`)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libsynx.so not built at {path}; run `python -m ants_b200.build`")
    lib = C.CDLL(path)
    P, I, D, F, V = C.POINTER, C.c_int, C.c_double, C.c_float, C.c_void_p
    sig = {
        "synx_params_default": (I, [P(SynxParams), I]),
        "synx_create": (I, [P(SynxParams), I, V, P(V)]),
        "synx_destroy": (I, [V]),
        "synx_last_error": (C.c_char_p, [V]),
        "synx_set_images": (I, [V, V, P(SynxGeom), V, P(SynxGeom)]),
        "synx_set_images_device": (I, [V, V, P(SynxGeom), V, P(SynxGeom)]),
        "synx_run": (I, [V]),
        "synx_run_level": (I, [V, I]),
        "synx_get_output_geom": (I, [V, P(SynxGeom)]),
        "synx_get_fields": (I, [V, V, V]),
        "synx_get_fields_device": (I, [V, V, V]),
        "synx_get_half_fields": (I, [V, V, V, V, V]),
        "synx_set_half_fields": (I, [V, V, V, V, V, P(SynxGeom)]),
        "synx_set_initial_half_fields": (I, [V, V, V, V, V, P(SynxGeom)]),
        "synx_get_log": (I, [V, V, V, V, V, V, C.c_int64, P(C.c_int64)]),
        "synx_get_profile": (I, [V, P(D), P(C.c_int64), P(C.c_int64), P(D), P(C.c_int64), P(C.c_int64)]),
        "synx_reset_profile": (I, [V]),
        "synx_get_level_profile": (I, [V, I, P(D), P(D), P(D), P(D), P(C.c_int64), P(C.c_int64), P(C.c_int64)]),
        "synx_get_device_bytes": (I, [V, P(C.c_int64)]),
        "synx_get_launch_count": (I, [P(C.c_int64)]),
        "synx_gaussian_kernel": (I, [D, D, I, V, I, P(I)]),
        "synx_smooth_image": (I, [V, V, P(SynxGeom), D, I, V]),
        "synx_warp_image": (I, [V, P(SynxGeom), V, P(SynxGeom), V, V]),
        "synx_warp_image_nearest": (I, [V, P(SynxGeom), V, P(SynxGeom), V, V]),
        "synx_warp_image_label": (I, [V, P(SynxGeom), V, P(SynxGeom), V, V]),
        "synx_histogram_match": (I, [V, C.c_int64, V, C.c_int64, C.c_int32, C.c_int32, C.c_int32, V, V]),
        "synx_cc_metric": (I, [V, V, P(SynxGeom), I, V, V, P(D), V]),
        "synx_cc_metric_noalloc": (I, [V, V, P(SynxGeom), I, V, V, P(D), V]),
        "synx_cc_metric_ex": (I, [V, V, P(SynxGeom), I, I, V, V, P(D), V]),
        "synx_noalloc_last_error": (C.c_char_p, []),
        "synx_smooth_field": (I, [V, V, P(SynxGeom), D, P(D), V]),
        "synx_compose": (I, [V, V, P(SynxGeom), F, V, V]),
        "synx_invert_field": (I, [V, V, P(SynxGeom), I, D, D, P(I), V]),
        "synx_resample_field": (I, [V, P(SynxGeom), V, P(SynxGeom), V]),
        "synx_shrink_geom": (I, [P(SynxGeom), I, P(SynxGeom)]),
        "synx_batch_create": (I, [I, P(V)]),
        "synx_batch_destroy": (I, [V]),
        "synx_batch_last_error": (C.c_char_p, [V]),
        "synx_batch_step": (I, [V, P(V), I, V, P(I)]),
        "synx_batch_run": (I, [V, P(V), I, V]),
        "synx_footprint": (I, [P(SynxParams), P(SynxGeom), P(SynxGeom), P(C.c_int64)]),
        "synx_server_create": (I, [P(SynxServerConfig), P(V)]),
        "synx_server_destroy": (I, [V]),
        "synx_server_last_error": (C.c_char_p, [V]),
        "synx_server_submit": (I, [V, P(SynxParams), V, P(SynxGeom), V, P(SynxGeom), V, V, P(C.c_int64)]),
        "synx_server_wait": (I, [V, C.c_int64, D, P(SynxRequestInfo)]),
        "synx_server_get_stats": (I, [V, P(SynxServerStats)]),
        "synx_read_linear_transform": (I, [C.c_char_p, I, I, P(SynxLinear)]),
        "synx_linear_from_parameters": (I, [C.c_char_p, P(D), I, P(D), I, I, P(SynxLinear)]),
        "synx_linear_field": (I, [P(SynxLinear), I, P(SynxGeom), V]),
        "synx_write_linear_transform": (I, [C.c_char_p, P(SynxLinear)]),
        "synx_initial_translation": (I, [V, P(SynxGeom), V, P(SynxGeom), I, P(SynxLinear)]),
        "synx_set_masks": (I, [V, V, P(SynxGeom), V, P(SynxGeom)]),
        "synx_cc_metric_masked": (I, [V, V, V, P(SynxGeom), I, V, V, P(D), V]),
        "synx_tuning_load": (I, [C.c_char_p]),
        "synx_tuning_path": (C.c_char_p, []),
        "synx_level_plan": (I, [V, I, P(C.c_int32), P(C.c_int32), P(C.c_int32)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class SynxError(RuntimeError):
    pass


def _check(rc: int, ctx=None) -> None:
    if rc != 0:
        lib = load_library()
        msg = lib.synx_last_error(ctx).decode(errors="replace") if lib else ""
        raise SynxError(f"synx error {rc} ({ERRORS.get(rc, '?')}): {msg}")


def _ptr(a) -> int:
    """Raw pointer of a numpy array or torch tensor (device pointers for CUDA tensors)."""
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    return a.data_ptr()


def _dev(t, numel: int, name: str) -> int:
    """Device pointer of a contiguous float32 CUDA tensor with at least `numel` values.  Anything else
    is refused here: a host pointer or a short buffer reaching a kernel would be a memory fault."""
    if isinstance(t, np.ndarray) or not getattr(t, "is_cuda", False):
        raise SynxError(f"{name}: a CUDA tensor is required")
    if str(t.dtype) != "torch.float32" or not t.is_contiguous():
        raise SynxError(f"{name}: a contiguous float32 tensor is required")
    if t.numel() < numel:
        raise SynxError(f"{name}: {t.numel()} values, the geometry needs {numel}")
    return t.data_ptr()


def _host(a, numel: int, name: str) -> np.ndarray:
    """A C-contiguous float32 copy (or view) of a host array with exactly `numel` values."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.size != numel:
        raise SynxError(f"{name}: {a.size} values, the geometry needs {numel}")
    return a


# ---- stage parameters --------------------------------------------------------------------------
@dataclass
class SyNParams:
    """A SyN stage with the CC metric, as antsRegistration's -t/-m/-c/-f/-s options give it."""

    dim: int = 3
    learning_rate: float = 0.1
    update_variance: float = 3.0
    total_variance: float = 0.0
    cc_radius: int = 4
    iterations: Sequence[int] = (1,)
    shrink_factors: Sequence[int] = (1,)
    smoothing_sigmas: Sequence[float] = (0.0,)
    sigmas_in_mm: bool = False
    convergence_threshold: float = 1e-6
    convergence_window: int = 10
    preprocess: bool = True
    winsor_lower: float = 0.0
    winsor_upper: float = 1.0
    inv_max_iter: int = 20
    inv_mean_tol: float = 0.001
    inv_max_tol: float = 0.1
    flags: int = 0
    persistent_blocks: int = 0  # launch shape of the persistent level kernel (0: automatic)
    persistent_max_voxels: int = 0  # largest level it runs (0: automatic)
    test_inject: int = 0  # SYNX_INJECT_* (failure-detection tests)
    histogram_match: bool = False  # --use-histogram-matching 1: the moving image matched to the fixed one
    smooth_tile_rows: int = 0  # 3-D smoothing: 8/16 slab, -1 two kernels, -2/-3 pipelined xy, 0 table / model
    cc_z_chunks: int = 0  # CC kernel z chunks, 0 tuned table / model
    tuning: int = 0  # 0: per-level plans from the tuning table; 1: built-in cost models only

    def to_c(self) -> SynxParams:
        n = len(self.iterations)
        if not (len(self.shrink_factors) == n and len(self.smoothing_sigmas) == n):
            raise ValueError("iterations, shrink factors and smoothing sigmas must have one entry per level")
        if n < 1 or n > SYNX_MAX_LEVELS:
            raise ValueError("between 1 and 8 levels")
        p = SynxParams()  # zero-initialised; every field is set below
        p.dim = self.dim
        p.n_levels = n
        p.learning_rate = self.learning_rate
        p.update_variance = self.update_variance
        p.total_variance = self.total_variance
        p.cc_radius = self.cc_radius
        p.sigmas_in_mm = int(self.sigmas_in_mm)
        for i in range(n):
            p.iterations[i] = int(self.iterations[i])
            p.shrink_factors[i] = int(self.shrink_factors[i])
            p.smoothing_sigmas[i] = float(self.smoothing_sigmas[i])
        p.convergence_threshold = self.convergence_threshold
        p.convergence_window = self.convergence_window
        p.preprocess = int(self.preprocess)
        p.winsor_lower = self.winsor_lower
        p.winsor_upper = self.winsor_upper
        p.inv_max_iter = self.inv_max_iter
        p.inv_mean_tol = self.inv_mean_tol
        p.inv_max_tol = self.inv_max_tol
        p.flags = self.flags
        p.persistent_blocks = self.persistent_blocks
        p.persistent_max_voxels = self.persistent_max_voxels
        p.test_inject = self.test_inject
        p.histogram_match = int(self.histogram_match)
        p.smooth_tile_rows = int(self.smooth_tile_rows)
        p.cc_z_chunks = int(self.cc_z_chunks)
        p.tuning = int(self.tuning)
        return p


@dataclass
class LogRecord:
    level: int
    iteration: int
    metric: float
    convergence: float
    inverse_iterations: int


def footprint(params: "SyNParams", fixed_geom: "Geom", moving_geom: "Geom") -> int:
    """Device bytes a stage holds for these grids (synx_footprint)."""
    lib = load_library()
    cp, gf, gm = params.to_c(), fixed_geom.to_c(), moving_geom.to_c()
    b = C.c_int64(0)
    _check(lib.synx_footprint(C.byref(cp), C.byref(gf), C.byref(gm), C.byref(b)))
    return b.value


class Server:
    """The serving loop (synx_server_*): submit registration requests from any thread; a server
    thread admits them by device footprint and advances all resident ones together, one pyramid
    level per step.  Results go to host arrays this object allocates per request."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, max_active: int = 0):
        self.lib = load_library()
        cfg = SynxServerConfig(device, max_active, hbm_budget_bytes)
        h = C.c_void_p()
        rc = self.lib.synx_server_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise SynxError(f"synx error {rc}: {self.lib.synx_server_last_error(None).decode(errors='replace')}")
        self.h = h
        self._live = {}

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.synx_server_destroy(self.h)
            self.h = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _err(self, rc):
        raise SynxError(f"synx error {rc} ({ERRORS.get(rc, '?')}): "
                        f"{self.lib.synx_server_last_error(self.h).decode(errors='replace')}")

    def submit(self, params: "SyNParams", fixed: np.ndarray, fixed_geom: "Geom", moving: np.ndarray,
               moving_geom: "Geom", out: tuple | None = None) -> int:
        """Queue a request; `out` = (forward, inverse) float32 host arrays of shape
        fixed_geom.shape + (dim,) to receive the fields (allocated here when omitted; pass pinned
        arrays for faster copies)."""
        f = _host(fixed, fixed_geom.count, "fixed")
        m = _host(moving, moving_geom.count, "moving")
        shp = tuple(fixed_geom.shape) + (params.dim,)
        if out is None:
            fwd = np.empty(shp, np.float32)
            inv = np.empty(shp, np.float32)
        else:
            fwd, inv = out
            if fwd.shape != shp or inv.shape != shp or fwd.dtype != np.float32 or inv.dtype != np.float32 or \
                    not (fwd.flags["C_CONTIGUOUS"] and inv.flags["C_CONTIGUOUS"]):
                raise ValueError(f"output arrays must be C-contiguous float32 of shape {shp}")
        cp, gf, gm = params.to_c(), fixed_geom.to_c(), moving_geom.to_c()
        rid = C.c_int64(0)
        rc = self.lib.synx_server_submit(self.h, C.byref(cp), _ptr(f), C.byref(gf), _ptr(m), C.byref(gm), _ptr(fwd),
                                         _ptr(inv), C.byref(rid))
        if rc != 0:
            self._err(rc)
        self._live[rid.value] = (f, m, fwd, inv)
        return rid.value

    def wait(self, rid: int, timeout: float = -1.0):
        """Blocks until request `rid` is done; returns (forward, inverse, info dict)."""
        info = SynxRequestInfo()
        rc = self.lib.synx_server_wait(self.h, rid, float(timeout), C.byref(info))
        if rc != 0:
            if rc != -2:  # a timeout leaves the request running; anything else ended it
                self._live.pop(rid, None)
            self._err(rc)
        _, _, fwd, inv = self._live.pop(rid)
        d = {k: getattr(info, k) for k in ("status", "levels_done", "device_bytes", "t_submit", "t_admit", "t_done")}
        return fwd, inv, d

    def stats(self) -> dict:
        st = SynxServerStats()
        rc = self.lib.synx_server_get_stats(self.h, C.byref(st))
        if rc != 0:
            self._err(rc)
        return {k: getattr(st, k) for k, _ in SynxServerStats._fields_}


class Batch:
    """Advances many SyN stages together (synx_batch_*): each step runs every stage's next level,
    the small levels of all stages sharing cooperative launches.  A stage's results do not depend
    on what else is in the batch."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        _check(self.lib.synx_batch_create(device, C.byref(h)))
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.synx_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _ck(self, rc):
        if rc != 0:
            msg = self.lib.synx_batch_last_error(self.h).decode(errors="replace")
            raise SynxError(f"synx error {rc} ({ERRORS.get(rc, '?')}): {msg}")

    @staticmethod
    def _handles(stages):
        arr = (C.c_void_p * max(len(stages), 1))()
        for i, st in enumerate(stages):
            arr[i] = st.h
        return arr

    def step(self, stages, stream: int | None = None) -> int:
        """Run the next level of every stage that has one; returns how many ran a level."""
        adv = C.c_int(0)
        self._ck(self.lib.synx_batch_step(self.h, self._handles(stages), len(stages), C.c_void_p(stream or 0),
                                          C.byref(adv)))
        return adv.value

    def run(self, stages, stream: int | None = None) -> None:
        """Run every remaining level of every stage."""
        self._ck(self.lib.synx_batch_run(self.h, self._handles(stages), len(stages), C.c_void_p(stream or 0)))


class SyNStage:
    """One registration context on one GPU (synx_create ... synx_destroy)."""

    def __init__(self, params: SyNParams, device: int = 0, stream: int | None = None):
        self.lib = load_library()
        self.params = params
        self._cp = params.to_c()
        h = C.c_void_p()
        _check(self.lib.synx_create(C.byref(self._cp), device, C.c_void_p(stream or 0), C.byref(h)))
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.synx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _ck(self, rc):
        _check(rc, self.h)

    def set_masks(self, fixed_mask=None, fixed_mask_geom: Geom | None = None, moving_mask=None,
                  moving_mask_geom: Geom | None = None) -> None:
        """Metric masks (antsRegistration -x): host arrays, nonzero = inside, on their own grids;
        None for none.  They stay set across set_images calls."""
        args = []
        keep = []
        for m, gm in ((fixed_mask, fixed_mask_geom), (moving_mask, moving_mask_geom)):
            if m is None:
                args += [None, None]
                continue
            if gm is None:
                raise SynxError("a mask needs its geometry")
            a = np.ascontiguousarray(m, dtype=np.float32)
            if a.size != gm.count:
                raise SynxError("mask size does not match its geometry")
            gc = gm.to_c()
            keep += [a, gc]
            args += [_ptr(a), C.byref(gc)]
        self._ck(self.lib.synx_set_masks(self.h, *args))

    def set_images(self, fixed, fixed_geom: Geom, moving, moving_geom: Geom, moving_initial=None) -> None:
        """Host numpy float32 arrays (copied host->device) or CUDA tensors (device->device).
        `moving_initial`: a LinearTransform or a list of them (first applied first), the
        antsRegistration -r initial moving transform; it is folded into the moving geometry."""
        if moving_initial is not None:
            moving_geom = fold_moving_geometry(moving_geom, moving_initial)
        gf, gm = fixed_geom.to_c(), moving_geom.to_c()
        if isinstance(fixed, np.ndarray):
            f = _host(fixed, fixed_geom.count, "fixed")
            m = _host(moving, moving_geom.count, "moving")
            self._keep = (f, m)
            self._ck(self.lib.synx_set_images(self.h, _ptr(f), C.byref(gf), _ptr(m), C.byref(gm)))
        else:
            self._ck(self.lib.synx_set_images_device(self.h, _dev(fixed, fixed_geom.count, "fixed"), C.byref(gf),
                                                     _dev(moving, moving_geom.count, "moving"), C.byref(gm)))

    def run(self) -> None:
        self._ck(self.lib.synx_run(self.h))

    def run_level(self, level: int) -> None:
        self._ck(self.lib.synx_run_level(self.h, level))

    def output_geom(self) -> Geom:
        g = SynxGeom()
        self._ck(self.lib.synx_get_output_geom(self.h, C.byref(g)))
        return Geom.from_c(g)

    def fields(self, fwd: np.ndarray | None = None, inv: np.ndarray | None = None) -> tuple[np.ndarray, np.ndarray]:
        """Forward and inverse fields, interleaved: shape grid.shape + (dim,) (optionally into
        caller-provided, e.g. pinned, host arrays)."""
        g = self.output_geom()
        shp = g.shape + (g.dim,)
        if fwd is None:
            fwd = np.empty(shp, np.float32)
        if inv is None:
            inv = np.empty(shp, np.float32)
        assert fwd.shape == shp and inv.shape == shp and fwd.dtype == np.float32 and inv.dtype == np.float32
        self._ck(self.lib.synx_get_fields(self.h, _ptr(fwd), _ptr(inv)))
        return fwd, inv

    def fields_device(self, fwd, inv) -> None:
        g = self.output_geom()
        n = g.dim * g.count
        self._ck(self.lib.synx_get_fields_device(self.h, _dev(fwd, n, "fwd"), _dev(inv, n, "inv")))

    def half_fields(self) -> tuple:
        g = self.output_geom()
        shp = g.shape + (g.dim,)
        out = [np.empty(shp, np.float32) for _ in range(4)]
        self._ck(self.lib.synx_get_half_fields(self.h, *[_ptr(a) for a in out]))
        return tuple(out)

    def set_half_fields(self, phi_f, psi_f, phi_m, psi_m, grid: Geom) -> None:
        arrs = [_host(a, grid.dim * grid.count, "half field") for a in (phi_f, psi_f, phi_m, psi_m)]
        g = grid.to_c()
        self._ck(self.lib.synx_set_half_fields(self.h, *[_ptr(a) for a in arrs], C.byref(g)))

    def set_initial_half_fields(self, phi_f=None, psi_f=None, phi_m=None, psi_m=None, grid: Geom | None = None) -> None:
        """The stage's starting half-fields (interleaved host arrays on `grid`, as half_fields()
        returns them), resampled to the first level's grid instead of zero fields: a stage resumed
        from a saved registration state.  All None clears them."""
        if phi_f is None and psi_f is None and phi_m is None and psi_m is None:
            self._ck(self.lib.synx_set_initial_half_fields(self.h, None, None, None, None, None))
            return
        if grid is None:
            raise SynxError("initial half-fields need their grid")
        arrs = [_host(a, grid.dim * grid.count, "initial half field") for a in (phi_f, psi_f, phi_m, psi_m)]
        g = grid.to_c()
        self._ck(self.lib.synx_set_initial_half_fields(self.h, *[_ptr(a) for a in arrs], C.byref(g)))

    def log(self) -> list[LogRecord]:
        n = C.c_int64()
        self._ck(self.lib.synx_get_log(self.h, None, None, None, None, None, 0, C.byref(n)))
        k = n.value
        lv = np.zeros(k, np.int32)
        it = np.zeros(k, np.int32)
        me = np.zeros(k, np.float64)
        cv = np.zeros(k, np.float64)
        ii = np.zeros(k, np.int32)
        if k:
            self._ck(self.lib.synx_get_log(self.h, _ptr(lv), _ptr(it), _ptr(me), _ptr(cv), _ptr(ii), k, C.byref(n)))
        return [LogRecord(int(lv[i]), int(it[i]), float(me[i]), float(cv[i]), int(ii[i])) for i in range(k)]

    def profile(self) -> dict:
        a, b, c_, d, e, f = C.c_double(), C.c_int64(), C.c_int64(), C.c_double(), C.c_int64(), C.c_int64()
        self._ck(self.lib.synx_get_profile(self.h, C.byref(a), C.byref(b), C.byref(c_), C.byref(d), C.byref(e),
                                           C.byref(f)))
        return {"inverse_ms": a.value, "inverse_launches": b.value, "inverse_voxels": c_.value, "cc_ms": d.value,
                "cc_launches": e.value, "cc_voxels": f.value}

    def level_plan(self, level: int) -> dict:
        """The tile plan `level` runs with: persistent level kernel or not, smoothing tile rows (-1:
        xy and z kernels), CC z chunks (0: cost model)."""
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        self._ck(self.lib.synx_level_plan(self.h, level, C.byref(a), C.byref(b), C.byref(c)))
        return {"persistent": a.value, "smooth_rows": b.value, "cc_z_chunks": c.value}

    def reset_profile(self) -> None:
        self._ck(self.lib.synx_reset_profile(self.h))

    def level_profile(self) -> list[dict]:
        out = []
        for lv in range(len(self.params.iterations)):
            d = [C.c_double() for _ in range(4)]
            n = [C.c_int64() for _ in range(3)]
            self._ck(self.lib.synx_get_level_profile(self.h, lv, *[C.byref(x) for x in d], *[C.byref(x) for x in n]))
            out.append({"level": lv, "setup_ms": d[0].value, "iterate_ms": d[1].value, "inverse_ms": d[2].value,
                        "cc_ms": d[3].value, "iterations": n[0].value, "inverse_subiterations": n[1].value,
                        "voxels": n[2].value})
        return out

    def device_bytes(self) -> int:
        n = C.c_int64()
        self._ck(self.lib.synx_get_device_bytes(self.h, C.byref(n)))
        return n.value


def launch_count() -> int:
    """Kernel launches issued by libsynx in this process so far."""
    n = C.c_int64()
    _check(load_library().synx_get_launch_count(C.byref(n)))
    return n.value


# ---- step entry points (device tensors, component-plane fields) --------------------------------
def gaussian_kernel(variance: float, max_error: float, max_width: int) -> np.ndarray:
    lib = load_library()
    n = C.c_int()
    _check(lib.synx_gaussian_kernel(variance, max_error, max_width, None, 0, C.byref(n)))
    out = np.zeros(n.value, np.float64)
    _check(lib.synx_gaussian_kernel(variance, max_error, max_width, _ptr(out), n.value, C.byref(n)))
    return out


def tuning_load(path: str | None = None) -> int:
    """(Re)load the tile-plan table; None reloads the default ($SYNX_TUNING_TABLE or
    tuning_b200.txt beside libsynx.so).  Returns the number of entries."""
    n = load_library().synx_tuning_load(path.encode() if path else None)
    if n < 0:
        _check(n)
    return n


def tuning_path() -> str:
    return load_library().synx_tuning_path().decode()


def shrink_geom(g: Geom, factor: int) -> Geom:
    lib = load_library()
    o = SynxGeom()
    gi = g.to_c()
    _check(lib.synx_shrink_geom(C.byref(gi), factor, C.byref(o)))
    return Geom.from_c(o)


def _stream(stream) -> C.c_void_p:
    return C.c_void_p(stream or 0)


def smooth_image(img, out, g: Geom, sigma: float, sigma_in_mm: bool = False, stream=None) -> None:
    gc = g.to_c()
    _check(load_library().synx_smooth_image(_dev(img, g.count, "img"), _dev(out, g.count, "out"), C.byref(gc),
                                            sigma, int(sigma_in_mm),
                                            _stream(stream)))


def warp_image(img, img_geom: Geom, u, grid: Geom, out, stream=None, nearest: bool = False,
               label: bool = False) -> None:
    """out(x) = img(x + u(x)) on `grid`, 0 outside: linear, nearest-neighbour (nearest=True) or
    generic label interpolation over the linear interpolator (label=True)."""
    a, b = img_geom.to_c(), grid.to_c()
    lib = load_library()
    fn = lib.synx_warp_image_label if label else lib.synx_warp_image_nearest if nearest else lib.synx_warp_image
    _check(fn(_dev(img, img_geom.count, "img"), C.byref(a), _dev(u, grid.dim * grid.count, "u"), C.byref(b),
              _dev(out, grid.count, "out"), _stream(stream)))


def histogram_match(src, ref, out, levels: int = 256, match_points: int = 12, threshold_at_mean: bool = True,
                    stream=None) -> None:
    """out = src with its histogram matched to ref's (device float tensors; out may be src).  The
    defaults are those antsRegistration's --use-histogram-matching 1 runs with."""
    n = int(src.numel())
    _check(load_library().synx_histogram_match(_dev(src, n, "src"), n, _dev(ref, 1, "ref"), int(ref.numel()), levels,
                                               match_points, int(threshold_at_mean), _dev(out, n, "out"),
                                               _stream(stream)))


def cc_metric(F, M, g: Geom, radius: int, gF, gM, stream=None, fp32_sums: bool = False) -> float:
    """CC value and both update directions; fp32_sums selects float window sums (precision study)."""
    gc = g.to_c()
    v = C.c_double()
    flags = SYNX_F_CC_FP32_SUMS if fp32_sums else 0
    n = g.count
    _check(load_library().synx_cc_metric_ex(_dev(F, n, "F"), _dev(M, n, "M"), C.byref(gc), radius, flags,
                                            _dev(gF, g.dim * n, "gF"), _dev(gM, g.dim * n, "gM"),
                                            C.byref(v), _stream(stream)))
    return v.value


def cc_metric_masked(F, M, valid, g: Geom, radius: int, gF, gM, stream=None) -> float:
    """CC over the valid voxels only; `valid` is a contiguous uint8 CUDA tensor (nonzero = valid)."""
    if isinstance(valid, np.ndarray) or not getattr(valid, "is_cuda", False):
        raise SynxError("valid: a CUDA tensor is required")
    if str(valid.dtype) != "torch.uint8" or not valid.is_contiguous() or valid.numel() < g.count:
        raise SynxError("valid: a contiguous uint8 tensor with one byte per voxel is required")
    gc = g.to_c()
    v = C.c_double()
    n = g.count
    _check(load_library().synx_cc_metric_masked(_dev(F, n, "F"), _dev(M, n, "M"), valid.data_ptr(), C.byref(gc),
                                                radius, _dev(gF, g.dim * n, "gF"), _dev(gM, g.dim * n, "gM"),
                                                C.byref(v), _stream(stream)))
    return v.value


def cc_metric_noalloc(F, M, g: Geom, radius: int, gF, gM, stream=None, read_value: bool = True):
    """cc_metric without any device allocation: the kernel's scratch is a fixed device array
    inside libsynx (for callers that cannot allocate, e.g. inside graph capture).  Calls on one
    device share that array, so calls that overlap on the GPU race.  With read_value=False the call
    does not wait for its stream and returns None (the form a stream capture takes)."""
    lib = load_library()
    gc = g.to_c()
    v = C.c_double()
    n = g.count
    rc = lib.synx_cc_metric_noalloc(_dev(F, n, "F"), _dev(M, n, "M"), C.byref(gc), radius, _dev(gF, g.dim * n, "gF"),
                                    _dev(gM, g.dim * n, "gM"), C.byref(v) if read_value else None,
                                    _stream(stream))
    if rc != 0:
        raise SynxError(f"synx error {rc} ({ERRORS.get(rc, '?')}): {lib.synx_noalloc_last_error().decode()}")
    return v.value if read_value else None


def smooth_field(u, out, g: Geom, variance: float, stream=None) -> float:
    gc = g.to_c()
    mx = C.c_double()
    n = g.dim * g.count
    _check(load_library().synx_smooth_field(_dev(u, n, "u"), _dev(out, n, "out"), C.byref(gc), variance, C.byref(mx),
                                            _stream(stream)))
    return mx.value


def compose(d, w, g: Geom, out, scale: float = 1.0, stream=None) -> None:
    gc = g.to_c()
    n = g.dim * g.count
    _check(load_library().synx_compose(_dev(d, n, "d"), _dev(w, n, "w"), C.byref(gc), scale, _dev(out, n, "out"),
                                       _stream(stream)))


def invert_field(phi, psi, g: Geom, max_iter=20, mean_tol=0.001, max_tol=0.1, stream=None) -> int:
    gc = g.to_c()
    it = C.c_int()
    n = g.dim * g.count
    _check(load_library().synx_invert_field(_dev(phi, n, "phi"), _dev(psi, n, "psi"), C.byref(gc), max_iter, mean_tol,
                                            max_tol,
                                            C.byref(it), _stream(stream)))
    return it.value


def resample_field(u, gi: Geom, out, go: Geom, stream=None) -> None:
    a, b = gi.to_c(), go.to_c()
    _check(load_library().synx_resample_field(_dev(u, gi.dim * gi.count, "u"), C.byref(a),
                                              _dev(out, go.dim * go.count, "out"), C.byref(b), _stream(stream)))


@dataclass
class LinearTransform:
    """A linear transform of an ITK transform file: T(p) = matrix (p - center) + translation + center."""

    matrix: np.ndarray  # (dim, dim)
    translation: np.ndarray  # (dim,)
    center: np.ndarray  # (dim,)

    @property
    def dim(self) -> int:
        return self.matrix.shape[0]

    def to_c(self) -> SynxLinear:
        t = SynxLinear()
        d = self.dim
        t.dim = d
        t.has_center = 1
        m = np.eye(3)
        m[:d, :d] = self.matrix
        for k in range(9):
            t.matrix[k] = float(m.flat[k])
        for k in range(d):
            t.translation[k] = float(self.translation[k])
            t.center[k] = float(self.center[k])
        return t


def fold_moving_geometry(g: Geom, transforms) -> Geom:
    """The moving image's geometry with initial linear transforms folded in: voxel i is placed at
    Init^-1(p_i), so sampling the result at q reads the image at Init(q).  `transforms` is one
    LinearTransform or a list applied first to last (Init = T_n o ... o T_1), the composite ITK's SyN
    samples the moving image through (Init(x + psi_M(x)))."""
    if isinstance(transforms, LinearTransform):
        transforms = [transforms]
    d = g.dim
    M, b = np.eye(d), np.zeros(d)
    for t in transforms:
        A = np.asarray(t.matrix, float)
        tb = np.asarray(t.translation, float) + np.asarray(t.center, float) - A @ np.asarray(t.center, float)
        M, b = A @ M, A @ b + tb
    Mi = np.linalg.inv(M)
    return Geom(g.size, g.spacing, tuple(Mi @ np.asarray(g.origin) - Mi @ b), Mi @ g.direction)


def count_linear_transforms(path, dim: int) -> int:
    """Number of linear transforms in an ITK transform file (.mat or .txt)."""
    rc = load_library().synx_read_linear_transform(os.fsencode(str(path)), dim, 0, None)
    if rc < 0:
        _check(rc)
    return rc


def read_linear_transform(path, dim: int, index: int = 0) -> LinearTransform:
    """Transform `index` of an ITK transform file (.mat MATLAB v4 or .txt Insight text)."""
    t = SynxLinear()
    rc = load_library().synx_read_linear_transform(os.fsencode(str(path)), dim, index, C.byref(t))
    if rc < 0:
        _check(rc)
    m = np.array(list(t.matrix), dtype=np.float64).reshape(3, 3)[:dim, :dim]
    return LinearTransform(m, np.array(list(t.translation)[:dim]), np.array(list(t.center)[:dim]))


def linear_from_parameters(type_name: str, params, fixed, dim: int) -> LinearTransform:
    """A linear transform from its ITK type name, parameters and fixed parameters (the entries of
    a transform file), in matrix-offset form."""
    p = np.ascontiguousarray(params, dtype=np.float64).reshape(-1)
    f = np.ascontiguousarray(fixed, dtype=np.float64).reshape(-1)
    t = SynxLinear()
    dp = C.POINTER(C.c_double)
    _check(load_library().synx_linear_from_parameters(type_name.encode(), p.ctypes.data_as(dp), p.size,
                                                      f.ctypes.data_as(dp), f.size, dim, C.byref(t)))
    m = np.array(list(t.matrix), dtype=np.float64).reshape(3, 3)[:dim, :dim]
    return LinearTransform(m, np.array(list(t.translation)[:dim]), np.array(list(t.center)[:dim]))


def initial_translation(fixed, gf: Geom, moving, gm: Geom, feature: int) -> LinearTransform:
    """The translation antsRegistration derives for -r [fixed,moving,feature]: 0 geometric centers,
    1 centers of intensity mass, 2 origins (center = the fixed image's feature point)."""
    a, b = gf.to_c(), gm.to_c()
    F = None if fixed is None else np.ascontiguousarray(fixed, dtype=np.float32)
    M = None if moving is None else np.ascontiguousarray(moving, dtype=np.float32)
    t = SynxLinear()
    _check(load_library().synx_initial_translation(None if F is None else _ptr(F), C.byref(a),
                                                   None if M is None else _ptr(M), C.byref(b), feature, C.byref(t)))
    d = gf.dim
    return LinearTransform(np.eye(d), np.array(list(t.translation)[:d]), np.array(list(t.center)[:d]))


def write_linear_transform(path, t: LinearTransform) -> None:
    """Write `t` as an ITK AffineTransform file (.mat MATLAB v4, as antsRegistration writes
    prefix0GenericAffine.mat, or .txt Insight text)."""
    tc = t.to_c()
    _check(load_library().synx_write_linear_transform(os.fsencode(str(path)), C.byref(tc)))


def linear_field(t: LinearTransform, g: Geom, invert: bool = False) -> np.ndarray:
    """Displacement T(p) - p (or T^-1(p) - p) at every voxel of `g`, as component planes (the
    layout of the step functions): shape (dim,) + g.shape."""
    out = np.empty((g.dim,) + g.shape, dtype=np.float32)
    tc, gc = t.to_c(), g.to_c()
    _check(load_library().synx_linear_field(C.byref(tc), int(bool(invert)), C.byref(gc), _ptr(out)))
    return out
