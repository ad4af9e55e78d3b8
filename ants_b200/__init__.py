"""synx: B200-native SyN + neighbourhood-CC registration stage (antsRegistration drop-in).

The compute path is libsynx.so (hand-written sm_100a CUDA behind the C ABI in include/synx.h);
this package is its Python mirror.
"""
from .synx import (  # noqa: F401
    Geom,
    LogRecord,
    SyNParams,
    SyNStage,
    SynxError,
    cc_metric,
    compose,
    gaussian_kernel,
    invert_field,
    load_library,
    resample_field,
    shrink_geom,
    smooth_field,
    smooth_image,
    warp_image,
)

__all__ = [
    "Geom", "LogRecord", "SyNParams", "SyNStage", "SynxError", "cc_metric", "compose", "gaussian_kernel",
    "invert_field", "load_library", "resample_field", "shrink_geom", "smooth_field", "smooth_image", "warp_image",
]
