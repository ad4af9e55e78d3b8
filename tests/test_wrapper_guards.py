"""The Python wrappers refuse, before any call into the library, a buffer that would reach a kernel
as a host pointer, in the wrong type or layout, or shorter than its geometry needs (CPU only).

A stand-in object that looks like a CUDA tensor to the checks carries the type, layout and size
cases; every case here fails a check, so no pointer of it reaches the library."""
import numpy as np
import pytest
import torch

from ants_b200 import synx
from ants_b200.synx import Geom, SynxError

G = Geom((8, 6, 4))
N = G.count


class FakeCuda:
    is_cuda = True

    def __init__(self, n, dtype="torch.float32", contiguous=True):
        self.n, self.dtype, self.contiguous = n, dtype, contiguous

    def is_contiguous(self):
        return self.contiguous

    def numel(self):
        return self.n

    def data_ptr(self):
        return 0x1000


def ok(n):
    return FakeCuda(n)


@pytest.mark.parametrize("bad,needle", [
    (np.zeros(N, np.float32), "CUDA tensor"),
    (torch.zeros(N), "CUDA tensor"),
    (FakeCuda(N, dtype="torch.float64"), "float32"),
    (FakeCuda(N, contiguous=False), "contiguous"),
    (FakeCuda(N - 1), "geometry needs"),
])
def test_image_operand_checks(bad, needle):
    synx.load_library()
    with pytest.raises(SynxError, match=needle):
        synx.smooth_image(bad, ok(N), G, 1.0)


@pytest.mark.parametrize("call", [
    lambda: synx.smooth_image(ok(N), ok(N - 1), G, 1.0),
    lambda: synx.warp_image(ok(N), G, ok(3 * N - 1), G, ok(N)),
    lambda: synx.warp_image(ok(N), G, ok(3 * N), G, ok(N - 1), label=True),
    lambda: synx.cc_metric(ok(N), ok(N), G, 2, ok(3 * N), ok(3 * N - 1)),
    lambda: synx.cc_metric_noalloc(ok(N), ok(N - 1), G, 2, ok(3 * N), ok(3 * N)),
    lambda: synx.smooth_field(ok(3 * N), ok(3 * N - 1), G, 3.0),
    lambda: synx.compose(ok(3 * N), ok(3 * N - 1), G, ok(3 * N)),
    lambda: synx.invert_field(ok(3 * N - 1), ok(3 * N), G),
    lambda: synx.resample_field(ok(3 * N), G, ok(3 * Geom((16, 12, 8)).count - 1), Geom((16, 12, 8))),
    lambda: synx.histogram_match(ok(N), ok(N), ok(N - 1)),
    lambda: synx.histogram_match(ok(N), torch.zeros(N), ok(N)),
])
def test_every_device_operator_checks_its_buffers(call):
    synx.load_library()
    with pytest.raises(SynxError):
        call()


def test_host_arrays_must_match_the_geometry():
    assert synx._host(np.zeros((4, 6, 8)), N, "x").dtype == np.float32
    with pytest.raises(SynxError, match="geometry needs"):
        synx._host(np.zeros(N + 1, np.float32), N, "x")
