"""The allocation-free CC entry point (synx_cc_metric_noalloc).

It serves callers that must not allocate device memory themselves: a plug-in whose host
application (a viewer, a deep-learning framework with its own caching allocator, a serving process)
owns the GPU's memory and its budget, or a latency-bound loop that cannot afford the device-wide
synchronisation a cudaMalloc/cudaFree pair can cause.  It keeps the CC kernel's scratch in a fixed
array inside libsynx instead.  The GPU tests call it twice in a row through the C ABI, and inside a
CUDA graph capture replayed on new inputs, and check each result against synx_cc_metric on the same
inputs, with the tolerances of the CC parity tests.  The
file name sorts after every other test file, so pytest collects it last and a run which stops at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from ants_b200 import synx
from ants_b200.synx import Geom


def test_noalloc_rejects_grids_beyond_its_scratch():
    # 8192 x 1040 voxels per slice needs more CC blocks than the fixed scratch holds; the check runs
    # on the host before any device work, so this needs no GPU
    lib = synx.load_library()
    g = Geom((8192, 1040, 1)).to_c()
    v = C.c_double()
    dummy = C.c_void_p(256)
    rc = lib.synx_cc_metric_noalloc(dummy, dummy, C.byref(g), 2, dummy, dummy, C.byref(v), None)
    assert rc == -1
    msg = lib.synx_noalloc_last_error().decode()
    assert "at most 32768" in msg


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_twice(cuda):
    import torch

    cases = [
        (Geom((37, 29, 23), (1.0, 1.2, 0.9)), 4, 11),
        (Geom((61, 47), (1.0, 1.0)), 2, 12),
    ]
    for g, radius, seed in cases:
        rng = np.random.default_rng(seed)
        F = rng.uniform(0, 1, g.shape).astype(np.float32)
        M = (0.6 * np.roll(F, 1, axis=-1) + 0.1 * rng.standard_normal(g.shape)).astype(np.float32)
        Fd = torch.from_numpy(F).to(cuda)
        Md = torch.from_numpy(M).to(cuda)
        shape = (g.dim,) + g.shape
        ref_f = torch.empty(shape, device=cuda)
        ref_m = torch.empty(shape, device=cuda)
        v_ref = synx.cc_metric(Fd, Md, g, radius, ref_f, ref_m)
        for _ in range(2):  # the second call reuses the scratch left by the first
            out_f = torch.full(shape, float("nan"), device=cuda)
            out_m = torch.full(shape, float("nan"), device=cuda)
            v = synx.cc_metric_noalloc(Fd, Md, g, radius, out_f, out_m)
            torch.cuda.synchronize()
            assert abs(v - v_ref) < 1e-9
            for a, b in ((out_f, ref_f), (out_m, ref_m)):
                a, b = a.cpu().numpy(), b.cpu().numpy()
                scale = max(np.abs(b).max(), 1e-20)
                np.testing.assert_allclose(a, b, atol=1e-6 * scale, rtol=1e-5)


@pytest.mark.gpu
def test_noalloc_inside_graph_capture(cuda):
    # captured into a CUDA graph (value not read), each replay recomputes both gradients from the
    # inputs' current contents; a call that asks for the value while the stream captures is refused
    # before it touches the stream, and the capture goes on
    import torch

    g = Geom((37, 29, 23), (1.0, 1.2, 0.9))
    radius = 3
    rng = np.random.default_rng(13)

    def pair():
        F = rng.uniform(0, 1, g.shape).astype(np.float32)
        M = (0.6 * np.roll(F, 1, axis=-1) + 0.1 * rng.standard_normal(g.shape)).astype(np.float32)
        return torch.from_numpy(F).to(cuda), torch.from_numpy(M).to(cuda)

    Fd, Md = pair()
    shape = (g.dim,) + g.shape
    out_f = torch.empty(shape, device=cuda)
    out_m = torch.empty(shape, device=cuda)
    synx.cc_metric_noalloc(Fd, Md, g, radius, out_f, out_m)  # first call on the device: before any capture
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        s = torch.cuda.current_stream().cuda_stream
        with pytest.raises(synx.SynxError, match="must be NULL while the stream is being captured"):
            synx.cc_metric_noalloc(Fd, Md, g, radius, out_f, out_m, stream=s)
        assert synx.cc_metric_noalloc(Fd, Md, g, radius, out_f, out_m, stream=s, read_value=False) is None
    ref_f = torch.empty(shape, device=cuda)
    ref_m = torch.empty(shape, device=cuda)
    for _ in range(2):
        F2, M2 = pair()
        Fd.copy_(F2)
        Md.copy_(M2)
        out_f.fill_(float("nan"))
        out_m.fill_(float("nan"))
        graph.replay()
        synx.cc_metric(Fd, Md, g, radius, ref_f, ref_m)
        torch.cuda.synchronize()
        for a, b in ((out_f, ref_f), (out_m, ref_m)):
            a, b = a.cpu().numpy(), b.cpu().numpy()
            scale = max(np.abs(b).max(), 1e-20)
            np.testing.assert_allclose(a, b, atol=1e-6 * scale, rtol=1e-5)
    del graph
