"""loc_fit_batch_static, the allocation-free form of the batched fit.

It serves callers that may not allocate device memory (a framework whose
caching allocator owns the device heap, a plugin handed only its input and
output buffers, an acquisition loop that must not cudaMalloc between
frames): its scratch is one file-scope device array shared by all calls.
These checks call it through the C ABI twice in a row, on different inputs,
and compare each result with loc_fit_batch's on the same inputs; then they
check that an oversized batch is refused before any device work. This file
is collected last so that a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

import localizer_b200 as L
from tests import _golden as G

pytestmark = pytest.mark.gpu

# both entry points run the same kernels on the same inputs: rows agree to
# this tolerance (they are in fact expected to be identical)
RTOL = 1e-12
ATOL = 1e-12


def _inputs(name):
    import torch
    g = G.load(name)
    frames, cands = g["frames"], g["cands"]
    d_frames = torch.from_numpy(frames.view(np.int16)).cuda()
    d_cands = torch.from_numpy(np.ascontiguousarray(cands).view(np.uint8)).cuda()
    return g, frames, cands, d_frames, d_cands


def _outputs(n, method):
    import torch
    ncol = L.lib().loc_output_columns(method)
    return (torch.full((n, ncol), -7.0, dtype=torch.float64, device="cuda"),
            torch.full((n,), 77, dtype=torch.uint8, device="cuda"))


def test_static_entry_matches_batched_fit_twice():
    import torch
    lib = L.lib()
    eng = L.Engine(0)
    stream = torch.cuda.current_stream().cuda_stream
    try:
        for name, method in (("uneven", 7), ("small", 0)):
            g, frames, cands, d_frames, d_cands = _inputs(name)
            n = len(cands)
            n_frames, n_cols, n_rows = frames.shape
            ref_out, ref_flags = _outputs(n, method)
            eng.fit_device(d_frames.data_ptr(), n_frames, n_rows, n_cols, d_cands.data_ptr(), n, method, g["w0"],
                           1.0, ref_out.data_ptr(), ref_flags.data_ptr(), stream)
            eng.sync(stream)
            out, flags = _outputs(n, method)
            opts = L.default_options()
            rc = lib.loc_fit_batch_static(C.c_void_p(d_frames.data_ptr()), n_frames, n_rows, n_cols,
                                          C.c_void_p(d_cands.data_ptr()), n, method, g["w0"], 1.0, C.byref(opts),
                                          C.c_void_p(out.data_ptr()), C.c_void_p(flags.data_ptr()),
                                          C.c_void_p(stream))
            assert rc == 0, lib.loc_last_error()
            torch.cuda.synchronize()
            np.testing.assert_array_equal(flags.cpu().numpy(), ref_flags.cpu().numpy())
            np.testing.assert_allclose(out.cpu().numpy(), ref_out.cpu().numpy(), rtol=RTOL, atol=ATOL,
                                       equal_nan=True)
            assert np.sum(flags.cpu().numpy() == 0) > 0.5 * n
    finally:
        eng.close()


def test_static_entry_allocates_no_device_memory():
    """After the first call on the device (which resolves the array's
    address), a call leaves the device's free memory unchanged: its scratch
    is the static array, not an allocation. No context is alive here."""
    import torch
    lib = L.lib()
    g, frames, cands, d_frames, d_cands = _inputs("uneven")
    n = len(cands)
    n_frames, n_cols, n_rows = frames.shape
    out, flags = _outputs(n, 7)
    stream = torch.cuda.current_stream().cuda_stream

    def call():
        rc = lib.loc_fit_batch_static(C.c_void_p(d_frames.data_ptr()), n_frames, n_rows, n_cols,
                                      C.c_void_p(d_cands.data_ptr()), n, 7, g["w0"], 1.0, None,
                                      C.c_void_p(out.data_ptr()), C.c_void_p(flags.data_ptr()), C.c_void_p(stream))
        assert rc == 0, lib.loc_last_error()
        torch.cuda.synchronize()

    call()
    free0 = torch.cuda.mem_get_info()[0]
    call()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, (free0, free1)
    assert np.sum(flags.cpu().numpy() == 0) > 0.5 * n


def test_static_entry_refuses_unsupported_modes():
    lib = L.lib()
    rc = lib.loc_fit_batch_static(None, 1, 64, 64, None, 0, 6, 1.3, 1.0, None, None, None, None)
    assert rc == -4


def test_static_entry_refuses_oversized_batch():
    lib = L.lib()
    rc = lib.loc_fit_batch_static(None, 1, 64, 64, None, 16385, 0, 1.3, 1.0, None, None, None, None)
    assert rc == -4
    assert b"16384" in lib.loc_last_error()
