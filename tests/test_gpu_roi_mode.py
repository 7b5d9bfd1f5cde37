"""ROI mode of the host-buffer calls: when the candidates' ROIs are a small
part of the frames, loc_fit_host and loc_fit_host_async copy the candidates'
ROIs, packed each at its own size, instead of the frames. The rows and flags must be those of the
whole-frame upload (host_roi_mode = -1) and of the device-pointer call, bit
for bit, including the candidates the input and edge rules reject before any
pixel is read, mixed ROI half-widths, and a caller's half-width cap."""
import numpy as np
import pytest

import localizer_b200 as L
from localizer_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    e = L.Engine(0)
    yield e
    e.close()


def _stack(name, n_frames, seed):
    w = synth.scaled(synth.workloads()[name], n_frames, seed)
    frames, _ = synth.make(w)
    cands = L.find_candidates(frames, 30.0, w.w0)
    rng = np.random.default_rng(seed + 17)
    cands["half_width"] = rng.choice(np.array(w.half_widths), size=len(cands))
    return w, frames, cands


def _with_rejects(cands, frames):
    """Append candidates that the input and edge rules reject."""
    n_frames, n_cols, n_rows = frames.shape
    extra = np.zeros(7, dtype=L.CANDIDATE_DTYPE)
    extra["x"] = [1.5, n_rows - 2.0, np.nan, 40.0, 40.0, 40.0, 40.25]
    extra["y"] = [40.0, 40.0, 40.0, 1.2, 40.0, 40.0, 40.75]
    extra["intensity"] = 300.0
    extra["background"] = 100.0
    extra["frame"] = [0, 0, 0, 0, n_frames, -1, 0]
    extra["half_width"] = [4, 4, 0, 5, 0, 0, 17]
    return np.concatenate([cands, extra])


@pytest.mark.parametrize("name,method", [("stress", 0), ("uneven", 7), ("uneven", 5), ("small", 1)])
def test_roi_mode_rows_match_frame_upload(engine, name, method):
    w, frames, cands = _stack(name, 24, 700)
    cands = _with_rejects(cands, frames)
    h0, _ = engine.host_bytes()
    rows_f, flags_f = engine.fit_host(frames, cands, method, w.w0, options=L.default_options(host_roi_mode=-1))
    h1, _ = engine.host_bytes()
    rows_r, flags_r = engine.fit_host(frames, cands, method, w.w0, options=L.default_options(host_roi_mode=1))
    h2, _ = engine.host_bytes()
    np.testing.assert_array_equal(flags_r, flags_f)
    np.testing.assert_array_equal(rows_r, rows_f)
    assert h1 - h0 >= frames.nbytes
    assert h2 - h1 < frames.nbytes + cands.nbytes + 4 * len(cands)   # ROI mode was taken
    # the packed stack holds exactly the (2r+1)^2 pixels of each candidate that reads pixels
    r = np.where(cands["half_width"] > 0, cands["half_width"], int(np.ceil(4 * w.w0)))
    reads = (flags_r != 1) & (flags_r != 10)
    assert h2 - h1 == 2 * int(((2 * r[reads] + 1) ** 2).sum()) + cands.nbytes + 4 * len(cands)
    # the rejects: edge (2), bad input (NaN, frame range, half-width above the cap)
    assert list(flags_r[-7:]) == [1, 1, 10, 1, 10, 10, 10]


def test_roi_mode_with_half_width_cap_and_device_call(engine):
    import torch
    w, frames, cands = _stack("uneven", 16, 710)
    # a cap below some candidates' half-width: those are bad input in both modes
    opts = L.default_options(max_half_width=5)
    rows_r, flags_r = engine.fit_host(frames, cands, 7, w.w0, options=L.default_options(max_half_width=5,
                                                                                         host_roi_mode=1))
    rows_f, flags_f = engine.fit_host(frames, cands, 7, w.w0, options=L.default_options(max_half_width=5,
                                                                                         host_roi_mode=-1))
    np.testing.assert_array_equal(flags_r, flags_f)
    np.testing.assert_array_equal(rows_r, rows_f)
    assert np.all(flags_r[cands["half_width"] > 5] == 10)
    d_frames = torch.from_numpy(frames.view(np.int16)).cuda()
    d_cands = torch.from_numpy(cands.view(np.uint8)).cuda()
    n, ncol = len(cands), L.lib().loc_output_columns(7)
    d_out = torch.empty((n, ncol), dtype=torch.float64, device="cuda")
    d_flags = torch.empty(n, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    engine.fit_device(d_frames.data_ptr(), frames.shape[0], frames.shape[2], frames.shape[1], d_cands.data_ptr(), n,
                      7, w.w0, 1.0, d_out.data_ptr(), d_flags.data_ptr(), stream, opts)
    engine.sync(stream)
    np.testing.assert_array_equal(d_flags.cpu().numpy(), flags_r)
    np.testing.assert_array_equal(d_out.cpu().numpy(), rows_r)


def test_roi_mode_async_stream_of_stacks(engine):
    """ROI-mode and whole-frame async calls interleaved over stacks of
    different sizes (staging buffers reused and grown while calls are in
    flight) give the synchronous whole-frame rows."""
    jobs = []
    for name, nf, method, mode in (("stress", 20, 0, 1), ("uneven", 8, 7, 1), ("uneven", 30, 7, -1),
                                   ("stress", 40, 0, 1), ("uneven", 12, 5, 0), ("stress", 20, 0, 1)):
        w, frames, cands = _stack(name, nf, 720 + nf)
        jobs.append((w, frames, cands, method, mode))
    expect = [engine.fit_host(fr, c, m, w.w0, options=L.default_options(host_roi_mode=-1))
              for w, fr, c, m, _ in jobs]
    outs = []
    for w, frames, cands, method, mode in jobs:
        n, ncol = len(cands), L.lib().loc_output_columns(method)
        out, flags = np.full((n, ncol), -7.0), np.full(n, 99, dtype=np.uint8)
        engine.fit_host_async(frames, cands, method, w.w0, 1.0, out, flags,
                              options=L.default_options(host_roi_mode=mode))
        outs.append((out, flags))
    engine.wait()
    for (rows, flags), (out, fl) in zip(expect, outs):
        np.testing.assert_array_equal(fl, flags)
        np.testing.assert_array_equal(out, rows)


def test_dense_candidates_fall_back_to_frames(engine):
    """Candidates whose ROIs cover the frames several times over: the whole
    frames are copied even when ROI mode is asked for (the ROI stack would be
    larger)."""
    w, frames, _ = _stack("small", 4, 730)
    n_frames, n_cols, n_rows = frames.shape
    ys, xs = np.meshgrid(np.arange(8, n_cols - 8, 2), np.arange(8, n_rows - 8, 2), indexing="ij")
    per = xs.size
    c = np.zeros(per * n_frames, dtype=L.CANDIDATE_DTYPE)
    c["x"] = np.tile(xs.ravel() + 0.3, n_frames)
    c["y"] = np.tile(ys.ravel() + 0.6, n_frames)
    c["intensity"] = 200.0
    c["background"] = 100.0
    c["frame"] = np.repeat(np.arange(n_frames), per)
    h0, _ = engine.host_bytes()
    rows_r, flags_r = engine.fit_host(frames, c, 0, w.w0, options=L.default_options(host_roi_mode=1))
    h1, _ = engine.host_bytes()
    rows_f, flags_f = engine.fit_host(frames, c, 0, w.w0, options=L.default_options(host_roi_mode=-1))
    assert h1 - h0 >= frames.nbytes
    np.testing.assert_array_equal(flags_r, flags_f)
    np.testing.assert_array_equal(rows_r, rows_f)
