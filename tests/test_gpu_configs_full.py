"""The small (512 frames of 128 x 128, method 0), precision-stress (5,000
frames of 256 x 256, method 0) and batched-uneven (10,000 frames of
256 x 256, method 7) workloads at their full sizes, every candidate fitted
three ways: the FP32 path (product default), the all-FP64 GPU path, and the
reference's own fitter classes (FP64, compiled from its sources, one call per
frame and ROI half-width as its workers make them, on all host threads).

Gates on every candidate: flag agreement >= 99.9 %, and the converged,
jointly kept positions within 1e-3 px except the named, count-bounded
classes of tests/test_gpu_parity.py (rounding-sensitive, FP32-only).
"""
import os
import threading

import numpy as np
import pytest

import localizer_b200 as L
from localizer_b200 import synth
from oracle import oracle as O
from tests.test_gpu_parity import FLAG_AGREEMENT, check_classes, parity_classes

pytestmark = pytest.mark.gpu

REF_MAX_ITER = 200


def _ref_fit_threads(frames, cands, method, w0, threads):
    """Reference fitter over whole frames per host thread."""
    frame_ids = np.unique(cands["frame"])
    chunks = [c for c in np.array_split(frame_ids, threads) if len(c)]
    n = len(cands)
    out = np.full((n, O.REF_COLUMNS[method]), np.nan)
    kept = np.zeros(n, dtype=bool)
    iters = np.zeros(n, dtype=np.int32)

    def work(ch):
        idx = np.nonzero(np.isin(cands["frame"], ch))[0]
        o, k, it, _ = O.ref_fit(frames, np.ascontiguousarray(cands[idx]), method, w0)
        out[idx], kept[idx], iters[idx] = o, k == 1, it

    ths = [threading.Thread(target=work, args=(c,)) for c in chunks]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    return out, kept, iters


def _fit(engine, d_frames, cands, method, w0, precision):
    import torch
    n = len(cands)
    ncol = L.lib().loc_output_columns(method)
    d_c = torch.from_numpy(cands.view(np.uint8)).cuda()
    d_o = torch.empty((n, ncol), dtype=torch.float64, device="cuda")
    d_f = torch.empty(n, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    engine.fit_device(d_frames.data_ptr(), d_frames.shape[0], d_frames.shape[2], d_frames.shape[1], d_c.data_ptr(),
                      n, method, w0, 1.0, d_o.data_ptr(), d_f.data_ptr(), stream,
                      L.default_options(max_half_width=int(cands["half_width"].max()), precision=precision))
    engine.sync(stream)
    return d_o.cpu().numpy(), d_f.cpu().numpy()


@pytest.mark.parametrize("wname,method,n_frames,min_cands", [("small", 0, 512, 20_000),
                                                             ("stress", 0, 5000, 200_000),
                                                             ("uneven", 7, 10_000, 1_500_000)])
def test_workload_full_size_against_reference(wname, method, n_frames, min_cands):
    w = synth.workloads()[wname]
    assert w.n_frames == n_frames
    d_frames, _ = synth.make_device(w)
    raw, n = L.find_candidates_device(d_frames, 30.0, w.w0)
    cands = raw.cpu().numpy().view(L.CANDIDATE_DTYPE).copy()
    del raw
    assert n >= min_cands
    cands["half_width"] = np.random.default_rng(w.seed + 17).choice(np.array(w.half_widths), size=n)
    engine = L.Engine(0)
    try:
        rows, flags = _fit(engine, d_frames, cands, method, w.w0, 0)
        rows64, flags64 = _fit(engine, d_frames, cands, method, w.w0, 1)
    finally:
        engine.close()
    frames = d_frames.cpu().numpy().view(np.uint16)
    del d_frames
    out, kept, iters = _ref_fit_threads(frames, cands, method, w.w0, max(os.cpu_count() or 1, 1))
    agree = np.mean((flags == 0) == kept)
    assert agree >= FLAG_AGREEMENT, agree
    capped = iters >= REF_MAX_ITER
    assert np.mean(capped) < 0.01
    c = parity_classes(rows, flags, rows64, flags64, out, kept, ~capped, method)
    assert c["n"] > 0.8 * n, c
    check_classes(c)
