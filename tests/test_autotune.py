"""loc_autotune: the launch-shape tuner of the FP32 solver.

It times shapes on a sample with CUDA events and keeps one only if it gives
the default shape's results (a launch shape changes the FP32 summation order
and nothing else). Checked here: the tuned shape is one of the documented
values, it is no slower than the default on the sample it was tuned on, it
is applied to later calls that leave the shape options at 0, and those
calls' rows match a default-shape fit of the same candidates to the
tolerance the tuner enforces."""
import numpy as np
import pytest

import localizer_b200 as L
from localizer_b200 import synth

pytestmark = pytest.mark.gpu


def _workload(n_frames=200):
    import torch
    w = synth.scaled(synth.workloads()["uneven"], n_frames, seed=4242)
    frames, _ = synth.make_device(w)
    raw, n = L.find_candidates_device(frames, 30.0, w.w0)
    cands = raw.cpu().numpy().view(L.CANDIDATE_DTYPE).copy()
    cands["half_width"] = np.random.default_rng(3).choice(np.array(w.half_widths), size=n)
    return w, frames, cands, torch.from_numpy(cands.view(np.uint8)).cuda()


def _fit(eng, frames, d_cands, n, method, w0, opts):
    import torch
    ncol = L.lib().loc_output_columns(method)
    o = torch.empty((n, ncol), dtype=torch.float64, device="cuda")
    f = torch.empty(n, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    eng.fit_device(frames.data_ptr(), frames.shape[0], frames.shape[2], frames.shape[1], d_cands.data_ptr(), n,
                   method, w0, 1.0, o.data_ptr(), f.data_ptr(), s, opts)
    eng.sync(s)
    return o.cpu().numpy(), f.cpu().numpy()


@pytest.mark.parametrize("method", [7, 0])
def test_tuned_shape_is_applied_and_keeps_results(method):
    w, frames, cands, d_cands = _workload()
    n = len(cands)
    eng = L.Engine(0)
    ref_eng = L.Engine(0)
    try:
        base = L.default_options(max_half_width=6)
        t = eng.autotune(frames.data_ptr(), frames.shape[0], frames.shape[2], frames.shape[1], d_cands.data_ptr(),
                         n, method, w.w0, options=base)
        assert t["threads_per_fit"] in (1, 4, 8, 16) and t["tail_threads_per_fit"] in (4, 8)
        assert t["level0_budget"] in (16, 24, 32, 48, 64) and t["threads_per_block"] in (64, 96, 128)
        assert t["rerun_threads_per_fit"] in (1, 2, 4, 8) and t["long_rerun_threads_per_fit"] in (2, 4, 8)
        assert t["trials"] >= 10 and 0 < t["ms_tuned"] <= t["ms_default"]
        lim = max(1, n // 10000)
        assert t["flag_changes"] <= lim and t["position_changes"] <= lim
        rows_t, flags_t = _fit(eng, frames, d_cands, n, method, w.w0, L.default_options(max_half_width=6))
        explicit = L.default_options(max_half_width=6, threads_per_fit=t["threads_per_fit"],
                                     tail_threads_per_fit=t["tail_threads_per_fit"],
                                     level0_budget=t["level0_budget"],
                                     rerun_threads_per_fit=t["rerun_threads_per_fit"],
                                     long_rerun_threads_per_fit=t["long_rerun_threads_per_fit"],
                                     threads_per_block=t["threads_per_block"])
        rows_e, flags_e = _fit(ref_eng, frames, d_cands, n, method, w.w0, explicit)
        # the tuned context applies exactly the tuned shape
        np.testing.assert_array_equal(flags_t, flags_e)
        np.testing.assert_array_equal(rows_t, rows_e)
        rows_d, flags_d = _fit(ref_eng, frames, d_cands, n, method, w.w0, L.default_options(max_half_width=6))
        assert np.sum((flags_t == 0) != (flags_d == 0)) <= lim
        both = (flags_t == 0) & (flags_d == 0)
        xi = 4 if method == 7 else 3
        err = np.abs(rows_t[both, xi:xi + 2] - rows_d[both, xi:xi + 2]).max(axis=1)
        assert np.sum(err >= 1e-3) <= lim
    finally:
        eng.close()
        ref_eng.close()


def test_autotune_rejects_bad_input():
    lib = L.lib()
    t = L.Tuning()
    assert lib.loc_autotune(None, None, 1, 8, 8, None, 1, 0, 1.3, 1.0, None, t, None) == -1


@pytest.mark.parametrize("method", [0, 7])
def test_every_shape_finishes_every_fit(method):
    """Each shape the tuner may pick (threads per fit in either level, first-
    level budget, FP64 re-run threads) finishes every enqueued fit, in a
    fresh context whose scratch holds no earlier call's solver state, and
    gives the default shape's flags for all but a handful of fits."""
    w, frames, cands, d_cands = _workload(60)
    n = len(cands)
    base = L.default_options(max_half_width=6)
    eng = L.Engine(0)
    try:
        rows0, flags0 = _fit(eng, frames, d_cands, n, method, w.w0, base)
        enqueued = int(np.sum((flags0 != 1) & (flags0 != 10)))
        assert eng.stats()["fits"] == enqueued
    finally:
        eng.close()
    shapes = [dict(threads_per_fit=t, level0_budget=b) for t in (1, 4, 8, 16) for b in (16, 64)]
    shapes += [dict(tail_threads_per_fit=4), dict(tail_threads_per_fit=1), dict(rerun_threads_per_fit=1),
               dict(rerun_threads_per_fit=8, long_rerun_threads_per_fit=2), dict(threads_per_block=64)]
    for kw in shapes:
        eng = L.Engine(0)
        try:
            rows, flags = _fit(eng, frames, d_cands, n, method, w.w0, L.default_options(max_half_width=6, **kw))
            assert eng.stats()["fits"] == enqueued, kw
            assert np.sum(flags != flags0) <= max(2, n // 2000), kw
        finally:
            eng.close()
