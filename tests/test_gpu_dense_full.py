"""The dense workload at its full size: 50,000 frames of 512 x 512 uint16
(26.2 GB resident), 300-1000 emitters per frame, ROI half-widths 3-6,
symmetric (method 0) and ellipsoidal (method 7) fits interleaved by frame.

At this size the FP64 oracle cannot check every fit, so the whole run is
checked through properties that do not depend on its size:

* every candidate gets its row (frame column = its frame), rejected rows are
  NaN except the frame, kept rows have finite frame, position, angle and
  background (and all columns but for < 0.1 % of degenerate fits) and their
  centre lies in the candidate's ROI window (the reference's window rule);
* the solver fitted exactly the candidates that the edge rule kept;
* a fit does not depend on the batch around it: the candidates of a sample
  of frames fitted as a small batch give bit-identical rows and flags;
* on that sample the FP64 oracle's gates hold (flags; positions <= 1e-3 px
  except the named classes of tests/test_gpu_parity.py, bounded by count).
"""
import numpy as np
import pytest

import localizer_b200 as L
from localizer_b200 import synth
from oracle import oracle as O
from tests.test_gpu_parity import check_classes, parity_classes

pytestmark = pytest.mark.gpu

XCOL = {0: 3, 7: 4}
FINITE_COLS = {0: [0, 1, 2, 3, 4, 5], 7: [0, 4, 5, 6, 7]}   # always finite in kept rows
SAMPLE_FRAMES = 40


def _fit(engine, d_frames, cands, method, w0, precision=0):
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
    return d_c, d_o, d_f


def test_dense_workload_full_size():
    import torch
    w = synth.workloads()["dense"]
    d_frames, _ = synth.make_device(w)
    assert tuple(d_frames.shape) == (50000, 512, 512)
    raw, n = L.find_candidates_device(d_frames, 30.0, w.w0)
    cands = raw.cpu().numpy().view(L.CANDIDATE_DTYPE).copy()
    del raw
    assert n > 20_000_000
    cands["half_width"] = np.random.default_rng(w.seed + 17).choice(np.array(w.half_widths), size=n)
    engine = L.Engine(0)
    rng = np.random.default_rng(5)
    sample = np.sort(rng.choice(w.n_frames, size=SAMPLE_FRAMES, replace=False))
    for method in (0, 7):
        part = cands[cands["frame"] % 2 == (0 if method == 0 else 1)]
        d_c, d_o, d_f = _fit(engine, d_frames, part, method, w.w0)
        st = engine.stats()
        ncol = d_o.shape[1]
        ref = O.REF_COLUMNS[method]
        frame = torch.from_numpy(part["frame"].astype(np.float64)).cuda()
        assert torch.equal(d_o[:, 0], frame)
        assert int(d_f.max()) <= 11
        kept = d_f == 0
        edge = (d_f == 1) | (d_f == 10)
        assert st["fits"] == len(part) - int(edge.sum())
        # Frame, position, angle and background are finite for every kept row.
        # Integral, widths and deviations follow the reference's formulas:
        # |rho| >= 1 gives sqrt of a negative number for the integral and the
        # smaller axis, and (J^T J)^-1 fails to factorise for collapsed
        # ellipsoids; the reference's own values there are NaN, inf or 1e14-1e19.
        finite = torch.isfinite(d_o[kept, :ref])
        bad_cols = (~finite).sum(dim=0).tolist()
        assert bool(finite[:, FINITE_COLS[method]].all()), bad_cols
        assert float((~finite).any(dim=1).float().mean()) < 1e-3, bad_cols
        assert bool(torch.isnan(d_o[~kept, 1:ref]).all())
        hw = torch.from_numpy(part["half_width"].astype(np.float64)).cuda()
        xi = XCOL[method]
        for c, col in ((torch.from_numpy(np.ascontiguousarray(part["x"])).cuda(), xi),
                       (torch.from_numpy(np.ascontiguousarray(part["y"])).cuda(), xi + 1)):
            lo = torch.floor(c - hw)
            v = d_o[:, col]
            assert bool(((v[kept] >= lo[kept]) & (v[kept] <= lo[kept] + 2 * hw[kept])).all())
        assert float(kept.float().mean()) > 0.4
        assert bool((d_o[:, ncol - 2] <= 200).all())

        # a sample of whole frames, fitted again as a small batch: bit-identical
        sel = np.nonzero(np.isin(part["frame"], sample))[0]
        rows_full = d_o[torch.from_numpy(sel).cuda()].cpu().numpy()
        flags_full = d_f[torch.from_numpy(sel).cuda()].cpu().numpy()
        del d_c, d_o, d_f
        _, s_o, s_f = _fit(engine, d_frames, part[sel], method, w.w0)
        np.testing.assert_array_equal(s_f.cpu().numpy(), flags_full)
        np.testing.assert_array_equal(s_o.cpu().numpy(), rows_full)

        # the FP64 oracle on the sample
        sub = part[sel].copy()
        frames_s = d_frames[torch.from_numpy(sample).cuda()].cpu().numpy().view(np.uint16)
        sub["frame"] = np.searchsorted(sample, sub["frame"])
        out, oflags, _, _ = O.fit(frames_s, sub, method, w.w0, nthreads=16)
        okept = oflags == 0
        gkept = flags_full == 0
        capped = out[:, ref + 1] == 1
        assert np.sum(gkept != okept) <= max(1, int(0.001 * len(sub))), np.mean(gkept == okept)
        # the same fits in FP64 on the GPU name the rounding-sensitive ones
        _, o64, f64 = _fit(engine, d_frames, part[sel], method, w.w0, precision=1)
        check_classes(parity_classes(rows_full, flags_full, o64.cpu().numpy(), f64.cpu().numpy(), out, okept, ~capped,
                                     method))
    engine.close()
