"""Candidate finder against the reference's own GLRT segmentation.

The reference detects emitters with ThresholdImage_GLRT_FFT
(source/Segmentation.cpp:241-430), whose Gaussian correlation runs through an
FFT (Convolver.cpp:120-256) at power-of-two frame sizes. oracle/Makefile
compiles that code unmodified into oracle/_ref, on the FFTW subset restated
in oracle/fftw_shim.c. These tests pin the masks and candidates of the
finders here (the C restatement in oracle/loc_oracle.c, the product's host
finder and its GPU finder) to the reference's own: a pixel may differ only
where the test statistic lies within EPS (relative) of the threshold, where
an FFT and a direct sum can round to different sides.
"""
import numpy as np
import pytest

import localizer_b200 as L
from localizer_b200 import synth
from oracle import oracle as O
from tests import _golden as G

EPS = 1e-9
FIELDS = ("x", "y", "intensity", "background", "frame")

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference build absent")


def _seeded(name, n_frames, seed=77):
    w = synth.scaled(synth.workloads()[name], n_frames)
    em, bg = synth.draw_stack(w)
    return w, synth.render_frames(w, em, bg, list(range(n_frames)), seed=seed)


def _check_masks(frames, pfa, w0):
    ws = int(np.ceil(4 * w0))
    ws += 1 - ws % 2
    thr = 1.0 - np.exp(-pfa / (ws * ws))
    n_diff = 0
    for f in range(frames.shape[0]):
        a = O.ref_glrt_mask(frames[f], pfa, w0)
        b = O.glrt_mask(frames[f], pfa, w0)
        d = np.argwhere(a != b)
        if len(d):
            st = O.glrt_statistic(frames[f], w0, [(x, y) for y, x in d])
            near = (np.abs(st - thr) <= EPS * thr) | (np.abs(st - 1.0) <= EPS)
            assert near.all(), (f, d[~near][:5], st[~near][:5], thr)
        n_diff += len(d)
    return n_diff


@pytest.mark.parametrize("name", G.CASES)
def test_reference_glrt_reproduces_golden_candidates(name):
    g = G.load(name)
    assert _check_masks(g["frames"], g["pfa"], g["w0"]) == 0
    c = O.ref_find_candidates(g["frames"], g["pfa"], g["w0"])
    ref = g["cands"][:G.n_found(name, g)]
    assert len(c) == len(ref)
    for k in FIELDS:
        assert np.array_equal(c[k], ref[k]), k


@pytest.mark.parametrize("name,n_frames", [("dense", 3), ("uneven", 8), ("small", 16), ("stress", 8)])
def test_masks_and_host_finder_match_reference_on_seeded_frames(name, n_frames):
    w, frames = _seeded(name, n_frames)
    n_diff = _check_masks(frames, 30.0, w.w0)
    ref = O.ref_find_candidates(frames, 30.0, w.w0)
    got = L.find_candidates(frames, 30.0, w.w0, n_threads=2)
    if n_diff == 0:
        assert len(got) == len(ref)
        for k in FIELDS:
            assert np.array_equal(got[k], ref[k]), k
    else:
        assert abs(len(got) - len(ref)) <= n_diff


@pytest.mark.gpu
def test_gpu_finder_matches_reference_on_dense_frames():
    import torch
    w, frames = _seeded("dense", 12, seed=5)
    d = torch.from_numpy(frames.view(np.int16)).cuda()
    raw, n = L.find_candidates_device(d, 30.0, w.w0)
    got = raw.cpu().numpy().view(L.CANDIDATE_DTYPE)
    ref = O.ref_find_candidates(frames, 30.0, w.w0)
    assert _check_masks(frames, 30.0, w.w0) == 0
    assert n == len(ref)
    for k in FIELDS:
        assert np.array_equal(got[k], ref[k]), k
