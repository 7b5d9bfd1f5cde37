"""GPU GLRT + adjacent-8 finder against the host finder (itself bit-exact
with the reference's ParticleFinder_adjacent8 on the golden frames): same
candidates, same order, every field bit-identical."""
import numpy as np
import pytest

import localizer_b200 as L
from localizer_b200 import synth
from tests import _golden as G

pytestmark = pytest.mark.gpu


def _gpu(frames_np, pfa, w, cap=None):
    import torch
    d = torch.from_numpy(np.ascontiguousarray(frames_np).view(np.int16)).cuda()
    if cap is None:
        raw, n = L.find_candidates_device(d, pfa, w)
        return raw.cpu().numpy().view(L.CANDIDATE_DTYPE), n
    out = torch.empty(max(cap, 1) * 40, dtype=torch.uint8, device="cuda")
    import ctypes as C
    n = L.lib().loc_find_candidates(C.c_void_p(d.data_ptr()), d.shape[0], d.shape[2], d.shape[1], pfa, w,
                                    C.c_void_p(out.data_ptr()), cap, None)
    return out.cpu().numpy().view(L.CANDIDATE_DTYPE)[:min(cap, n)], n


def _same(a, b):
    assert len(a) == len(b)
    for f in L.CANDIDATE_DTYPE.names:
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)


@pytest.mark.parametrize("name", ["small", "uneven", "stress"])
def test_gpu_finder_matches_host_on_golden(name):
    g = G.load(name)
    frames = g["frames"]
    host = L.find_candidates(frames, 30.0, float(g["w0"]))
    gpu, n = _gpu(frames, 30.0, float(g["w0"]))
    assert n == len(host) and n > 0
    _same(gpu, host)


def test_gpu_finder_matches_host_on_seeded_stack():
    w = synth.scaled(synth.workloads()["uneven"], 300, seed=777)
    frames, _ = synth.make(w)
    for pfa, width in ((30.0, 1.5), (20.0, 1.3), (60.0, 2.0)):
        host = L.find_candidates(frames, pfa, width)
        gpu, n = _gpu(frames, pfa, width)
        assert n == len(host)
        _same(gpu, host)


def test_gpu_finder_edge_cases():
    rng = np.random.default_rng(5)
    # odd frame sizes (the test area is trimmed to even extents), a flat frame, noise only
    odd = rng.poisson(100, size=(3, 77, 101)).astype(np.uint16)
    odd[1, 30:33, 40:43] += 900
    flat = np.full((2, 64, 64), 100, dtype=np.uint16)
    for frames in (odd, flat):
        host = L.find_candidates(frames, 30.0, 1.5)
        gpu, n = _gpu(frames, 30.0, 1.5)
        assert n == len(host)
        _same(gpu, host)
    assert _gpu(flat, 30.0, 1.5)[1] == 0
    # a buffer smaller than the result: the count is still the total
    g = G.load("small")
    host = L.find_candidates(g["frames"], 30.0, float(g["w0"]))
    part, n = _gpu(g["frames"], 30.0, float(g["w0"]), cap=10)
    assert n == len(host)
    _same(part, host[:10])


@pytest.mark.parametrize("name,n_frames", [("uneven", 300), ("stress", 200)])
def test_device_synthesis_is_reproducible(name, n_frames):
    """Frames rendered on the GPU (the bench's workload) are identical across
    renders of the same seed, and so are the candidates found in them."""
    import torch
    w = synth.scaled(synth.workloads()[name], n_frames, seed=77)
    a, _ = synth.make_device(w)
    b, _ = synth.make_device(w)
    assert torch.equal(a, b)
    ca, na = L.find_candidates_device(a, 30.0, w.w0)
    cb, nb = L.find_candidates_device(b, 30.0, w.w0)
    assert na == nb and torch.equal(ca, cb)
