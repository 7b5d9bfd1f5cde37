"""The boundary from C++: the FitPositions_GPU adapter
(tests/capi/fitpositions_gpu.cpp, compiled against the reference's own
Localization.h / Storage.h and linked with the product library) driven the
way the reference's worker drives a fitter (source/PALMAnalysis.cpp:196-240:
one fit_positions call per frame, setFrameNumbers, merge), next to the
reference's own fitter on the same particle lists; and the reference-DLL
entry point LocalizerFitEmitters (source/LocalizerDLL.cpp:89-129) against
the reference pipeline it replaces (GLRT + adjacent-8 +
FitPositions_EllipsoidalGaussian(psfWidth, 1.0))."""
import os

import numpy as np
import pytest

import localizer_b200 as L
from oracle import oracle as O
from tests import _golden as G

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

XCOL = {0: 3, 1: 2, 5: 4, 6: 3, 7: 4}


def _index(cands):
    return {(int(c["frame"]), float(c["x"]), float(c["y"])): k for k, c in enumerate(cands)}


def _compare_in_child(name, method, tmp_path):
    """Run the adapter and the reference fitter in a child process (a fault
    in either then fails this test with its stderr instead of ending the
    session) and load both results."""
    import subprocess
    import sys
    out = tmp_path / "cmp.npz"
    code = ("import sys, numpy as np; sys.path.insert(0, {root!r}); "
            "from oracle import oracle as O; from tests import _golden as G; "
            "g = G.load({name!r}); c = g['cands'].copy(); c['half_width'] = 0; "
            "r = O.capi_compare(g['frames'], c, {method}, g['w0']); "
            "np.savez({out!r}, **r)").format(root=ROOT, name=name, method=method, out=str(out))
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    z = np.load(out)
    return {k: z[k] for k in z.files}


@pytest.mark.skipif(not O.capi_available(), reason="adapter library not built (needs the reference tree)")
@pytest.mark.parametrize("name,method", list(G.all_cases()))
def test_fitpositions_gpu_adapter_matches_reference_fitter(name, method, tmp_path):
    g = G.load(name)
    # the adapter, like the reference's fitter constructors, fits every
    # candidate with the ROI half-width ceil(4 w0) (Localization.h:68)
    cands = g["cands"].copy()
    cands["half_width"] = 0
    r = _compare_in_child(name, method, tmp_path)
    _, ref_kept, ref_iters, _ = O.ref_fit(g["frames"], cands, method, g["w0"])
    gm, rm, gl, rl = r["gpu_matrix"], r["ref_matrix"], r["gpu_left"], r["ref_left"]
    if method == 5:
        _check_sympsf(cands, gm, rm, gl, rl, ref_kept, ref_iters)
        return
    # one container row per particle left in the list, on both sides
    assert len(gm) == len(gl) and len(rm) == len(rl)
    idx = _index(cands)
    gi = np.array([idx[(int(m[0]), float(p[0]), float(p[1]))] for m, p in zip(gm, gl)], dtype=int)
    ri = np.array([idx[(int(m[0]), float(p[0]), float(p[1]))] for m, p in zip(rm, rl)], dtype=int)
    gk = np.zeros(len(cands), bool)
    rk = np.zeros(len(cands), bool)
    gk[gi] = True
    rk[ri] = True
    # the reference side's list erasure is that of the harness run
    assert np.array_equal(rk, ref_kept == 1)
    assert np.sum(gk != rk) <= max(1, int(0.001 * len(cands)))
    # rows of particles both sides kept, in the reference's column order
    both = np.nonzero(gk & rk)[0]
    pos_g = {k: n for n, k in enumerate(gi)}
    pos_r = {k: n for n, k in enumerate(ri)}
    a = gm[[pos_g[k] for k in both]]
    b = rm[[pos_r[k] for k in both]]
    np.testing.assert_array_equal(a[:, 0], b[:, 0])           # frame numbers from setFrameNumbers
    conv = ref_iters[both] < 200
    xi = XCOL[method]
    err = np.abs(a[conv, xi:xi + 2] - b[conv, xi:xi + 2]).max(axis=1)
    assert len(err) > 0.3 * len(cands)
    assert err.max() < 1e-3, np.sort(err)[-5:]


def _check_sympsf(cands, gm, rm, gl, rl, ref_kept, ref_iters):
    """Method 5: the lists keep the particles the symmetric-PSF filter drops
    (the inner ellipsoidal fit erases its own rejects), so the lists of both
    sides are compared as sets of particles, and the containers row by row
    in particle order."""
    lim = max(1, int(0.001 * len(cands)))
    gs = {(float(x), float(y)) for x, y in gl}
    rs = {(float(x), float(y)) for x, y in rl}
    assert len(gs ^ rs) <= lim
    assert abs(len(gm) - len(rm)) <= lim
    if len(gm) == len(rm):
        np.testing.assert_array_equal(gm[:, 0], rm[:, 0])
        err = np.abs(gm[:, 4:6] - rm[:, 4:6]).max(axis=1)
        assert np.sum(err >= 1e-3) <= lim, np.sort(err)[-5:]


def _reference_pipeline(frames, pfa, w0):
    cands = O.candidates(frames, pfa, w0, use_ref=True)
    out, kept, _, _ = O.ref_fit(frames, cands, 7, w0, 1.0)
    return cands, out[kept == 1]


@pytest.mark.parametrize("name", ["uneven", "small"])
def test_localizer_fit_emitters_matches_reference_pipeline(name):
    g = G.load(name)
    frames, w0, pfa = g["frames"], g["w0"], g["pfa"]
    got = L.LocalizerFitEmitters(frames, w0, pfa)
    cands, ref = _reference_pipeline(frames, pfa, w0)
    assert got.shape[1] == 16
    assert abs(len(got) - len(ref)) <= max(1, int(0.001 * len(cands)))
    # rows pair up by frame and position
    xi = XCOL[7]
    matched = 0
    for row in ref:
        same = got[got[:, 0] == row[0]]
        d = np.abs(same[:, xi:xi + 2] - row[xi:xi + 2]).max(axis=1) if len(same) else np.array([np.inf])
        matched += bool(d.min() < 1e-3)
    assert matched >= len(ref) - max(1, int(0.002 * len(ref)))
    # frames in ascending order, as the reference's sorted container
    assert np.all(np.diff(got[:, 0]) >= 0)


def test_localizer_fit_emitters_empty_stack():
    frames = np.zeros((0, 64, 64), dtype=np.uint16)
    got = L.LocalizerFitEmitters(frames, 1.5, 30.0)
    assert got.shape == (0, 16)
