"""TEST INFRASTRUCTURE ONLY — ctypes access to the CPU oracle.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only as the checker. Two libraries:

* ``liboracle.so`` — the C restatement of the fit path (loc_oracle.c),
  needs no reference tree;
* ``_ref/libloc_ref.so`` — the reference's own Localization.cpp / Storage.cpp
  / ParticleFinding.cpp built unmodified against the lmsder restatement
  (oracle/Makefile); present wherever it was built.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libloc_ref.so")
REF_FAST_SO = os.path.join(HERE, "_ref", "libloc_ref_fast.so")
CAPI_SO = os.path.join(HERE, "_ref", "libfitpositions_gpu.so")

CAND_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("intensity", "<f8"), ("background", "<f8"),
                       ("frame", "<i4"), ("half_width", "<i4")], align=True)
assert CAND_DTYPE.itemsize == 40

REF_COLUMNS = {0: 12, 1: 10, 5: 16, 6: 8, 7: 16}
N_PARAMS = {0: 5, 1: 4, 5: 7, 6: 5, 7: 7}


class _Options(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("epsabs", C.c_double), ("epsrel", C.c_double),
                ("nthreads", C.c_int), ("init_params", C.c_void_p)]


_lib = None
_ref = None
_ref_fast = None


# the reference tree the Makefile compiles from: $LOC_REFERENCE, else the
# Makefile's own default (its REF variable)
DEFAULT_REF = "/root/reference"


def reference_tree() -> str:
    return os.environ.get("LOC_REFERENCE", DEFAULT_REF)


def build():
    """Compile the oracle, and, when the reference tree exists, the reference
    build and the C++ adapter test library (after the product library)."""
    import subprocess
    ref = reference_tree()
    targets = ["oracle"]
    if os.path.isdir(os.path.join(ref, "source")):
        targets += ["ref", "reffast", "capi"]
    subprocess.run(["make", "-s", "-C", HERE, f"REF={ref}"] + targets, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.oracle_fit.restype = C.c_int
        L.oracle_fit.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                 C.c_double, C.c_double, C.POINTER(_Options), C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p]
        L.oracle_model_jacobian.restype = C.c_int
        L.oracle_model_jacobian.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                            C.c_double, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_glrt_mask.restype = C.c_int
        L.oracle_glrt_mask.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p]
        L.oracle_find_adjacent8.restype = C.c_int
        L.oracle_find_adjacent8.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
        L.oracle_trajectory.restype = C.c_int
        L.oracle_trajectory.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.oracle_last_counters.restype = None
        L.oracle_last_counters.argtypes = [C.POINTER(C.c_long)] * 4
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_fast_available() -> bool:
    return os.path.exists(REF_FAST_SO)


def ref(fast: bool = False):
    """The reference build (strict FP64: the yardstick), or with fast=True
    the same sources built with the reference's release flags (-O2
    -ffast-math), for timing only."""
    global _ref, _ref_fast
    if fast:
        if _ref_fast is None:
            _ref_fast = _bind_ref(C.CDLL(REF_FAST_SO))
        return _ref_fast
    if _ref is None:
        _ref = _bind_ref(C.CDLL(REF_SO))
    return _ref


def _bind_ref(L):
    L.ref_fit.restype = C.c_int
    L.ref_fit.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                          C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.ref_find_adjacent8.restype = C.c_int
    L.ref_find_adjacent8.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
    L.ref_glrt_mask.restype = C.c_int
    L.ref_glrt_mask.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p]
    L.ref_find_candidates.restype = C.c_long
    L.ref_find_candidates.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                      C.c_void_p, C.c_long]
    L.ref_write_positions.restype = C.c_int
    L.ref_write_positions.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                      C.c_double, C.c_double, C.c_char_p, C.c_char_p]
    return L


def _stack_dims(frames: np.ndarray):
    assert frames.dtype == np.uint16 and frames.ndim == 3 and frames.flags.c_contiguous
    n_frames, n_cols, n_rows = frames.shape
    return n_frames, n_rows, n_cols


def fit(frames, cands, method, w0, sigma=1.0, max_iter=200, eps=1e-4, nthreads=1, init_params=None):
    """Oracle fit. Returns (out[nc, cols+2], flags[nc], params[nc, p], fnorm[nc])."""
    n_frames, n_rows, n_cols = _stack_dims(frames)
    cands = np.ascontiguousarray(cands, dtype=CAND_DTYPE)
    nc = len(cands)
    ncol = REF_COLUMNS[method] + 2
    p = N_PARAMS[method]
    out = np.zeros((nc, ncol))
    flags = np.zeros(nc, dtype=np.uint8)
    params = np.zeros((nc, p))
    fnorm = np.zeros(nc)
    ip = None
    if init_params is not None:
        ip = np.ascontiguousarray(init_params, dtype=np.float64)
        assert ip.shape == (nc, p)
    opt = _Options(max_iter, eps, eps, nthreads, ip.ctypes.data if ip is not None else None)
    rc = lib().oracle_fit(frames.ctypes.data, n_frames, n_rows, n_cols, cands.ctypes.data, nc, method,
                          w0, sigma, C.byref(opt), out.ctypes.data, flags.ctypes.data,
                          params.ctypes.data, fnorm.ctypes.data)
    if rc != 0:
        raise ValueError(f"oracle_fit failed: {rc}")
    return out, flags, params, fnorm


def last_counters():
    v = [C.c_long() for _ in range(4)]
    lib().oracle_last_counters(*[C.byref(x) for x in v])
    return dict(iterate_calls=v[0].value, f_evals=v[1].value, df_evals=v[2].value,
                lambda_trials=v[3].value)


def model_jacobian(method, params, w0, sigma, x_off, y_off, r, roi):
    params = np.ascontiguousarray(params, dtype=np.float64)
    roi = np.ascontiguousarray(roi, dtype=np.float64)
    n = (2 * r + 1) ** 2
    f = np.zeros(n)
    J = np.zeros((n, N_PARAMS[method]))
    rc = lib().oracle_model_jacobian(method, params.ctypes.data, w0, sigma, x_off, y_off, r,
                                     roi.ctypes.data, f.ctypes.data, J.ctypes.data)
    if rc != 0:
        raise ValueError(rc)
    return f, J


def trajectory(method, roi, r, x_off, y_off, w0, sigma, x0, max_rec=200):
    """(cumulative trial evaluations, point) after each iterate() call."""
    roi = np.ascontiguousarray(roi, dtype=np.float64)
    x0 = np.ascontiguousarray(x0, dtype=np.float64)
    p = N_PARAMS[method]
    trials = np.zeros(max_rec, dtype=np.int32)
    xs = np.zeros((max_rec, p))
    k = lib().oracle_trajectory(method, roi.ctypes.data, r, x_off, y_off, w0, sigma, x0.ctypes.data, max_rec,
                                trials.ctypes.data, xs.ctypes.data)
    return trials[:k], xs[:k]


def glrt_mask(frame2d, pfa, psf_width):
    frame2d = np.ascontiguousarray(frame2d, dtype=np.uint16)
    n_cols, n_rows = frame2d.shape
    mask = np.zeros((n_cols, n_rows), dtype=np.int32)
    lib().oracle_glrt_mask(frame2d.ctypes.data, n_rows, n_cols, pfa, psf_width, mask.ctypes.data)
    return mask


def _find(fn, frame2d, mask, max_out=1 << 16):
    frame2d = np.ascontiguousarray(frame2d, dtype=np.uint16)
    mask = np.ascontiguousarray(mask, dtype=np.int32)
    n_cols, n_rows = frame2d.shape
    out = np.zeros((max_out, 4))
    n = fn(frame2d.ctypes.data, n_rows, n_cols, mask.ctypes.data, out.ctypes.data, max_out)
    if n < 0:
        raise ValueError(n)
    return out[:min(n, max_out)].copy()


def ref_glrt_mask(frame2d, pfa, psf_width):
    """The reference's own ThresholdImage_GLRT_FFT mask (FFT correlation on
    fftw_shim.c) of one frame [y, x]: 255 where detected."""
    frame2d = np.ascontiguousarray(frame2d, dtype=np.uint16)
    n_cols, n_rows = frame2d.shape
    mask = np.zeros((n_cols, n_rows), dtype=np.int32)
    if ref().ref_glrt_mask(frame2d.ctypes.data, n_rows, n_cols, pfa, psf_width, mask.ctypes.data) != 0:
        raise RuntimeError("ref_glrt_mask failed")
    return mask


def ref_find_candidates(frames, pfa, psf_width):
    """The reference's own candidate pipeline (GLRT + adjacent-8, one
    thresholder and finder for the stack) as a CAND_DTYPE array in frame
    order, half_width 0."""
    n_frames, n_rows, n_cols = _stack_dims(frames)
    cap = max(1024, 64 * n_frames)
    while True:
        out = np.zeros((cap, 5))
        n = ref().ref_find_candidates(frames.ctypes.data, n_frames, n_rows, n_cols, pfa, psf_width,
                                      out.ctypes.data, cap)
        if n < 0:
            raise RuntimeError("ref_find_candidates failed")
        if n <= cap:
            break
        cap = n
    c = np.zeros(n, dtype=CAND_DTYPE)
    for k, name in enumerate(("x", "y", "intensity", "background")):
        c[name] = out[:n, k]
    c["frame"] = out[:n, 4].astype(np.int32)
    return c


def glrt_statistic(frame2d, psf_width, pixels):
    """The GLRT test statistic (Segmentation.cpp:400-420) at the given
    (x, y) pixels, by direct sums in FP64 (exact box sums)."""
    f = np.asarray(frame2d, dtype=np.float64)
    ws = int(np.ceil(4 * psf_width))
    ws += 1 - ws % 2
    half = ws // 2
    npix = float(ws * ws)
    d = np.arange(-half, half + 1, dtype=np.float64)
    g = 1.0 / (1.77245385 * psf_width) * np.exp(-1.0 / (2.0 * psf_width * psf_width) *
                                              (d[None, :] ** 2 + d[:, None] ** 2))
    g = g - g.sum() / npix
    sumsq = float((g * g).sum())
    out = []
    for x, y in pixels:
        win = f[y - half:y + half + 1, x - half:x + half + 1]
        s1, s2 = win.sum(), (win * win).sum()
        avg = s1 / npix
        null_h = s2 - avg * avg * npix
        alpha = float((win * g).sum()) / sumsq
        out.append(alpha * alpha / null_h * sumsq)
    return np.array(out)


def find_adjacent8(frame2d, mask):
    return _find(lib().oracle_find_adjacent8, frame2d, mask)


def ref_find_adjacent8(frame2d, mask):
    return _find(ref().ref_find_adjacent8, frame2d, mask)


def candidates(frames, pfa, psf_width, half_widths=(0,), seed=0, use_ref=False):
    """GLRT + adjacent-8 candidates for every frame, as a CAND_DTYPE array in
    frame order; half-widths drawn uniformly from ``half_widths``."""
    rng = np.random.default_rng(seed)
    rows = []
    for f in range(frames.shape[0]):
        m = glrt_mask(frames[f], pfa, psf_width)
        parts = ref_find_adjacent8(frames[f], m) if use_ref else find_adjacent8(frames[f], m)
        for p in parts:
            rows.append((p[0], p[1], p[2], p[3], f, int(rng.choice(half_widths))))
    return np.array(rows, dtype=CAND_DTYPE)


def group_for_reference(cands):
    """Stable order in which runs of equal (frame, half_width) are contiguous;
    the reference harness fits one such run per fit_positions() call."""
    return np.lexsort((cands["half_width"], cands["frame"]))


def ref_fit(frames, cands, method, w0, sigma=1.0, fast=False):
    """The reference's own fitter classes (fast=True: the release-flag build).
    Returns (out[nc, cols], kept[nc], iters[nc], status[nc]) in the order of
    ``cands`` (grouped internally)."""
    n_frames, n_rows, n_cols = _stack_dims(frames)
    cands = np.ascontiguousarray(cands, dtype=CAND_DTYPE)
    order = group_for_reference(cands)
    cs = np.ascontiguousarray(cands[order])
    nc = len(cs)
    ncol = REF_COLUMNS[method]
    out = np.full((nc, ncol), np.nan)
    kept = np.zeros(nc, dtype=np.int32)
    iters = np.zeros(nc, dtype=np.int32)
    status = np.zeros(nc, dtype=np.int32)
    rc = ref(fast).ref_fit(frames.ctypes.data, n_frames, n_rows, n_cols, cs.ctypes.data, nc, method, w0,
                       sigma, out.ctypes.data, kept.ctypes.data, iters.ctypes.data, status.ctypes.data)
    if rc != 0:
        raise ValueError(f"ref_fit failed: {rc}")
    inv = np.empty_like(order)
    inv[order] = np.arange(nc)
    return out[inv], kept[inv], iters[inv], status[inv]


def ref_write_positions(frames, cands, method, w0, path, header="", sigma=1.0):
    """The reference's own writePositionsToFile for one frame's candidates
    (same frame and ROI half-width). Returns the number of positions."""
    n_frames, n_rows, n_cols = _stack_dims(frames)
    cands = np.ascontiguousarray(cands, dtype=CAND_DTYPE)
    rc = ref().ref_write_positions(frames.ctypes.data, n_frames, n_rows, n_cols, cands.ctypes.data, len(cands),
                                   method, w0, sigma, path.encode(), header.encode())
    if rc < 0:
        raise RuntimeError(f"ref_write_positions failed: {rc}")
    return rc


def capi_available() -> bool:
    return os.path.exists(CAPI_SO)


def capi_compare(frames, cands, method, w0, sigma=1.0, device=0):
    """Per-frame fit_positions calls of the C++ FitPositions_GPU adapter
    (tests/capi/fitpositions_gpu.cpp, over the product's C ABI) and of the
    reference's own fitter on the same particle lists, merged per side as
    the reference's controller merges them. Returns a dict with both merged
    matrices (N x C) and the (x, y) of the particles each side left in its
    lists."""
    L = C.CDLL(CAPI_SO)
    fn = L.fpgpu_compare
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double,
                   C.c_double, C.c_int, C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.POINTER(C.c_int), C.c_int,
                   C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.POINTER(C.c_int)]
    n_frames, n_rows, n_cols = _stack_dims(frames)
    cands = np.ascontiguousarray(cands, dtype=CAND_DTYPE)
    n = len(cands)
    parts = np.ascontiguousarray(np.stack([cands["x"], cands["y"], cands["intensity"], cands["background"]], axis=1))
    frame_of = np.ascontiguousarray(cands["frame"], dtype=np.int32)
    ncol = REF_COLUMNS[method]
    gm, rm = np.zeros((max(n, 1), ncol)), np.zeros((max(n, 1), ncol))
    gl, rl = np.zeros((max(n, 1), 2)), np.zeros((max(n, 1), 2))
    ng, nr, ngl, nrl = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    rc = fn(frames.ctypes.data, n_frames, n_rows, n_cols, parts.ctypes.data, frame_of.ctypes.data, n, method, w0,
            sigma, device, gm.ctypes.data, C.byref(ng), rm.ctypes.data, C.byref(nr), max(n, 1), gl.ctypes.data,
            C.byref(ngl), rl.ctypes.data, C.byref(nrl))
    if rc != 0:
        raise RuntimeError("fpgpu_compare failed")
    return {"gpu_matrix": gm[:ng.value], "ref_matrix": rm[:nr.value], "gpu_left": gl[:ngl.value],
            "ref_left": rl[:nrl.value]}
