"""localizer_b200 — B200-native Gaussian PSF localization fits.

Host-side mirror of the reference's fitting interface (FitPositions_* of
Localizer, source/Localization.h:55-121) over the C ABI of
``liblocalizer_b200.so`` (include/localizer_b200.h). Every fit runs in the
CUDA kernels of that library; there is no CPU fallback: importing works
without a GPU, but any fit raises if the library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblocalizer_b200.so")

# method codes (Defines.h:157-163)
METHOD_2DGAUSS = 0
METHOD_2DGAUSS_FIXEDWIDTH = 1
METHOD_2DGAUSS_ELLIPSOIDAL = 5
METHOD_MLEWG = 6
METHOD_2DGAUSS_ELLIPSOIDAL_ASTIGMATISM = 7

FLAGS = {0: "kept", 1: "edge", 2: "amplitude", 3: "out_of_window", 4: "width_range", 5: "drift",
         6: "eigen", 7: "no_axis", 8: "sympsf_ratio", 9: "sympsf_width", 10: "bad_input"}

REF_COLUMNS = {0: 12, 1: 10, 5: 16, 6: 8, 7: 16}
N_PARAMS = {0: 5, 1: 4, 5: 7, 7: 7}

COLUMN_NAMES = {
    0: ["frame", "integral", "width", "x", "y", "background", "integral_dev", "width_dev", "x_dev", "y_dev",
        "background_dev", "n_frames"],
    1: ["frame", "integral", "x", "y", "background", "integral_dev", "x_dev", "y_dev", "background_dev",
        "n_frames"],
    7: ["frame", "integral", "sigma1", "sigma2", "x", "y", "theta", "background", "integral_dev", "sigma1_dev",
        "sigma2_dev", "x_dev", "y_dev", "theta_dev", "background_dev", "n_frames"],
}
COLUMN_NAMES[5] = COLUMN_NAMES[7]
COLUMN_NAMES[6] = ["frame", "integral", "width", "x", "y", "background", "position_dev", "n_frames"]

CANDIDATE_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("intensity", "<f8"), ("background", "<f8"),
                            ("frame", "<i4"), ("half_width", "<i4")], align=True)
assert CANDIDATE_DTYPE.itemsize == 40


class Options(C.Structure):
    _fields_ = [("max_iter", C.c_int32), ("epsabs", C.c_double), ("epsrel", C.c_double),
                ("precision", C.c_int32), ("pivot_threshold", C.c_float), ("threads_per_block", C.c_int32),
                ("blocks_per_sm", C.c_int32), ("stage_u16", C.c_int32), ("max_half_width", C.c_int32),
                ("d_init_params", C.c_void_p), ("d_params_out", C.c_void_p), ("d_diag", C.c_void_p),
                ("threads_per_fit", C.c_int32), ("tail_threads_per_fit", C.c_int32), ("level0_budget", C.c_int32),
                ("fp64_rerun", C.c_int32), ("rerun_margin", C.c_float), ("rerun_pivot", C.c_float),
                ("rerun_threads_per_fit", C.c_int32), ("serial_classes", C.c_int32),
                ("proposal", C.c_void_p), ("warm_iter_limit", C.c_int32), ("long_rerun_iters", C.c_int32),
                ("long_rerun_threads_per_fit", C.c_int32), ("compensated", C.c_int32),
                ("rerun_capped", C.c_int32), ("rerun_cond", C.c_float),
                ("rerun_iters", C.c_int32), ("rerun_skip_rejected", C.c_float),
                ("host_roi_mode", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("f_evals", "jacobian_evals", "lambda_solves", "fp64_escalations",
                                          "fits", "iterations", "pixels_f", "pixels_j", "kcycles_refill",
                                          "kcycles_step", "kcycles_pass", "kcycles_decide", "fits_fp64_rerun",
                                          "iterations_fp64_rerun", "kcycles_fp64_rerun",
                                          "kcycles_fp64_rerun_pass")] + \
               [(n, C.c_float) for n in ("queue_ms", "solver_ms", "finalize_ms", "proposal_ms")] + \
               [("kernel_launches", C.c_int32), ("fits_warm", C.c_uint64)]

    def as_dict(self):
        return {n: (float(getattr(self, n)) if n.endswith("_ms") else int(getattr(self, n)))
                for n, _ in self._fields_}


class Tuning(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("threads_per_fit", "tail_threads_per_fit", "level0_budget",
                                         "rerun_threads_per_fit", "long_rerun_threads_per_fit",
                                         "threads_per_block")] + \
               [("ms_default", C.c_float), ("ms_tuned", C.c_float)] + \
               [(n, C.c_int32) for n in ("trials", "flag_changes", "position_changes")]

    def as_dict(self):
        return {n: (float(getattr(self, n)) if n.startswith("ms_") else int(getattr(self, n))) for n, _ in self._fields_}


# names and prototypes of every exported entry point of include/localizer_b200.h
_PROTOS = {
    "loc_default_options": (None, [C.POINTER(Options)]),
    "loc_ctx_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int]),
    "loc_ctx_destroy": (C.c_int, [C.c_void_p]),
    "loc_last_error": (C.c_char_p, []),
    "loc_reference_columns": (C.c_int, [C.c_int]),
    "loc_output_columns": (C.c_int, [C.c_int]),
    "loc_parameter_count": (C.c_int, [C.c_int]),
    "loc_fit_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                C.c_double, C.c_double, C.POINTER(Options), C.c_void_p, C.c_void_p, C.c_void_p]),
    "loc_fit_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                               C.c_double, C.c_double, C.POINTER(Options), C.c_void_p, C.c_void_p]),
    "loc_fit_host_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                     C.c_int, C.c_double, C.c_double, C.POINTER(Options), C.c_void_p, C.c_void_p]),
    "loc_fit_host_wait": (C.c_int, [C.c_void_p]),
    "loc_host_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "loc_fit_batch_static": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                       C.c_double, C.c_double, C.POINTER(Options), C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
    "loc_sync": (C.c_int, [C.c_void_p, C.c_void_p]),
    "loc_autotune": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                               C.c_double, C.c_double, C.POINTER(Options), C.POINTER(Tuning), C.c_void_p]),
    "loc_last_stats": (C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    "loc_compact_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int]),
    "loc_find_candidates_host": (C.c_long, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                            C.c_int, C.c_void_p, C.c_long]),
    "loc_synth_frames": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_float, C.c_ulonglong, C.c_void_p]),
    "LocalizerFitEmitters": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                       C.POINTER(C.c_int), C.POINTER(C.POINTER(C.c_double))]),
    "LocalizerFree": (None, [C.c_void_p]),
    "loc_ingest_frames": (C.c_longlong, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                         C.c_void_p]),
    "loc_write_positions_text": (C.c_long, [C.c_void_p, C.c_void_p, C.c_long, C.c_int, C.c_char_p, C.c_char_p]),
    "loc_find_candidates": (C.c_long, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p,
                                       C.c_long, C.c_void_p]),
    "loc_proposal_weight_count": (C.c_int, [C.c_int]),
    "loc_proposal_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_ulonglong]),
    "loc_proposal_destroy": (C.c_int, [C.c_void_p]),
    "loc_proposal_get_weights": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "loc_proposal_set_weights": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "loc_proposal_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
    "loc_proposal_gradient": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.POINTER(C.c_float), C.c_void_p]),
    "loc_proposal_train_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                          C.c_float, C.POINTER(C.c_float), C.c_void_p]),
    "loc_proposal_status": (C.c_int, [C.c_void_p]),
    "loc_synth_rois": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_ulonglong, C.c_void_p, C.c_void_p]),
}

_lib = None


class LocalizerError(RuntimeError):
    pass


def lib():
    """The native library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise LocalizerError(f"{LIB_PATH} is missing: build it with `python -m localizer_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc < 0:
        raise LocalizerError(f"localizer_b200 error {rc}: {lib().loc_last_error().decode()}")
    return rc


def default_options(**kw) -> Options:
    o = Options()
    lib().loc_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def as_candidates(cands) -> np.ndarray:
    """Candidates as a contiguous CANDIDATE_DTYPE array."""
    if isinstance(cands, np.ndarray) and cands.dtype == CANDIDATE_DTYPE:
        return np.ascontiguousarray(cands)
    a = np.asarray(cands)
    if a.dtype.names:
        out = np.zeros(len(a), dtype=CANDIDATE_DTYPE)
        for n in CANDIDATE_DTYPE.names:
            if n in a.dtype.names:
                out[n] = a[n]
        return out
    a = np.atleast_2d(np.asarray(cands, dtype=np.float64))
    out = np.zeros(len(a), dtype=CANDIDATE_DTYPE)
    for k, n in enumerate(("x", "y", "intensity", "background", "frame", "half_width")):
        if k < a.shape[1]:
            out[n] = a[:, k]
    return out


class Engine:
    """One device context (loc_ctx)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        self._inflight = []
        _check(lib().loc_ctx_create(C.byref(self._h), device))

    def close(self):
        if self._h:
            lib().loc_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def fit_device(self, d_frames: int, n_frames: int, n_rows: int, n_cols: int, d_cands: int, n_cands: int,
                   method: int, w0: float, sigma: float, d_out: int, d_flags: int, stream: int = 0,
                   options: Options | None = None):
        """loc_fit_batch on device pointers (asynchronous on `stream`)."""
        o = options if options is not None else default_options()
        _check(lib().loc_fit_batch(self._h, C.c_void_p(d_frames), n_frames, n_rows, n_cols, C.c_void_p(d_cands),
                                   n_cands, method, w0, sigma, C.byref(o), C.c_void_p(d_out), C.c_void_p(d_flags),
                                   C.c_void_p(stream)))

    def autotune(self, d_frames: int, n_frames: int, n_rows: int, n_cols: int, d_cands: int, n_cands: int,
                 method: int, w0: float, sigma: float = 1.0, options: Options | None = None, stream: int = 0) -> dict:
        """loc_autotune on a device sample; the tuned shape is kept in this
        context for `method`. Returns the loc_tuning fields."""
        t = Tuning()
        _check(lib().loc_autotune(self._h, C.c_void_p(d_frames), n_frames, n_rows, n_cols, C.c_void_p(d_cands),
                                  n_cands, method, w0, sigma, C.byref(options) if options is not None else None,
                                  C.byref(t), C.c_void_p(stream)))
        return t.as_dict()

    def sync(self, stream: int = 0):
        _check(lib().loc_sync(self._h, C.c_void_p(stream)))

    def stats(self) -> dict:
        s = Stats()
        _check(lib().loc_last_stats(self._h, C.byref(s)))
        return s.as_dict()

    def fit_host(self, frames: np.ndarray, cands, method: int, w0: float, sigma: float = 1.0,
                 options: Options | None = None):
        """loc_fit_host: frames (n_frames, n_cols, n_rows) uint16 [f, y, x].
        Returns (rows[n, loc_output_columns], flags[n])."""
        frames = np.ascontiguousarray(frames, dtype=np.uint16)
        if frames.ndim == 2:
            frames = frames[None]
        n_frames, n_cols, n_rows = frames.shape
        cands = as_candidates(cands)
        n = len(cands)
        ncol = _check(lib().loc_output_columns(method))
        out = np.zeros((n, ncol))
        flags = np.zeros(n, dtype=np.uint8)
        o = options if options is not None else default_options()
        _check(lib().loc_fit_host(self._h, frames.ctypes.data, n_frames, n_rows, n_cols, cands.ctypes.data, n,
                                  method, w0, sigma, C.byref(o), out.ctypes.data, flags.ctypes.data))
        return out, flags

    def fit_host_async(self, frames: np.ndarray, cands: np.ndarray, method: int, w0: float, sigma: float,
                       out: np.ndarray, flags: np.ndarray, options: Options | None = None):
        """loc_fit_host_async: enqueue the fit of one stack and return.
        `frames` (n_frames, n_cols, n_rows) uint16, `cands` (CANDIDATE_DTYPE),
        `out` (n, loc_output_columns) float64 and `flags` (n,) uint8 are
        C-contiguous arrays, kept referenced here until wait(); page-locked
        arrays let the copies overlap the fits."""
        n_frames, n_cols, n_rows = frames.shape
        n = len(cands)
        ncol = _check(lib().loc_output_columns(method))
        for a in (frames, cands, out, flags):
            if not a.flags["C_CONTIGUOUS"]:
                raise LocalizerError("fit_host_async needs C-contiguous arrays")
        if frames.dtype.itemsize != 2 or cands.dtype != CANDIDATE_DTYPE or out.shape != (n, ncol) or \
                out.dtype != np.float64 or flags.shape != (n,) or flags.dtype != np.uint8:
            raise LocalizerError("fit_host_async: array types or shapes do not match the call")
        o = options if options is not None else default_options()
        self._inflight.append((frames, cands, out, flags, o))
        _check(lib().loc_fit_host_async(self._h, frames.ctypes.data, n_frames, n_rows, n_cols, cands.ctypes.data,
                                        n, method, w0, sigma, C.byref(o), out.ctypes.data, flags.ctypes.data))

    def wait(self):
        """loc_fit_host_wait: block until every fit_host_async call is done."""
        try:
            _check(lib().loc_fit_host_wait(self._h))
        finally:
            self._inflight = []

    def host_bytes(self):
        """loc_host_bytes: (host -> device, device -> host) bytes copied by
        the context's host-buffer calls so far."""
        h2d, d2h = C.c_uint64(), C.c_uint64()
        _check(lib().loc_host_bytes(self._h, C.byref(h2d), C.byref(d2h)))
        return h2d.value, d2h.value


_default_engine = None


def default_engine() -> Engine:
    global _default_engine
    if _default_engine is None:
        _default_engine = Engine(0)
    return _default_engine


def compact(rows: np.ndarray, flags: np.ndarray, method: int) -> np.ndarray:
    """The reference's positions matrix (kept rows, reference columns)."""
    rows = np.ascontiguousarray(rows, dtype=np.float64)
    flags = np.ascontiguousarray(flags, dtype=np.uint8)
    n = len(flags)
    kept = _check(lib().loc_compact_host(rows.ctypes.data, flags.ctypes.data, n, method, None, 0))
    m = np.zeros(REF_COLUMNS[method] * max(kept, 1))
    _check(lib().loc_compact_host(rows.ctypes.data, flags.ctypes.data, n, method, m.ctypes.data, kept))
    # column-major N x C, as the reference's Eigen matrix
    return m[:REF_COLUMNS[method] * kept].reshape(REF_COLUMNS[method], kept).T.copy()


def find_candidates(frames: np.ndarray, pfa: float, psf_width: float, n_threads: int = 0) -> np.ndarray:
    """GLRT + adjacent-8 candidates (host), CANDIDATE_DTYPE in frame order."""
    frames = np.ascontiguousarray(frames, dtype=np.uint16)
    if frames.ndim == 2:
        frames = frames[None]
    n_frames, n_cols, n_rows = frames.shape
    cap = max(1024, n_frames * 64)
    while True:
        out = np.zeros(cap, dtype=CANDIDATE_DTYPE)
        n = _check(lib().loc_find_candidates_host(frames.ctypes.data, n_frames, n_rows, n_cols, pfa, psf_width,
                                                  n_threads, out.ctypes.data, cap))
        if n <= cap:
            return out[:n].copy()
        cap = n


def find_candidates_device(frames, pfa: float, psf_width: float, stream: int = 0):
    """GLRT + adjacent-8 candidates on the GPU for a device frame stack
    (torch int16/uint16 tensor (n_frames, n_cols, n_rows), [f, y, x]).
    Returns (device uint8 tensor of n * 40 bytes, n); identical to
    find_candidates on the same frames."""
    import torch
    n_frames, n_cols, n_rows = frames.shape
    cap = max(1024, n_frames * 64)
    while True:
        out = torch.empty(cap * CANDIDATE_DTYPE.itemsize, dtype=torch.uint8, device=frames.device)
        n = _check(lib().loc_find_candidates(C.c_void_p(frames.data_ptr()), n_frames, n_rows, n_cols, pfa,
                                             psf_width, C.c_void_p(out.data_ptr()), cap, C.c_void_p(stream)))
        if n <= cap:
            return out[:n * CANDIDATE_DTYPE.itemsize], n
        cap = n


STORAGE_FORMATS = {"int8": 2, "uint8": 3, "int16": 4, "uint16": 5, "int32": 6, "uint32": 7, "int64": 8,
                   "uint64": 9, "float32": 10, "float64": 11}


def ingest_frames(src, row_major: bool = False, stream: int = 0):
    """Camera frames (device tensor (n_frames, a, b) of any supported dtype;
    column-major frames are (n_frames, n_cols, n_rows), row-major ones
    (n_frames, n_rows, n_cols)) -> (uint16 stack as int16 tensor (n_frames,
    n_cols, n_rows), number of pixels rounded or clamped)."""
    import torch
    name = str(src.dtype).replace("torch.", "")
    if name not in STORAGE_FORMATS:
        raise LocalizerError(f"unsupported frame dtype {src.dtype}")
    src = src.contiguous()
    n_frames = src.shape[0]
    n_rows, n_cols = (src.shape[1], src.shape[2]) if row_major else (src.shape[2], src.shape[1])
    out = torch.empty((n_frames, n_cols, n_rows), dtype=torch.int16, device=src.device)
    lossy = _check(lib().loc_ingest_frames(C.c_void_p(src.data_ptr()), STORAGE_FORMATS[name], n_frames, n_rows,
                                           n_cols, int(row_major), C.c_void_p(out.data_ptr()), C.c_void_p(stream)))
    return out, lossy


def write_positions(path: str, rows: np.ndarray, flags: np.ndarray | None, method: int, header: str = "") -> int:
    """Write the kept rows as the reference's localized-positions text file
    (loc_write_positions_text); returns the number of positions written."""
    rows = np.ascontiguousarray(rows, dtype=np.float64)
    n = rows.shape[0]
    fl = None if flags is None else np.ascontiguousarray(flags, dtype=np.uint8)
    return _check(lib().loc_write_positions_text(rows.ctypes.data, fl.ctypes.data if fl is not None else None, n,
                                                 method, path.encode(), header.encode()))


class LocalizedPositions:
    """Output of fit_positions: the reference's positions matrix plus names."""

    def __init__(self, matrix: np.ndarray, method: int):
        self.matrix = matrix
        self.method = method
        self.columns = COLUMN_NAMES[method]

    def __len__(self):
        return self.matrix.shape[0]

    def column(self, name: str) -> np.ndarray:
        return self.matrix[:, self.columns.index(name)]


class FitPositions:
    """Base of the fitters (reference FitPositions, Localization.h:55-61)."""

    method = -1

    def __init__(self, initialPSFWidth: float, sigma: float = 1.0, half_width: int = 0, engine: Engine | None = None):
        self.initialPSFWidth = float(initialPSFWidth)
        self.sigma = float(sigma)
        self.half_width = int(half_width)
        self._engine = engine

    @property
    def engine(self) -> Engine:
        return self._engine if self._engine is not None else default_engine()

    def fit_positions(self, image: np.ndarray, particles: list) -> LocalizedPositions:
        """Fit one frame. Like the reference, erases rejected candidates from
        `particles` (a list of (x, y, intensity, background)) in place and
        returns the kept positions (Localization.cpp:107-212)."""
        image = np.asarray(image)
        cands = as_candidates([tuple(p)[:4] + (0, self.half_width) for p in particles]) if particles else \
            np.zeros(0, dtype=CANDIDATE_DTYPE)
        rows, flags = self.engine.fit_host(image[None] if image.ndim == 2 else image, cands, self.method,
                                           self.initialPSFWidth, self.sigma)
        keep = flags == 0
        particles[:] = [p for p, k in zip(particles, keep) if k]
        return LocalizedPositions(rows[keep, :REF_COLUMNS[self.method]], self.method)

    def fit_stack(self, frames: np.ndarray, cands):
        """Batched fit over a whole stack: (rows, flags) per candidate."""
        return self.engine.fit_host(frames, cands, self.method, self.initialPSFWidth, self.sigma)


class FitPositions_SymmetricGaussian(FitPositions):
    method = METHOD_2DGAUSS


class FitPositions_FixedWidthGaussian(FitPositions):
    method = METHOD_2DGAUSS_FIXEDWIDTH


class FitPositions_EllipsoidalGaussian(FitPositions):
    method = METHOD_2DGAUSS_ELLIPSOIDAL_ASTIGMATISM


class FitPositions_EllipsoidalGaussian_SymmetricPSF(FitPositions):
    method = METHOD_2DGAUSS_ELLIPSOIDAL


class FitPositions_MLEwG(FitPositions):
    """Maximum-likelihood fit with a Gaussian (reference FitPositions_MLEwG,
    Localization.h:126-136): takes the PSF width only."""
    method = METHOD_MLEWG

    def __init__(self, initialPSFWidth: float, half_width: int = 0, engine: Engine | None = None):
        super().__init__(initialPSFWidth, 1.0, half_width, engine)


def LocalizerFitEmitters(image_data: np.ndarray, psf_width: float, glrt_insensitivity: float) -> np.ndarray:
    """Reference DLL entry (LocalizerDLL.h:53): frames -> N x 16 positions."""
    frames = np.ascontiguousarray(image_data, dtype=np.uint16)
    n_images, n_cols, n_rows = frames.shape
    n = C.c_int()
    ptr = C.POINTER(C.c_double)()
    rc = lib().LocalizerFitEmitters(frames.ctypes.data, n_rows, n_cols, n_images, psf_width, glrt_insensitivity,
                                    C.byref(n), C.byref(ptr))
    if rc != 0:
        raise LocalizerError("LocalizerFitEmitters failed")
    m = np.ctypeslib.as_array(ptr, shape=(16 * n.value,)).copy() if n.value else np.zeros(0)
    lib().LocalizerFree(ptr)
    return m.reshape(16, n.value).T.copy()
