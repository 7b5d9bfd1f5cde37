"""The C ABI library without a GPU: it loads, exports every entry point the
public header declares, and its host-only functions behave (no device
compute is called here)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import localizer_b200 as L
from oracle import oracle as O
from tests import _golden as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            names |= set(re.findall(r"LOC_API\s+[\w\s\*]+?\b(\w+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    names = declared_symbols()
    assert "loc_fit_batch" in names and "LocalizerFitEmitters" in names
    for n in sorted(names):
        assert hasattr(lib, n), n
    assert names <= set(L._PROTOS), names - set(L._PROTOS)


def test_struct_layouts_match_header():
    assert L.CANDIDATE_DTYPE.itemsize == 40 == O.CAND_DTYPE.itemsize
    assert L.CANDIDATE_DTYPE.fields["frame"][1] == 32
    o = L.default_options()
    assert (o.max_iter, o.epsabs, o.epsrel, o.precision) == (200, 1e-4, 1e-4, 0)


def test_columns_and_errors():
    lib = L.lib()
    assert [lib.loc_reference_columns(m) for m in (0, 1, 5, 7)] == [12, 10, 16, 16]
    assert [lib.loc_output_columns(m) for m in (0, 1, 5, 7)] == [14, 12, 18, 18]
    assert [lib.loc_parameter_count(m) for m in (0, 1, 5, 7)] == [5, 4, 7, 7]
    assert lib.loc_reference_columns(3) == -4
    assert b"method" in lib.loc_last_error()
    # a fit without a context fails cleanly
    rc = lib.loc_fit_batch(None, None, 0, 8, 8, None, 0, 0, 1.3, 1.0, None, None, None, None)
    assert rc == -1


def test_compact_host_builds_reference_matrix():
    rows = np.arange(5 * 14, dtype=np.float64).reshape(5, 14)
    flags = np.array([0, 3, 0, 1, 0], dtype=np.uint8)
    m = L.compact(rows, flags, 0)
    assert m.shape == (3, 12)
    np.testing.assert_array_equal(m, rows[[0, 2, 4], :12])


@pytest.mark.parametrize("name", G.CASES)
def test_host_finder_matches_reference_finder(name):
    g = G.load(name)
    c = L.find_candidates(g["frames"], g["pfa"], g["w0"], n_threads=2)
    ref = g["cands"][:G.n_found(name, g)]
    assert len(c) == len(ref)
    for k in ("x", "y", "intensity", "background", "frame"):
        assert np.array_equal(c[k], ref[k]), k


def test_async_host_fit_checks_arrays_before_any_device_work():
    """Engine.fit_host_async refuses buffers that do not match the call
    (column count of the method, dtypes, contiguity) before the library
    touches a device, so the checks run without a GPU."""
    eng = object.__new__(L.Engine)   # no context: every call below must fail first
    eng._h = C.c_void_p()
    eng._inflight = []
    frames = np.zeros((1, 16, 16), np.uint16)
    cands = np.zeros(3, L.CANDIDATE_DTYPE)
    ncol = L.lib().loc_output_columns(0)
    good_out, good_flags = np.zeros((3, ncol)), np.zeros(3, np.uint8)
    bad = [
        (frames, cands, np.zeros((3, ncol - 1)), good_flags),             # wrong column count
        (frames, cands, np.zeros((3, ncol), np.float32), good_flags),     # wrong row dtype
        (frames, cands, good_out, np.zeros(2, np.uint8)),                 # wrong flag count
        (frames, cands[::-1].copy().view(np.uint8).view(np.float64), good_out, good_flags),  # not candidates
        (np.zeros((1, 16, 32), np.uint16)[:, :, ::2], cands, good_out, good_flags),          # not contiguous
    ]
    for fr, cd, out, fl in bad:
        with pytest.raises(L.LocalizerError):
            eng.fit_host_async(fr, cd, 0, 1.3, 1.0, out, fl)
    assert eng._inflight == []
