"""Localized-positions text files: byte-identical to the reference's own
writePositionsToFile (compiled from the reference sources into oracle/_ref)
for the same positions, for every method; error behaviour as the
reference's (no positions -> error)."""
import os
import tempfile

import numpy as np
import pytest

import localizer_b200 as L
from oracle import oracle as O
from tests import _golden as G


def _frame_group(g):
    cands = g["cands"]
    frames = cands["frame"]
    f = int(np.bincount(frames).argmax())          # the frame with most candidates
    c = np.ascontiguousarray(cands[frames == f]).copy()
    c["half_width"] = 0
    return c


@pytest.mark.skipif(not O.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("name,method", [("small", 0), ("small", 1), ("uneven", 7), ("uneven", 5), ("stress", 0),
                                         ("mlewg", 6)])
def test_text_file_matches_reference_writer(name, method):
    g = G.load(name)
    frames = g["frames"]
    c = _frame_group(g)
    w0 = float(g["w0"])
    with tempfile.TemporaryDirectory() as d:
        ref_path, our_path = os.path.join(d, "ref.txt"), os.path.join(d, "ours.txt")
        header = f"golden {name}, method {method}"
        n_ref = O.ref_write_positions(frames, c, method, w0, ref_path, header)
        out, kept, _, _ = O.ref_fit(frames, c, method, w0)
        ncol = L.lib().loc_output_columns(method)
        rows = np.zeros((len(c), ncol))
        rows[:, :ncol - 2] = out[:, :ncol - 2]      # the reference's columns of every candidate
        flags = (kept != 1).astype(np.uint8)
        n_ours = L.write_positions(our_path, rows, flags, method, header)
        assert n_ours == n_ref == int(kept.sum()) > 0
        assert open(our_path, "rb").read() == open(ref_path, "rb").read()


def test_writer_errors_and_all_rows():
    rows = np.zeros((3, 14))
    rows[:, 0] = [4, 4, 5]
    rows[:, 1] = [1234.5678, 1e-7, -2.5]
    rows[:, 11] = 1
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "x.txt")
        with pytest.raises(L.LocalizerError):
            L.write_positions(p, rows, np.ones(3, np.uint8), 0)
        assert L.write_positions(p, rows, None, 0, "h") == 3
        lines = open(p).read().splitlines()
        assert lines[:3] == ["Localized positions using symmetric 2D Gauss fitting", "h", "DATA FOLLOWS"]
        assert lines[4].split("\t")[:2] == ["4", "1234.57"] and lines[5].split("\t")[1] == "1e-07"
        assert len(lines) == 7
