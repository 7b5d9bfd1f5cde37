"""Generate the golden fixtures in this folder from the reference's own code.

Runs the reference's ParticleFinder_adjacent8 and FitPositions_* classes
(compiled unmodified into oracle/_ref by oracle/Makefile, linked to the
lmsder restatement) on small seeded synthetic stacks and stores frames,
candidates and the reference's output matrices, kept flags and iteration
counts. Needs the reference tree, so it runs only where it exists:

    python tests/golden/make_golden.py            # all fixtures
    python tests/golden/make_golden.py mlewg      # mlewg.npz only
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from localizer_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

CASES = [
    # name, workload, frames, w0 for the fitter, GLRT PFA, methods
    ("small", "small", 4, 1.3, 30.0, (0, 1, 5, 7)),
    ("uneven", "uneven", 2, 1.5, 30.0, (7, 5, 0, 1)),
    ("stress", "stress", 2, 1.5, 30.0, (0, 7)),
]


def edge_candidates(frames, w0, r):
    """Hand-placed candidates: inside, at and beyond the frame edges."""
    n_frames, n_cols, n_rows = frames.shape
    pts = [(r + 0.0, r + 0.0), (r - 0.01, 20.0), (20.0, r - 0.5), (n_rows - 1 - r + 0.49, 30.0),
           (n_rows - 1 - r + 0.5, 30.0), (40.0, n_cols - 1 - r + 0.2), (40.0, n_cols - r + 0.0),
           (0.0, 0.0), (n_rows - 1.0, n_cols - 1.0)]
    rows = []
    for (x, y) in pts:
        xi, yi = int(min(max(round(x), 0), n_rows - 1)), int(min(max(round(y), 0), n_cols - 1))
        v = float(frames[0, yi, xi])
        rows.append((x, y, max(v - 100.0, 1.0), 100.0, 0, r))
    return np.array(rows, dtype=O.CAND_DTYPE)


def main():
    if not O.ref_available():
        O.build()
    for name, wname, nf, w0, pfa, methods in CASES:
        w = synth.scaled(synth.workloads()[wname], nf)
        frames, em = synth.make(w)
        cands = O.candidates(frames, pfa, w0, half_widths=w.half_widths, seed=w.seed, use_ref=True)
        if name == "small":
            cands = np.concatenate([cands, edge_candidates(frames, w0, 4)])
        payload = dict(frames=frames, cands=cands.view(np.uint8).reshape(len(cands), -1), w0=w0,
                       pfa=pfa, methods=np.array(methods), truth_x=em.x, truth_y=em.y,
                       truth_frame=em.frame)
        for m in methods:
            out, kept, iters, status = O.ref_fit(frames, cands, m, w0)
            payload[f"out_{m}"] = out
            payload[f"kept_{m}"] = kept
            payload[f"iters_{m}"] = iters
            payload[f"status_{m}"] = status
            print(f"{name} method {m}: {len(cands)} candidates, {kept.sum()} kept, "
                  f"mean iterations {iters[iters >= 0].mean():.2f}")
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **payload)


def main_mlewg():
    """mlewg.npz: the reference's MLEwG fitter (FitPositions_MLEwG, method 6)
    on the small workload's frames and candidates (the Nelder-Mead minimiser
    it calls is the restatement in oracle/nmsimplex_core.c)."""
    if not O.ref_available():
        O.build()
    w = synth.scaled(synth.workloads()["small"], 4)
    frames, _ = synth.make(w)
    cands = O.candidates(frames, 30.0, 1.3, half_widths=w.half_widths, seed=w.seed, use_ref=True)
    cands = np.concatenate([cands, edge_candidates(frames, 1.3, 4)])
    out, kept, iters, status = O.ref_fit(frames, cands, 6, 1.3)
    print(f"mlewg: {len(cands)} candidates, {kept.sum()} kept, mean iterations {iters[iters >= 0].mean():.1f}")
    np.savez_compressed(os.path.join(OUT, "mlewg.npz"), frames=frames,
                        cands=cands.view(np.uint8).reshape(len(cands), -1), w0=1.3, pfa=30.0,
                        methods=np.array([6]), out_6=out, kept_6=kept, iters_6=iters, status_6=status)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "mlewg":
        main_mlewg()
    else:
        main()
        main_mlewg()
