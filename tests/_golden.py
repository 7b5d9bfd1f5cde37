"""Loader of the golden fixtures (tests/golden/*.npz, made by make_golden.py
from the reference's own fitter and finder classes)."""
import os

import numpy as np

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("small", "uneven", "stress")


def load(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    d = {k: z[k] for k in z.files}
    d["cands"] = np.ascontiguousarray(d["cands"]).view(O.CAND_DTYPE).reshape(-1)
    d["w0"] = float(d["w0"])
    d["pfa"] = float(d["pfa"])
    d["methods"] = [int(m) for m in d["methods"]]
    return d


def all_cases():
    for name in CASES:
        d = load(name)
        for m in d["methods"]:
            yield name, m


N_EDGE_EXTRA = {"small": 9}


def n_found(name, d):
    """Number of finder candidates (the rest are hand-placed edge cases)."""
    return len(d["cands"]) - N_EDGE_EXTRA.get(name, 0)
