"""The Python ctypes mirrors of the public structs (loc_options, loc_stats,
loc_candidate) have the C header's sizes and field offsets: a small C
program compiled against include/localizer_b200.h prints them."""
import ctypes as C
import os
import shutil
import subprocess
import tempfile

import pytest

import localizer_b200 as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _c_layout(struct, fields):
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "localizer_b200.h"', "int main(void) {",
           f'  printf("%zu\\n", sizeof({struct}));']
    src += [f'  printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    src += ["  return 0;", "}"]
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write("\n".join(src))
        subprocess.run(["gcc", "-std=c11", "-I" + os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    return [int(x) for x in out]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
@pytest.mark.parametrize("cls,struct", [(L.Options, "loc_options"), (L.Stats, "loc_stats")])
def test_ctypes_mirror_matches_header(cls, struct):
    names = [n for n, _ in cls._fields_]
    got = _c_layout(struct, names)
    assert got[0] == C.sizeof(cls), (struct, got[0], C.sizeof(cls))
    for n, off in zip(names, got[1:]):
        assert getattr(cls, n).offset == off, (struct, n)


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_candidate_dtype_matches_header():
    names = list(L.CANDIDATE_DTYPE.names)
    got = _c_layout("loc_candidate", names)
    assert got[0] == L.CANDIDATE_DTYPE.itemsize
    for n, off in zip(names, got[1:]):
        assert L.CANDIDATE_DTYPE.fields[n][1] == off, n
