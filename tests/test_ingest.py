"""Frame ingest against the reference's buffer-to-image mapping
(CopyBufferToImage: column-major pixel (i, j) at i + j*n_rows, row-major at
i*n_cols + j) followed by the fit path's uint16 conversion (round to
nearest, clamp to [0, 65535], count of pixels changed)."""
import numpy as np
import pytest

import localizer_b200 as L

pytestmark = pytest.mark.gpu


def _expected(src_np, row_major):
    x = src_np.astype(np.float64)
    if row_major:                       # (f, i, j) -> (f, j, i): x fastest
        x = x.transpose(0, 2, 1)
    r = np.clip(np.rint(np.nan_to_num(x, nan=0.0)), 0, 65535)
    lossy = int(np.sum(~(r == x)))
    return r.astype(np.uint16), lossy


@pytest.mark.parametrize("dtype", ["int8", "uint8", "int16", "uint16", "int32", "uint32", "int64", "uint64",
                                   "float32", "float64"])
@pytest.mark.parametrize("row_major", [False, True])
# (3, 45, 70): an odd side, single-pixel accesses; (3, 46, 70) and (2, 130, 196):
# even sides, paired / quad accesses; all with partial 64 x 64 transpose tiles
@pytest.mark.parametrize("shape", [(3, 45, 70), (3, 46, 70), (2, 130, 196)])
def test_ingest_matches_reference_mapping(dtype, row_major, shape):
    import torch
    rng = np.random.default_rng(sum(map(ord, dtype)) * 2 + int(row_major) + shape[1])
    info = np.iinfo(dtype) if dtype.startswith(("int", "uint")) else None
    lo = max(info.min, -300) if info else -300.0
    hi = min(info.max, 70000) if info else 70000.0
    if info:
        src = rng.integers(lo, hi, size=shape, endpoint=True).astype(dtype)
    else:
        src = rng.uniform(lo, hi, size=shape).astype(dtype)
        src.flat[7] = np.nan
    d = torch.from_numpy(src).cuda()
    out, lossy = L.ingest_frames(d, row_major=row_major)
    exp, exp_lossy = _expected(src, row_major)
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint16), exp)
    assert lossy == exp_lossy


def test_uint16_column_major_is_lossless_copy():
    import torch
    src = np.random.default_rng(1).integers(0, 65536, size=(5, 64, 48), dtype=np.uint16)
    out, lossy = L.ingest_frames(torch.from_numpy(src.view(np.int16)).cuda().view(torch.uint16), row_major=False)
    assert lossy == 0
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint16), src)
