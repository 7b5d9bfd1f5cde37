"""TEST INFRASTRUCTURE ONLY — numpy restatement of the learned start
proposal network (localizer_b200/csrc/loc_proposal.cu), used by tests/ to
check the GPU forward pass and the GPU gradients. Only tests/ may import it.

The network has no counterpart in the reference (the reference starts every
fit from the finder's centroid and the PSF width, Localization.cpp:122-142,
301-321, 466-491); this restatement follows the definition the CUDA code
documents:

  window (11 x 11, x fastest) -> normalise: b0 = mean of the 40 border
  pixels, s0 = max(mean of the central 3 x 3 - b0, 10), v = (w - b0) / s0
  conv1 3x3 (1 -> 16) + ReLU, conv2 3x3 (16 -> 32) + ReLU,
  conv3 3x3 (32 -> 32) + ReLU (valid convolutions, cross-correlation),
  linear head 800 -> P over the (channel, position) flattening.

With ``bf16=True`` the values the GPU rounds to BF16 are rounded the same way
(round to nearest even): the normalised window and the conv1 weights (conv1's
tensor-core operands), the conv2 and conv3 weights and the conv1 and conv2
activations. Everything else is FP64. The backward pass treats the rounding
as the identity (as the GPU's does) and ReLU's derivative as 1 where the
activation is positive.
"""
from __future__ import annotations

import numpy as np

KW1, KB1, KW2, KB2, KW3, KB3, KWH = 0, 144, 160, 4768, 4800, 14016, 14048
SIGMA_REF = 1.5


def weight_count(nout: int) -> int:
    return KWH + nout * 801


def nout_of(method: int) -> int:
    return {0: 5, 1: 4, 5: 7, 7: 7}[method]


def roles(nout: int):
    """0 amplitude, 1 width, 2 x, 3 y, 4 correlation, 5 offset, per output."""
    return {4: [0, 2, 3, 5], 5: [0, 1, 2, 3, 5], 7: [0, 1, 1, 2, 3, 4, 5]}[nout]


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to BF16 (nearest even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w: np.ndarray, nout: int):
    w = np.asarray(w, dtype=np.float64)
    return dict(W1=w[KW1:KB1].reshape(16, 9), b1=w[KB1:KW2], W2=w[KW2:KB2].reshape(32, 16, 9), b2=w[KB2:KW3],
                W3=w[KW3:KB3].reshape(32, 32, 9), b3=w[KB3:KWH], WH=w[KWH:KWH + nout * 800].reshape(nout, 32, 25),
                bh=w[KWH + nout * 800:KWH + nout * 801])


def normalise(windows: np.ndarray):
    """windows (n, 121) -> v (n, 11, 11), b0 (n,), s0 (n,)"""
    w = np.asarray(windows, dtype=np.float64).reshape(-1, 11, 11)
    border = np.ones((11, 11), bool)
    border[1:-1, 1:-1] = False
    b0 = w[:, border].sum(axis=1) / 40.0
    c = w[:, 4:7, 4:7].reshape(len(w), 9).sum(axis=1) / 9.0
    s0 = np.maximum(c - b0, 10.0)
    v = (w - b0[:, None, None]) / s0[:, None, None]
    return v, b0, s0


def _conv(x, W, b, out):
    """valid 3x3 cross-correlation: x (n, ci, H, H), W (co, ci, 9) -> (n, co, out, out)"""
    z = np.broadcast_to(b[None, :, None, None], (x.shape[0], W.shape[0], out, out)).copy()
    for t in range(9):
        dy, dx = divmod(t, 3)
        z += np.einsum("nchw,oc->nohw", x[:, :, dy:dy + out, dx:dx + out], W[:, :, t])
    return z


def _conv_dx(dz, W, inp):
    """input gradient of _conv: dz (n, co, out, out) -> (n, ci, inp, inp)"""
    n, co, out, _ = dz.shape
    dx = np.zeros((n, W.shape[1], inp, inp))
    for t in range(9):
        dy, dxx = divmod(t, 3)
        dx[:, :, dy:dy + out, dxx:dxx + out] += np.einsum("nohw,oc->nchw", dz, W[:, :, t])
    return dx


def _conv_dw(dz, x):
    """weight gradient of _conv: (co, ci, 9)"""
    out = dz.shape[2]
    g = np.zeros((dz.shape[1], x.shape[1], 9))
    for t in range(9):
        dy, dx = divmod(t, 3)
        g[:, :, t] = np.einsum("nohw,nchw->oc", dz, x[:, :, dy:dy + out, dx:dx + out])
    return g


def forward(w, windows, nout, bf16_round=True):
    """Raw head outputs (n, nout) and the cache for backward."""
    p = unpack(w, nout)
    rnd = bf16 if bf16_round else (lambda a: np.asarray(a, dtype=np.float64))
    v, b0, s0 = normalise(windows)
    v = rnd(v)
    z1 = _conv(v[:, None], rnd(p["W1"])[:, None, :], p["b1"], 9)
    a1 = rnd(np.maximum(z1, 0.0))
    W2, W3 = rnd(p["W2"]), rnd(p["W3"])
    z2 = _conv(a1, W2, p["b2"], 7)
    a2 = rnd(np.maximum(z2, 0.0))
    z3 = _conv(a2, W3, p["b3"], 5)
    a3 = np.maximum(z3, 0.0)
    out = np.einsum("ncp,jcp->nj", a3.reshape(len(a3), 32, 25), p["WH"]) + p["bh"]
    return out, dict(v=v, b0=b0, s0=s0, a1=a1, a2=a2, a3=a3, W2=W2, W3=W3, p=p)


def targets(labels, b0, s0, nout):
    """Parameter labels (positions relative to the window centre) -> targets."""
    lab = np.asarray(labels, dtype=np.float64)
    t = np.empty_like(lab)
    for j, r in enumerate(roles(nout)):
        x = lab[:, j]
        if r == 0:
            t[:, j] = np.log(np.maximum(x, 1.0) / s0)
        elif r == 1:
            t[:, j] = np.log(np.maximum(x, 0.05) / SIGMA_REF)
        elif r == 5:
            t[:, j] = (x - b0) / s0
        else:
            t[:, j] = x
    return t


def outputs_to_params(out, b0, s0, nout):
    """Head outputs -> parameters (positions relative to the window centre)."""
    o = np.asarray(out, dtype=np.float64)
    q = np.empty_like(o)
    for j, r in enumerate(roles(nout)):
        x = o[:, j]
        if r == 0:
            q[:, j] = s0 * np.exp(np.clip(x, -8, 8))
        elif r == 1:
            q[:, j] = SIGMA_REF * np.exp(np.clip(x, -3, 3))
        elif r == 4:
            q[:, j] = np.clip(x, -0.9, 0.9)
        elif r == 5:
            q[:, j] = b0 + s0 * x
        else:
            q[:, j] = x
    return q


def loss_and_grad(w, windows, labels, lam, nout, bf16_round=True):
    """Mean over windows of sum_j lam_j (o_j - t_j)^2 and its gradient in the
    flat weight layout."""
    out, c = forward(w, windows, nout, bf16_round)
    n = len(out)
    t = targets(labels, c["b0"], c["s0"], nout)
    lam = np.asarray(lam, dtype=np.float64)
    d = out - t
    loss = float(np.sum(lam * d * d) / n)
    dO = 2.0 * lam * d / n
    p = c["p"]
    a3 = c["a3"].reshape(n, 32, 25)
    g = np.zeros(weight_count(nout))
    g[KWH:KWH + nout * 800] = np.einsum("nj,ncp->jcp", dO, a3).ravel()
    g[KWH + nout * 800:] = dO.sum(axis=0)
    dz3 = np.einsum("nj,jcp->ncp", dO, p["WH"]) * (a3 > 0)
    dz3 = dz3.reshape(n, 32, 5, 5)
    g[KW3:KB3] = _conv_dw(dz3, c["a2"]).ravel()
    g[KB3:KWH] = dz3.sum(axis=(0, 2, 3))
    dz2 = _conv_dx(dz3, c["W3"], 7) * (c["a2"] > 0)
    g[KW2:KB2] = _conv_dw(dz2, c["a1"]).ravel()
    g[KB2:KW3] = dz2.sum(axis=(0, 2, 3))
    dz1 = _conv_dx(dz2, c["W2"], 9) * (c["a1"] > 0)
    g[KW1:KB1] = _conv_dw(dz1, c["v"][:, None]).ravel()
    g[KB1:KW2] = dz1.sum(axis=(0, 2, 3))
    return loss, g


def segments(nout):
    """Named weight segments of the flat layout."""
    return {"W1": (KW1, KB1), "b1": (KB1, KW2), "W2": (KW2, KB2), "b2": (KB2, KW3), "W3": (KW3, KB3),
            "b3": (KB3, KWH), "WH": (KWH, KWH + nout * 800), "bh": (KWH + nout * 800, KWH + nout * 801)}
