"""Seeded synthetic single-molecule frames (host side, numpy).

Frames are uint16 stacks laid out like the reference's images: for frame f,
pixel (x, y) sits at ``f * n_rows * n_cols + x + y * n_rows`` (x fastest,
``Image`` is column-major with rows = x, reference source/Defines.h:44 and
source/FileIO.cpp:195-234). In numpy terms a stack has shape
``(n_frames, n_cols, n_rows)`` and is indexed ``stack[f, y, x]``.

Forward model: expected photons per pixel are a per-frame background plus a
sum of point-sampled 2D Gaussians ``A exp(-(dx^2/2sx^2 + dy^2/2sy^2))``;
counts are Poisson draws plus Gaussian read noise, rounded and clipped to
uint16 (gain 1). The workloads below follow the synthetic benchmark
definitions for this fitting path; no public dataset is used.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Emitters:
    frame: np.ndarray
    x: np.ndarray
    y: np.ndarray
    amplitude: np.ndarray
    sigma_x: np.ndarray
    sigma_y: np.ndarray


@dataclass
class Workload:
    name: str
    n_frames: int
    size: int
    emitters_per_frame: tuple            # (lo, hi) inclusive
    sigma: tuple                         # (lo, hi) per emitter, per axis
    symmetric: bool                      # sx == sy per emitter
    amp_median: float
    amp_logsigma: float
    amp_uniform: tuple | None            # overrides lognormal when set
    background: tuple                    # (lo, hi) per frame
    read_noise: float = 2.0
    edge: float = 5.0
    pair_fraction: float = 0.0
    pair_distance: tuple = (1.5, 3.0)
    w0: float = 1.3                      # PSF width handed to the fitter
    half_widths: tuple = (4,)            # ROI half-widths drawn per candidate
    methods: tuple = (0,)
    seed: int = 1000
    extra: dict = field(default_factory=dict)


def workloads():
    """The five synthetic workloads of this path (seed = 1000 + index)."""
    return {
        "small": Workload("small", 512, 128, (50, 50), (1.3, 1.3), True, 500.0, 0.5, None,
                          (100.0, 100.0), w0=1.3, half_widths=(4,), methods=(0,), seed=1001),
        "uneven": Workload("uneven", 10000, 256, (20, 400), (1.0, 2.0), False, 800.0, 0.5, None,
                           (50.0, 200.0), w0=1.5, half_widths=(3, 4, 5, 6), methods=(7,), seed=1002),
        "stress": Workload("stress", 5000, 256, (50, 50), (1.5, 1.5), True, 0.0, 0.0, (50.0, 200.0),
                           (150.0, 150.0), pair_fraction=0.1, w0=1.5, half_widths=(5,), methods=(0,),
                           seed=1003),
        "dense": Workload("dense", 50000, 512, (300, 1000), (1.0, 2.0), False, 800.0, 0.5, None,
                          (50.0, 200.0), w0=1.5, half_widths=(3, 4, 5, 6), methods=(0, 7), seed=1005),
    }


def scaled(w: Workload, n_frames: int, seed: int | None = None) -> Workload:
    """Same distributions, fewer frames (parity-test sized)."""
    import dataclasses
    return dataclasses.replace(w, n_frames=n_frames, seed=w.seed if seed is None else seed)


def draw_emitters(w: Workload, rng: np.random.Generator) -> Emitters:
    lo, hi = w.emitters_per_frame
    counts = rng.integers(lo, hi + 1, size=w.n_frames)
    n = int(counts.sum())
    frame = np.repeat(np.arange(w.n_frames, dtype=np.int32), counts)
    x = rng.uniform(w.edge, w.size - 1 - w.edge, size=n)
    y = rng.uniform(w.edge, w.size - 1 - w.edge, size=n)
    if w.pair_fraction > 0 and n > 1:
        # move a fraction of emitters next to their predecessor in the same frame
        idx = np.nonzero(rng.random(n) < w.pair_fraction)[0]
        idx = idx[idx > 0]
        idx = idx[frame[idx] == frame[idx - 1]]
        d = rng.uniform(*w.pair_distance, size=idx.size)
        ang = rng.uniform(0, 2 * np.pi, size=idx.size)
        x[idx] = np.clip(x[idx - 1] + d * np.cos(ang), w.edge, w.size - 1 - w.edge)
        y[idx] = np.clip(y[idx - 1] + d * np.sin(ang), w.edge, w.size - 1 - w.edge)
    if w.amp_uniform is not None:
        amp = rng.uniform(*w.amp_uniform, size=n)
    else:
        amp = np.exp(np.log(w.amp_median) + w.amp_logsigma * rng.standard_normal(n))
    sx = rng.uniform(*w.sigma, size=n)
    sy = sx.copy() if w.symmetric else rng.uniform(*w.sigma, size=n)
    return Emitters(frame, x, y, amp, sx, sy)


def render(w: Workload, em: Emitters, rng: np.random.Generator) -> np.ndarray:
    """Render the emitters into a (n_frames, size, size) uint16 stack [f, y, x]."""
    s = w.size
    bg = rng.uniform(*w.background, size=w.n_frames)
    stack = np.empty((w.n_frames, s, s), dtype=np.uint16)
    coords = np.arange(s, dtype=np.float64)
    order = np.argsort(em.frame, kind="stable")
    starts = np.searchsorted(em.frame[order], np.arange(w.n_frames + 1))
    for f in range(w.n_frames):
        lam = np.full((s, s), bg[f])
        sel = order[starts[f]:starts[f + 1]]
        for k in sel:
            r = int(np.ceil(5 * max(em.sigma_x[k], em.sigma_y[k])))
            x0, y0 = em.x[k], em.y[k]
            xa, xb = max(0, int(x0) - r), min(s, int(x0) + r + 2)
            ya, yb = max(0, int(y0) - r), min(s, int(y0) + r + 2)
            gx = np.exp(-0.5 * ((coords[xa:xb] - x0) / em.sigma_x[k]) ** 2)
            gy = np.exp(-0.5 * ((coords[ya:yb] - y0) / em.sigma_y[k]) ** 2)
            lam[ya:yb, xa:xb] += em.amplitude[k] * np.outer(gy, gx)
        counts = rng.poisson(lam).astype(np.float64)
        counts += w.read_noise * rng.standard_normal((s, s))
        stack[f] = np.clip(np.rint(counts), 0, 65535).astype(np.uint16)
    return stack


def make(w: Workload):
    """Frames plus ground truth for a workload (deterministic in w.seed)."""
    rng = np.random.default_rng(w.seed)
    em = draw_emitters(w, rng)
    return render(w, em, rng), em


def draw_stack(w: Workload):
    """The emitters and per-frame backgrounds of a workload, drawn exactly as
    make_device draws them (same seed, same order of draws)."""
    rng = np.random.default_rng(w.seed)
    em = draw_emitters(w, rng)
    bg = rng.uniform(*w.background, size=w.n_frames).astype(np.float32)
    return em, bg


def render_frames(w: Workload, em: Emitters, bg: np.ndarray, frame_ids, seed: int) -> np.ndarray:
    """Host rendering of selected frames of a stack, (len(frame_ids), size,
    size) uint16 [f, y, x]: the same emitters and backgrounds as
    make_device's frames (draw_stack), the same forward model (point-sampled
    Gaussians within 5 sigma + 1 px of the emitter, Poisson + Gaussian read
    noise, rounded and clipped), with a host noise stream seeded per frame,
    so the pixels differ from the GPU renderer's while their distribution is
    the same. Vectorised per frame: every emitter's 23 x 23 box is summed
    into the frame with one bincount."""
    s = w.size
    order = np.argsort(em.frame, kind="stable")
    starts = np.searchsorted(em.frame[order], np.arange(w.n_frames + 1))
    off = np.arange(-11, 12, dtype=np.float64)
    out = np.empty((len(frame_ids), s, s), dtype=np.uint16)
    for k, f in enumerate(frame_ids):
        sel = order[starts[f]:starts[f + 1]]
        lam = np.full(s * s, float(bg[f]))
        if len(sel):
            x, y = em.x[sel][:, None], em.y[sel][:, None]
            sx, sy = em.sigma_x[sel][:, None], em.sigma_y[sel][:, None]
            px = np.floor(x) + off[None, :]
            py = np.floor(y) + off[None, :]
            dx, dy = px - x, py - y
            gx = np.exp(-0.5 * (dx / sx) ** 2) * ((np.abs(dx) <= 5 * sx + 1) & (px >= 0) & (px < s))
            gy = np.exp(-0.5 * (dy / sy) ** 2) * ((np.abs(dy) <= 5 * sy + 1) & (py >= 0) & (py < s))
            vals = em.amplitude[sel][:, None, None] * gy[:, :, None] * gx[:, None, :]
            idx = (np.clip(py, 0, s - 1).astype(np.int64)[:, :, None] * s +
                   np.clip(px, 0, s - 1).astype(np.int64)[:, None, :])
            lam += np.bincount(idx.ravel(), weights=vals.ravel(), minlength=s * s)
        g = np.random.default_rng([seed, int(f)])
        counts = g.poisson(lam).astype(np.float64) + w.read_noise * g.standard_normal(s * s)
        out[k] = np.clip(np.rint(counts), 0, 65535).astype(np.uint16).reshape(s, s)
    return out


def make_device(w: Workload, stream: int = 0):
    """Frames rendered on the GPU (loc_synth_frames) for the workload's
    emitters; returns (torch uint16-as-int16 tensor [f, y, x] on cuda,
    Emitters). The emitter draw is the same as make()'s; the noise stream is
    the device generator's, so frames differ from make()'s pixel by pixel."""
    import torch

    from . import lib
    em, bg = draw_stack(w)
    order = np.argsort(em.frame, kind="stable")
    packed = np.stack([em.x[order], em.y[order], em.amplitude[order], em.sigma_x[order], em.sigma_y[order]],
                      axis=1).astype(np.float32)
    starts = np.searchsorted(em.frame[order], np.arange(w.n_frames + 1)).astype(np.int32)
    d_em = torch.from_numpy(np.ascontiguousarray(packed)).cuda()
    d_st = torch.from_numpy(starts).cuda()
    d_bg = torch.from_numpy(bg).cuda()
    frames = torch.empty((w.n_frames, w.size, w.size), dtype=torch.int16, device="cuda")
    rc = lib().loc_synth_frames(frames.data_ptr(), w.n_frames, w.size, w.size, d_em.data_ptr(), d_st.data_ptr(),
                                d_bg.data_ptr(), w.read_noise, w.seed, stream)
    if rc != 0:
        raise RuntimeError(f"loc_synth_frames failed: {rc}")
    torch.cuda.synchronize()
    return frames, em
