"""Learned start proposal: training and use (host side).

The network and its training kernels are in csrc/loc_proposal.cu; this module
drives them through the C ABI:

* ``synth_rois`` draws 11 x 11 training windows from the fit's own forward
  model on the GPU (loc_synth_rois);
* ``label_rois`` labels them with the plain LM fit (loc_fit_batch on the
  windows as 11 x 11 frames, one candidate at the centre, ROI half-width 5),
  so the network learns to predict where the solver will end;
* ``train`` runs Adam over shuffled batches (loc_proposal_train_step: the
  tcgen05 forward pass, the CUDA-core backward pass and the optimiser, all on
  the GPU) and reports a held-out loss and parameter errors;
* ``Proposal`` is the handle passed to a fit as ``Options.proposal``.

There is no counterpart in the reference, which starts every fit from the
finder's centroid and the PSF width (Localization.cpp:122-142, 301-321,
466-491).
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import CANDIDATE_DTYPE, Engine, LocalizerError, _check, default_options, lib

# parameter roles per output: 0 amplitude, 1 width, 2 x, 3 y, 4 correlation, 5 offset
ROLES = {4: [0, 2, 3, 5], 5: [0, 1, 2, 3, 5], 7: [0, 1, 1, 2, 3, 4, 5]}
NOUT = {0: 5, 1: 4, 5: 7, 7: 7}
SIGMA_REF = 1.5
WINDOW = 11


class Proposal:
    """One proposal network (loc_proposal) on one device."""

    def __init__(self, method: int, device: int = 0, seed: int = 0):
        self.method = method
        self.nout = NOUT[method]
        self.device = device
        self._h = C.c_void_p()
        _check(lib().loc_proposal_create(C.byref(self._h), device, method, seed))
        self.n_weights = _check(lib().loc_proposal_weight_count(method))

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().loc_proposal_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def weights(self) -> np.ndarray:
        w = np.zeros(self.n_weights, dtype=np.float32)
        _check(lib().loc_proposal_get_weights(self._h, w.ctypes.data, self.n_weights))
        return w

    def set_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, dtype=np.float32)
        if w.size != self.n_weights:
            raise LocalizerError(f"expected {self.n_weights} weights, got {w.size}")
        _check(lib().loc_proposal_set_weights(self._h, w.ctypes.data, self.n_weights))

    def forward(self, rois, index=None, with_stat=False, stream: int = 0):
        """Raw head outputs (n, P) for a (N, 121) device window stack."""
        import torch
        n = len(index) if index is not None else rois.shape[0]
        out = torch.empty((n, self.nout), dtype=torch.float32, device=rois.device)
        stat = torch.empty((n, 2), dtype=torch.float32, device=rois.device) if with_stat else None
        _check(lib().loc_proposal_forward(self._h, C.c_void_p(rois.data_ptr()),
                                          C.c_void_p(index.data_ptr() if index is not None else 0), n,
                                          C.c_void_p(out.data_ptr()),
                                          C.c_void_p(stat.data_ptr() if stat is not None else 0), C.c_void_p(stream)))
        return (out, stat) if with_stat else out

    def gradient(self, rois, labels, lam, index=None, stream: int = 0):
        """(gradient in the flat weight layout, mean loss) over a batch."""
        import torch
        n = len(index) if index is not None else rois.shape[0]
        g = torch.empty(self.n_weights, dtype=torch.float32, device=rois.device)
        lam = np.ascontiguousarray(lam, dtype=np.float32)
        loss = C.c_float()
        _check(lib().loc_proposal_gradient(self._h, C.c_void_p(rois.data_ptr()),
                                           C.c_void_p(index.data_ptr() if index is not None else 0), n,
                                           C.c_void_p(labels.data_ptr()), lam.ctypes.data, C.c_void_p(g.data_ptr()),
                                           C.byref(loss), C.c_void_p(stream)))
        return g, loss.value

    def train_step(self, rois, labels, lam, lr: float, index=None, stream: int = 0, want_loss=True) -> float:
        n = len(index) if index is not None else rois.shape[0]
        lam = np.ascontiguousarray(lam, dtype=np.float32)
        loss = C.c_float()
        _check(lib().loc_proposal_train_step(self._h, C.c_void_p(rois.data_ptr()),
                                             C.c_void_p(index.data_ptr() if index is not None else 0), n,
                                             C.c_void_p(labels.data_ptr()), lam.ctypes.data, lr,
                                             C.byref(loss) if want_loss else None, C.c_void_p(stream)))
        return loss.value

    def status(self):
        _check(lib().loc_proposal_status(self._h))


def synth_rois(n: int, elliptic: bool, seed: int, truth: bool = False, stream: int = 0):
    """n synthetic 11 x 11 windows on the GPU, int16 tensor (n, 121) holding
    uint16 counts; optionally the (n, 6) truth of the central emitter."""
    import torch
    rois = torch.empty((n, WINDOW * WINDOW), dtype=torch.int16, device="cuda")
    tr = torch.empty((n, 6), dtype=torch.float32, device="cuda") if truth else None
    _check(lib().loc_synth_rois(C.c_void_p(rois.data_ptr()), n, int(elliptic), seed,
                                C.c_void_p(tr.data_ptr() if tr is not None else 0), C.c_void_p(stream)))
    return (rois, tr) if truth else rois


def label_rois(rois, method: int, w0: float = 1.5, engine: Engine | None = None):
    """Plain LM fit of every window (the window as an 11 x 11 frame, one
    candidate at the centre pixel, ROI half-width 5). Returns labels (n, P)
    float32 on the device, positions relative to the window centre, and a
    bool mask of the windows whose fit was kept."""
    import torch
    eng = engine or Engine(rois.device.index or 0)
    n = rois.shape[0]
    nout = NOUT[method]
    cands = np.zeros(n, dtype=CANDIDATE_DTYPE)
    r = rois.to(torch.int32) & 0xFFFF
    hi = r.max(dim=1).values.float().cpu().numpy()
    lo = r.min(dim=1).values.float().cpu().numpy()
    cands["x"] = 5.0
    cands["y"] = 5.0
    cands["intensity"] = hi - lo
    cands["background"] = lo
    cands["frame"] = np.arange(n, dtype=np.int32)
    cands["half_width"] = 5
    d_cands = torch.from_numpy(cands.view(np.uint8)).cuda(rois.device)
    ncol = _check(lib().loc_output_columns(method))
    out = torch.empty((n, ncol), dtype=torch.float64, device=rois.device)
    flags = torch.empty(n, dtype=torch.uint8, device=rois.device)
    params = torch.empty((n, nout), dtype=torch.float32, device=rois.device)
    opts = default_options(max_half_width=5, d_params_out=params.data_ptr())
    eng.fit_device(rois.data_ptr(), n, WINDOW, WINDOW, d_cands.data_ptr(), n, method, w0, 1.0, out.data_ptr(),
                   flags.data_ptr(), 0, opts)
    eng.sync(0)
    labels = params.clone()
    roles = ROLES[nout]
    labels[:, roles.index(2)] -= 5.0
    labels[:, roles.index(3)] -= 5.0
    valid = (flags == 0) & torch.isfinite(labels).all(dim=1)
    if engine is None:
        eng.close()
    return labels, valid


def frame_windows(frames, cands: np.ndarray, chunk: int = 1 << 18):
    """11 x 11 windows (n, 121) int16 on the device, cut from a frame stack
    (torch int16 (n_frames, n_cols, n_rows), [f, y, x]) around each
    candidate's position rounded to the nearest pixel, edges clamped: the
    windows the fit pipeline's proposal kernel sees."""
    import torch
    F, H, W = frames.shape
    flat = frames.reshape(-1)
    n = len(cands)
    out = torch.empty((n, WINDOW * WINDOW), dtype=torch.int16, device=frames.device)
    ar = torch.arange(WINDOW, device=frames.device)
    for a in range(0, n, chunk):
        c = cands[a:a + chunk]
        x0 = torch.from_numpy(np.floor(c["x"] + 0.5).astype(np.int64) - 5).to(frames.device)
        y0 = torch.from_numpy(np.floor(c["y"] + 0.5).astype(np.int64) - 5).to(frames.device)
        fr = torch.from_numpy(c["frame"].astype(np.int64)).to(frames.device)
        xs = (x0[:, None] + ar[None, :]).clamp(0, W - 1)
        ys = (y0[:, None] + ar[None, :]).clamp(0, H - 1)
        idx = fr[:, None, None] * (H * W) + ys[:, :, None] * W + xs[:, None, :]
        out[a:a + len(c)] = torch.take(flat, idx.reshape(len(c), -1))
    return out


def frame_labels(frames, cands: np.ndarray, method: int, w0: float, engine: Engine | None = None):
    """Plain LM fit of the candidates on their frames; labels (n, P) with
    positions relative to the window centre (the rounded candidate
    position), and the mask of kept fits."""
    import torch
    eng = engine or Engine(frames.device.index or 0)
    F, H, W = frames.shape
    n = len(cands)
    nout = NOUT[method]
    d_cands = torch.from_numpy(np.ascontiguousarray(cands).view(np.uint8)).cuda(frames.device)
    ncol = _check(lib().loc_output_columns(method))
    out = torch.empty((n, ncol), dtype=torch.float64, device=frames.device)
    flags = torch.empty(n, dtype=torch.uint8, device=frames.device)
    params = torch.empty((n, nout), dtype=torch.float32, device=frames.device)
    rmax = int(cands["half_width"].max()) if n else 0
    opts = default_options(max_half_width=rmax, d_params_out=params.data_ptr())
    eng.fit_device(frames.data_ptr(), F, W, H, d_cands.data_ptr(), n, method, w0, 1.0, out.data_ptr(),
                   flags.data_ptr(), 0, opts)
    eng.sync(0)
    roles = ROLES[nout]
    cx = torch.from_numpy(np.floor(cands["x"] + 0.5)).float().to(frames.device)
    cy = torch.from_numpy(np.floor(cands["y"] + 0.5)).float().to(frames.device)
    labels = params.clone()
    labels[:, roles.index(2)] -= cx
    labels[:, roles.index(3)] -= cy
    valid = (flags == 0) & torch.isfinite(labels).all(dim=1)
    if engine is None:
        eng.close()
    return labels, valid


def workload_windows(n_frames: int, method: int, seed: int, pfa: float = 30.0, workload: str = "uneven"):
    """Windows cut from synthetic frames of a workload type (the batched
    uneven one by default; seeded, disjoint from the evaluation seeds),
    labelled by the plain LM fit of their candidates at the candidates' own
    ROI half-widths."""
    from . import find_candidates_device
    from . import synth
    w = synth.scaled(synth.workloads()[workload], n_frames, seed=seed)
    frames, _ = synth.make_device(w)
    raw, _ = find_candidates_device(frames, pfa, w.w0)
    cands = raw.cpu().numpy().view(CANDIDATE_DTYPE).copy()
    del raw
    cands["half_width"] = np.random.default_rng(seed + 17).choice(np.array(w.half_widths), size=len(cands))
    labels, valid = frame_labels(frames, cands, method, w.w0)
    rois = frame_windows(frames, cands)
    del frames
    return rois, labels, valid


def window_stats(rois_np: np.ndarray):
    """Border mean b0 and scale s0 of each window (the network's normalisation)."""
    w = rois_np.astype(np.float64).reshape(-1, WINDOW, WINDOW)
    border = np.ones((WINDOW, WINDOW), bool)
    border[1:-1, 1:-1] = False
    b0 = w[:, border].sum(axis=1) / 40.0
    s0 = np.maximum(w[:, 4:7, 4:7].reshape(len(w), 9).sum(axis=1) / 9.0 - b0, 10.0)
    return b0, s0


def to_targets(labels: np.ndarray, b0: np.ndarray, s0: np.ndarray, nout: int) -> np.ndarray:
    t = np.empty_like(labels, dtype=np.float64)
    for j, r in enumerate(ROLES[nout]):
        x = labels[:, j].astype(np.float64)
        t[:, j] = (np.log(np.maximum(x, 1.0) / s0) if r == 0 else
                   np.log(np.maximum(x, 0.05) / SIGMA_REF) if r == 1 else
                   (x - b0) / s0 if r == 5 else x)
    return t


def to_params(out: np.ndarray, b0: np.ndarray, s0: np.ndarray, nout: int) -> np.ndarray:
    q = np.empty_like(out, dtype=np.float64)
    for j, r in enumerate(ROLES[nout]):
        x = out[:, j].astype(np.float64)
        q[:, j] = (s0 * np.exp(np.clip(x, -8, 8)) if r == 0 else
                   SIGMA_REF * np.exp(np.clip(x, -3, 3)) if r == 1 else
                   np.clip(x, -0.9, 0.9) if r == 4 else
                   b0 + s0 * x if r == 5 else x)
    return q


def train(method: int = 7, n_rois: int = 2_000_000, epochs: int = 8, batch: int = 4096, lr: float = 2e-3,
          seed: int = 7, device: int = 0, holdout: float = 0.02, log=None, frames: int = 0,
          workload: str = "uneven"):
    """Generate, label and train. Windows: n_rois isolated synthetic windows
    (loc_synth_rois), plus, if frames > 0, the candidates' windows of that
    many synthetic frames of the named workload type (the batched uneven one
    by default). Returns (Proposal, report dict)."""
    import torch
    t0 = time.time()
    nout = NOUT[method]
    parts_r, parts_l, parts_v = [], [], []
    if n_rois > 0:
        r = synth_rois(n_rois, elliptic=method in (5, 7), seed=seed)
        lab, val = label_rois(r, method)
        parts_r.append(r); parts_l.append(lab); parts_v.append(val)
    if frames > 0:
        r, lab, val = workload_windows(frames, method, seed=100_000 + seed, workload=workload)
        parts_r.append(r); parts_l.append(lab); parts_v.append(val)
    rois = torch.cat(parts_r) if len(parts_r) > 1 else parts_r[0]
    labels = torch.cat(parts_l) if len(parts_l) > 1 else parts_l[0]
    valid = torch.cat(parts_v) if len(parts_v) > 1 else parts_v[0]
    n_rois = rois.shape[0]
    torch.cuda.synchronize()
    t_data = time.time() - t0
    idx_all = torch.nonzero(valid).flatten().to(torch.int32)
    g = torch.Generator(device="cpu").manual_seed(seed)
    perm = idx_all[torch.randperm(len(idx_all), generator=g).to(idx_all.device)]
    n_hold = max(int(len(perm) * holdout), 1)
    hold, tr = perm[:n_hold], perm[n_hold:]
    # loss weights: unit variance per target over the training labels
    rois_np = rois.cpu().numpy().view(np.uint16)
    lab_np = labels.cpu().numpy()
    b0, s0 = window_stats(rois_np)
    tr_np = tr.cpu().numpy()
    tg = to_targets(lab_np[tr_np], b0[tr_np], s0[tr_np], nout)
    lam = (1.0 / np.maximum(tg.var(axis=0), 1e-6)).astype(np.float32)
    net = Proposal(method, device, seed)
    steps_per_epoch = max(len(tr) // batch, 1)
    total = steps_per_epoch * epochs
    # loss tracked on a fixed batch of held-out windows (no weight update)
    probe = hold[:batch].contiguous()
    loss0 = net.gradient(rois, labels, lam, index=probe)[1]
    hist = []
    t1 = time.time()
    step = 0
    for ep in range(epochs):
        order = tr[torch.randperm(len(tr), generator=g).to(tr.device)]
        for k in range(steps_per_epoch):
            cur = lr * 0.5 * (1.0 + math.cos(math.pi * step / total)) + 1e-5
            net.train_step(rois, labels, lam, cur, index=order[k * batch:(k + 1) * batch].contiguous(),
                           want_loss=False)
            step += 1
        hist.append(net.gradient(rois, labels, lam, index=probe)[1])
        if log:
            log(f"[proposal] epoch {ep + 1}/{epochs} held-out loss {hist[-1]:.4f}")
    torch.cuda.synchronize()
    t_train = time.time() - t1
    net.status()
    # held-out evaluation in parameter space
    out = net.forward(rois, index=hold.contiguous()).cpu().numpy()
    h = hold.cpu().numpy()
    pred = to_params(out, b0[h], s0[h], nout)
    truth = lab_np[h]
    err = np.abs(pred - truth)
    roles = ROLES[nout]
    ix, iy = roles.index(2), roles.index(3)
    rep = {"method": method, "windows": n_rois, "labelled": int(valid.sum().item()), "epochs": epochs,
           "batch": batch, "steps": step, "data_s": t_data, "train_s": t_train,
           "train_windows_per_s": step * batch / max(t_train, 1e-9),
           "loss_initial": loss0, "loss_first_epoch": hist[0], "loss_last_epoch": hist[-1],
           "loss_probe": f"weighted squared error on {len(probe)} held-out windows after each epoch",
           "loss_weights": lam.tolist(),
           "holdout": int(len(h)),
           "holdout_pos_rms_px": float(np.sqrt(np.mean(err[:, ix] ** 2 + err[:, iy] ** 2) / 2)),
           "holdout_pos_median_px": float(np.median(np.maximum(err[:, ix], err[:, iy]))),
           "holdout_param_median_abs_err": np.median(err, axis=0).tolist()}
    return net, rep
