#!/usr/bin/env python
"""Throughput of the B200 Gaussian-PSF fit engine (fits/s at the accuracy
gate) on the synthetic workloads of the per-emitter localization path.

    python bench.py [--config {1,2,3,4,5}] [--gpus N] [--steps K] [--warmup W]
                    [--impl reference]

Configurations (seeded synthetic frames, no dataset):

  5 (default, the headline): large dense -- 50,000 frames of 512 x 512 uint16
    resident in HBM (26.2 GB), 300-1000 emitters per frame, sigma_x, sigma_y
    ~ U[1, 2] px, ROI half-width per candidate in {3, 4, 5, 6} (7/9/11/13
    px), amplitude lognormal (median 800), background U[50, 200], Poisson +
    read noise; symmetric (method 0) and ellipsoidal (method 7) fits
    interleaved in alternating blocks of 5,000 frames.
  1: plain method, small -- 512 frames of 128 x 128, 50 emitters per frame,
    sigma 1.3, 9 x 9 ROI, method 0.
  2: batched uneven -- 10,000 frames of 256 x 256, 20-400 emitters per frame,
    ellipsoidal sigma U[1, 2], ROI half-width in {3, 4, 5, 6}, method 7.
  3: precision stress -- 5,000 frames of 256 x 256, amplitude U[50, 200],
    background 150, 10 % of emitters 1.5-3 px from a neighbour, sigma 1.5,
    11 x 11 ROI, method 0; the line adds the FP32 / GPU-FP64 / CPU-FP64
    precision report.
  4: learned proposal -- configuration 2's workload, with the start-proposal
    network trained on 2,000,000 synthetic 11 x 11 windows of the forward
    model instead of windows cut from frames.

Frames are rendered on the GPU from seeded emitters; candidates come from
the GPU GLRT + adjacent-8 finder. A step fits every candidate of the stack
(frames and candidates resident in HBM), one loc_fit_batch call per method.
Two arms run on the same candidates: the plain LM (the reference's start
values) and the learned-warm-start LM (a start-proposal network trained here
on the GPU, before timing, on windows of separately seeded frames of the same
workload type; warm fits it judges unreliable are re-run from the reference
start in FP64). `value` is the plain arm; both arms' fits/s, their ratio and
their accuracy against the reference's own fitter on a sample of the frames
are in the line. `e2e` runs the plain fit through the host-buffer C-ABI
calls (a stream of loc_fit_host_async calls from pinned host memory, one per
method block of frames on that method's context, uploads overlapping the
previous block's fit; where the candidates' ROIs are a small part of the
frames the calls upload only the ROIs, gathered by host threads). The CPU
reference arm (`--impl reference`) runs the reference's own fitter
(Localization.cpp compiled from the reference sources into oracle/_ref) on
all host cores, on frames of the same configuration rendered on the host,
without loading this package's native library.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fits/s at ≤1e-3 px vs FP64: learned-warm-start LM vs plain LM, 1 B200"
UNIT = "fits/s"
PFA = 30.0
# algorithmic FLOPs per ROI pixel of a Jacobian evaluation (model, analytic
# Jacobian, J^T J and J^T r accumulation) and of a trial evaluation, and per
# damped p x p Cholesky solve (p^3/3 + 2 p^2)
FLOP_J = {0: 58, 1: 46, 5: 115, 7: 115}
FLOP_F = 12
NPAR = {0: 5, 1: 4, 5: 7, 7: 7}
SM_COUNT = 148
FP32_LANES = 128
XCOL = {0: 3, 1: 2, 5: 4, 7: 4}
# DRAM bytes per fit of the whole plain-arm solver chain (every kernel of the
# step) from an ncu capture, or None while no capture of the current kernels
# exists
TRAFFIC_PER_FIT = {"bytes": 1925.0, "source": "profiles/launches_dense500_plain.md (dense workload, 500 frames)"}

# the two reference builds: strict FP64 (the yardstick) and the reference's
# own release flags (LinuxCompile.sh), which time the CPU baseline
REF_BUILD = {False: "-O2, no fast-math", True: "-O2 -ffast-math, the reference's release flags"}
# the launch-shape fields of loc_options that the tuner picks
SHAPE_KEYS = ("threads_per_fit", "tail_threads_per_fit", "level0_budget", "rerun_threads_per_fit",
              "long_rerun_threads_per_fit", "threads_per_block")

CONFIGS = {
    1: {"workload": "small", "block": 0,
        "label": "plain method, small: 512 frames 128x128 uint16, 50 emitters/frame, symmetric PSF sigma 1.3, "
                 "9x9 ROI, method 0"},
    2: {"workload": "uneven", "block": 0,
        "label": "batched uneven: 10000 frames 256x256 uint16, 20-400 emitters/frame, ellipsoidal PSF sigma "
                 "U[1,2], ROI half-width in {3,4,5,6}, method 7"},
    3: {"workload": "stress", "block": 0,
        "label": "precision stress: 5000 frames 256x256 uint16, 50 emitters/frame, amplitude U[50,200], "
                 "background 150, 10% of emitters 1.5-3 px from a neighbour, sigma 1.5, 11x11 ROI, method 0"},
    4: {"workload": "uneven", "block": 0, "train_rois": 2_000_000,
        "label": "learned proposal: network trained on 2M synthetic 11x11 forward-model windows (sigma U[1,2], "
                 "amplitude lognormal median 500, background U[50,200], Poisson + read noise, offsets U[-1,1] px) "
                 "labelled by the plain LM fit, applied as the warm start to the batched uneven workload "
                 "(10000 frames 256x256, method 7)"},
    5: {"workload": "dense", "block": 5000,
        "label": "large dense: 50000 frames 512x512 uint16 (26.2 GB resident), 300-1000 emitters/frame, "
                 "sigma U[1,2], ROI 7/9/11/13, symmetric (method 0) and ellipsoidal (method 7) fits in "
                 "alternating blocks of 5000 frames"},
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def config_workload(cfg: int, n_frames: int | None, rank: int = 0):
    """The configuration's workload (scaled to n_frames if given; each rank
    its own seed) and its method block length in frames (0: one method)."""
    from localizer_b200 import synth
    c = CONFIGS[cfg]
    base = synth.workloads()[c["workload"]]
    nf = n_frames or base.n_frames
    w = synth.scaled(base, nf, seed=base.seed + 7919 * rank)
    block = c["block"]
    if block and nf < base.n_frames:
        block = max(1, nf // 10)
    return w, block


def method_of(w, block: int, frame: np.ndarray) -> np.ndarray:
    """Fit method per candidate: the workload's method, or, for two methods,
    the first on even blocks of `block` frames and the second on odd ones."""
    if len(w.methods) == 1 or block <= 0:
        return np.full(len(frame), w.methods[0], dtype=np.int32)
    return np.where((frame // block) % 2 == 0, w.methods[0], w.methods[1]).astype(np.int32)


def assign_half_widths(w, cands):
    rng = np.random.default_rng(w.seed + 17)
    cands["half_width"] = rng.choice(np.array(w.half_widths), size=len(cands))


def make_workload(w):
    """GPU-rendered frames and GPU-found candidates of a workload."""
    import torch

    import localizer_b200 as L
    from localizer_b200 import synth
    t0 = time.time()
    frames_dev, _ = synth.make_device(w)
    t1 = time.time()
    L.find_candidates_device(frames_dev, PFA, w.w0)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    raw, n = L.find_candidates_device(frames_dev, PFA, w.w0)
    e.record()
    torch.cuda.synchronize()
    f_ms = s.elapsed_time(e)
    cands = raw.cpu().numpy().view(L.CANDIDATE_DTYPE).copy()
    del raw
    assign_half_widths(w, cands)
    finder = {"ms": f_ms, "frames_per_s": w.n_frames / (f_ms / 1e3), "candidates": int(n),
              "frame_read_gbs": frames_dev.numel() * 2 / (f_ms / 1e3) / 1e9,
              "kernels": "k_glrt, k_union, k_flatten, k_count_roots, k_assign, k_accumulate, k_emit"}
    log(f"[bench] {w.n_frames} frames rendered in {t1 - t0:.1f}s, {len(cands)} candidates found on the GPU in "
        f"{f_ms:.1f} ms")
    return frames_dev, cands, finder


def ref_fit_parallel(frames_host, cands, methods, w0, threads, fast=False):
    """The reference's own fitter (oracle/_ref; fast=True: its release-flag
    build) over the candidates, whole frames per host thread, one fitter call
    per (frame, half-width, method) group as the reference's workers make
    them. Returns (seconds, rows per method {m: (idx, rows, kept, iters)},
    threads)."""
    from oracle import oracle as O
    frame_ids = np.unique(cands["frame"])
    chunks = [c for c in np.array_split(frame_ids, threads) if len(c)]
    results = [None] * len(chunks)

    def work(k):
        m_sel = np.isin(cands["frame"], chunks[k])
        part = {}
        for m in np.unique(methods[m_sel]):
            idx = np.nonzero(m_sel & (methods == m))[0]
            out, kp, it, _ = O.ref_fit(frames_host, np.ascontiguousarray(cands[idx]), int(m), w0, fast=fast)
            part[int(m)] = (idx, out, kp == 1, it)
        results[k] = part

    t0 = time.perf_counter()
    ths = [threading.Thread(target=work, args=(k,)) for k in range(len(chunks))]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    dt = time.perf_counter() - t0
    merged = {}
    for part in results:
        for m, (idx, out, kp, it) in part.items():
            if m in merged:
                a = merged[m]
                merged[m] = (np.concatenate([a[0], idx]), np.concatenate([a[1], out]), np.concatenate([a[2], kp]),
                             np.concatenate([a[3], it]))
            else:
                merged[m] = (idx, out, kp, it)
    return dt, merged, len(chunks)


def sample_frames(n_frames, per_frame, n_target, threads):
    """Whole frames evenly spaced through the stack, about n_target fits."""
    nf = int(min(n_frames, max(threads, n_target / max(per_frame, 1.0))))
    return np.unique(np.linspace(0, n_frames - 1, nf).astype(int))


def calibrate_per_fit(frames_host, cands, methods, w0):
    """Seconds per reference fit on one host thread, from one frame's fits."""
    from oracle import oracle as O
    f0 = int(cands["frame"][0])
    sel = np.nonzero(cands["frame"] == f0)[0]
    t = time.perf_counter()
    for m in np.unique(methods[sel]):
        s = sel[methods[sel] == m]
        O.ref_fit(frames_host, np.ascontiguousarray(cands[s]), int(m), w0)
    return max((time.perf_counter() - t) / max(len(sel), 1), 1e-6)


def accuracy_report(rows, flags, ref_rows, ref_kept, ref_iters, method, rows64=None, flags64=None):
    """Flag agreement and position error against the reference fitter, with
    the tail split by class: fits the reference stopped at its 200-iteration
    cap (not converged) and fits it converged; among the converged ones
    beyond 1e-3 px, those the GPU's all-FP64 solve also misses
    (rounding-sensitive) and those only this path misses."""
    gk = flags == 0
    xi = XCOL[method]
    both = gk & ref_kept
    capped = ref_iters >= 200
    rep = {"fits": int(len(flags)), "flag_agreement": float(np.mean(gk == ref_kept)) if len(flags) else None,
           "flag_disagreements": int(np.sum(gk != ref_kept)), "jointly_kept": int(both.sum())}
    for name, cls in (("converged", both & ~capped), ("reference_capped", both & capped)):
        if cls.any():
            err = np.abs(rows[cls, xi:xi + 2] - ref_rows[cls, xi:xi + 2]).max(axis=1)
            rep[name] = {"n": int(cls.sum()), "position_within_1e-3px": float(np.mean(err < 1e-3)),
                         "n_beyond_1e-3px": int(np.sum(err >= 1e-3)), "position_max_err_px": float(err.max()),
                         "position_rms_err_px": float(np.sqrt(np.mean(err ** 2)))}
            if rows64 is not None and name == "converged":
                idx = np.nonzero(cls)[0]
                k64 = flags64[idx] == 0
                e64 = np.abs(rows64[idx, xi:xi + 2] - ref_rows[idx, xi:xi + 2]).max(axis=1)
                miss = err >= 1e-3
                rs = miss & (~k64 | (e64 >= 1e-3))
                only = miss & ~rs
                rep[name]["rounding_sensitive"] = int(rs.sum())
                rep[name]["fp32_only"] = int(only.sum())
                rep[name]["fp32_only_max_err_px"] = float(err[only].max()) if only.any() else 0.0
                rep[name]["fp64_gpu_within_1e-3px"] = float(np.mean(k64 & (e64 < 1e-3)))
        else:
            rep[name] = {"n": 0}
    return rep


def reference_arm(args):
    """The reference's own fitter on the host cores, on frames of the same
    configuration rendered on the host (numpy) from the same seeded emitters
    and candidates found by the reference's own GLRT + adjacent-8 pipeline
    (oracle/_ref); no part of the native library is loaded."""
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    from localizer_b200 import synth
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libloc_ref.so is absent"}))
        return 0
    w, block = config_workload(args.config, args.frames)
    threads = os.cpu_count() or 1
    em, bg = synth.draw_stack(w)
    per_frame = len(em.x) / w.n_frames
    budget = args.ref_budget or float(np.clip(150.0 / (args.steps + args.warmup), 2.0, 12.0))
    # calibrate on a few frames, then render the sample
    probe = synth.render_frames(w, em, bg, [0], seed=w.seed)
    pc = O.ref_find_candidates(probe, PFA, w.w0)
    pc["half_width"] = np.random.default_rng(w.seed + 17).choice(np.array(w.half_widths), size=len(pc))
    per_fit = calibrate_per_fit(probe, pc, method_of(w, block, np.zeros(len(pc), np.int64)), w.w0)
    chosen = sample_frames(w.n_frames, per_frame, budget * threads / per_fit, threads)
    t0 = time.time()
    frames = np.empty((len(chosen), w.size, w.size), dtype=np.uint16)
    found = [None] * threads
    pieces = np.array_split(np.arange(len(chosen)), threads)

    def prepare(k):
        ii = pieces[k]
        if len(ii) == 0:
            return
        frames[ii] = synth.render_frames(w, em, bg, chosen[ii], seed=w.seed)
        c = O.ref_find_candidates(np.ascontiguousarray(frames[ii]), PFA, w.w0)
        c["frame"] += ii[0]
        found[k] = c

    ths = [threading.Thread(target=prepare, args=(k,)) for k in range(threads)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    cands = np.concatenate([c for c in found if c is not None])
    assign_half_widths(w, cands)
    methods = method_of(w, block, chosen[cands["frame"]])
    log(f"[bench reference] {len(chosen)} frames rendered and {len(cands)} candidates found on the host in "
        f"{time.time() - t0:.1f}s; {budget:.1f}s of fits per step on {threads} threads")
    vals = []
    th = threads
    fast = O.ref_fast_available()
    for step in range(args.warmup + args.steps):
        dt, _, th = ref_fit_parallel(frames, cands, methods, w.w0, threads, fast=fast)
        if step >= args.warmup:
            vals.append(len(cands) / dt)
    value = float(np.mean(vals))
    sample = (f"{len(cands)} candidates of {len(chosen)} whole frames spread through the stack per step "
              f"(host-rendered from the configuration's seeded emitters); reference Localization.cpp FP64 "
              f"({REF_BUILD[fast]}) + lmsder restatement, {th} threads")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * len(cands) / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded emitters; host-rendered frames)",
            "impl": "reference",
            "config": {"workload": CONFIGS[args.config]["label"], "config": args.config, "frames": w.n_frames,
                       "sample_frames": int(len(chosen)), "sample_candidates": int(len(cands)),
                       "methods": sorted(set(int(m) for m in w.methods))},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": th, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


class Part:
    """The candidates of one method: their device copy, an engine (its own
    counters), and per-arm outputs."""

    def __init__(self, L, torch, method, idx, cands, device):
        self.method = method
        self.idx = idx
        self.cands = np.ascontiguousarray(cands[idx])
        self.n = len(idx)
        self.d_cands = torch.from_numpy(self.cands.view(np.uint8)).cuda()
        self.eng = L.Engine(device)
        self.ncol = L.lib().loc_output_columns(method)
        self.outs = {}
        self.stream = torch.cuda.Stream()

    def out(self, torch, arm):
        if arm not in self.outs:
            self.outs[arm] = (torch.empty((self.n, self.ncol), dtype=torch.float64, device="cuda"),
                              torch.empty(self.n, dtype=torch.uint8, device="cuda"))
        return self.outs[arm]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=5, choices=sorted(CONFIGS))
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=0, help="scale the configuration to this many frames")
    ap.add_argument("--e2e-steps", type=int, default=0, help="0: steps, at most 10")
    ap.add_argument("--ref-budget", type=float, default=0.0, help="seconds of CPU work per reference step")
    ap.add_argument("--ref-budget-repo", type=float, default=12.0,
                    help="seconds of CPU work of the reference sample beside the GPU arms")
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-warm", action="store_true", help="plain arm only (profiling runs)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-next-rows", action="store_true")
    ap.add_argument("--serial-parts", action="store_true", help="the method calls of a step one after the other")
    ap.add_argument("--autotune", type=int, default=1, help="1: tune the launch shapes before timing")
    ap.add_argument("--tune-sample", type=int, default=0,
                    help="candidates per method the tuner times (0: all of the method's candidates)")
    ap.add_argument("--rerun-iters", type=int, default=0,
                    help="plain arm: FP64 re-run of fits with at least this many FP32 iterations (0: library "
                         "default, < 0: off)")
    ap.add_argument("--warm-study", type=int, default=1,
                    help="1: add the warm-start study (iteration histograms, re-run limit 8/12/16)")
    ap.add_argument("--train-frames", type=int, default=3000, help="frames whose windows train each proposal")
    ap.add_argument("--train-epochs", type=int, default=8)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return reference_arm(args)

    import torch

    import localizer_b200 as L
    from localizer_b200 import dist as DI
    from localizer_b200 import proposal as PR
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    w, block = config_workload(args.config, args.frames or None, rank)
    frames_dev, cands, finder = make_workload(w)
    n = len(cands)
    methods = method_of(w, block, cands["frame"].astype(np.int64))
    parts = [Part(L, torch, int(m), np.nonzero(methods == m)[0], cands, local) for m in w.methods
             if np.any(methods == m)]
    n_frames, size = frames_dev.shape[0], frames_dev.shape[1]
    stream = torch.cuda.current_stream()
    mh = int(max(w.half_widths))

    # the proposal networks (one per method), trained on the GPU by the library's own kernels
    nets, train_rep = {}, {}
    if not args.no_warm:
        for p in parts:
            t_tr = time.time()
            n_syn = CONFIGS[args.config].get("train_rois", 0)
            net, rep = PR.train(method=p.method, n_rois=n_syn, frames=0 if n_syn else args.train_frames,
                                epochs=args.train_epochs, seed=7 + 1000 * rank, device=local,
                                workload=CONFIGS[args.config]["workload"])
            rep["wall_s"] = time.time() - t_tr
            nets[p.method], train_rep[p.method] = net, rep
            log(f"[bench] proposal for method {p.method} trained in {rep['wall_s']:.1f}s ({rep['labelled']} windows, "
                f"holdout position median {rep['holdout_pos_median_px']:.3f} px)")
    # launch shapes picked by the library's tuner on a sample of each method's
    # candidates (kept in that method's context; fields left at 0 use them)
    tuned = {}
    if args.autotune and args.precision == 0:
        for p in parts:
            k = min(p.n, args.tune_sample) if args.tune_sample > 0 else p.n
            t0 = time.time()
            tuned[p.method] = p.eng.autotune(frames_dev.data_ptr(), n_frames, size, size, p.d_cands.data_ptr(), k,
                                             p.method, w.w0, options=L.default_options(max_half_width=mh))
            tuned[p.method]["sample"] = k
            tuned[p.method]["wall_s"] = time.time() - t0
            log(f"[bench] method {p.method} tuned in {time.time() - t0:.1f}s: {tuned[p.method]}")
    arm_opts = {"plain": lambda m: L.default_options(max_half_width=mh, precision=args.precision,
                                                     rerun_iters=args.rerun_iters)}
    if not args.no_warm:
        arm_opts["warm"] = lambda m: L.default_options(max_half_width=mh, precision=args.precision,
                                                       proposal=nets[m].handle.value)
        if args.warm_study:
            # the warm-start re-run limit swept: warm fits needing more FP32
            # iterations than the limit are re-run from the reference start
            for lim in (12, 16):
                arm_opts[f"warm_limit{lim}"] = (lambda lim: lambda m: L.default_options(
                    max_half_width=mh, precision=args.precision, proposal=nets[m].handle.value,
                    warm_iter_limit=lim))(lim)
    if args.config == 3 and args.precision == 0:
        arm_opts["fp64"] = lambda m: L.default_options(max_half_width=mh, precision=1)
    opts = {arm: {p.method: f(p.method) for p in parts} for arm, f in arm_opts.items()}

    concurrent = len(parts) > 1 and not args.serial_parts

    def step(arm):
        # one call per method; with two methods the calls run on their own
        # streams (each context has its own), forked from and joined back to
        # the timing stream, so one call's long-fit tail overlaps the other
        if concurrent:
            fork = torch.cuda.Event()
            fork.record(stream)
        for p in parts:
            o, f = p.out(torch, arm)
            cs = stream
            if concurrent:
                cs = p.stream
                cs.wait_event(fork)
            p.eng.fit_device(frames_dev.data_ptr(), n_frames, size, size, p.d_cands.data_ptr(), p.n, p.method, w.w0,
                             1.0, o.data_ptr(), f.data_ptr(), cs.cuda_stream, opts[arm][p.method])
            if concurrent:
                done = torch.cuda.Event()
                done.record(cs)
                stream.wait_event(done)

    def timed(arm, steps):
        for _ in range(args.warmup):
            step(arm)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            torch.cuda.synchronize()
            start.record(stream)
            for _ in range(steps):
                step(arm)
            end.record(stream)
            torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        # whole-job throughput: summed work over the slowest rank's time
        total, ms, rate = DI.job_throughput(n * steps, start.elapsed_time(end))
        # counters and stage times of the last step, per method
        stats = {p.method: p.eng.stats() for p in parts}
        return {"value": rate, "ms": ms, "stats": stats, "clocks": clk.summary(),
                "solver_ms": float(sum(s["solver_ms"] for s in stats.values())),
                "proposal_ms": float(sum(max(s["proposal_ms"], 0.0) for s in stats.values()))}

    res = {}
    for arm in opts:
        k_steps = args.steps if arm in ("plain", "warm") else max(3, args.steps // 4)
        res[arm] = timed(arm, k_steps)
        res[arm]["steps"] = k_steps
        log(f"[bench] arm {arm}: {res[arm]['value'] / 1e6:.2f} M fits/s, {res[arm]['ms'] / k_steps:.1f} ms/step")
    value = res["plain"]["value"]
    elapsed_ms = res["plain"]["ms"]

    # roofline of the plain solver: algorithmic FLOPs / solver time vs FP32 peak
    st = res["plain"]["stats"]
    flops = 0.0
    for m, s in st.items():
        pp = NPAR[m]
        flops += s["pixels_j"] * FLOP_J[m] + s["pixels_f"] * FLOP_F + s["lambda_solves"] * (pp ** 3 / 3 + 2 * pp * pp)
    # device time of the solver: the stage events of the call, or, when the
    # method calls overlap, the whole step's device time (queue build and
    # finaliser included)
    k_ms = res["plain"]["ms"] / args.steps if concurrent else res["plain"]["solver_ms"]
    achieved = flops / (k_ms / 1e3) / 1e12
    clocks = res["plain"]["clocks"]
    peak_mhz = clocks["sm_max_mhz"] or 1965.0
    peak = SM_COUNT * FP32_LANES * 2 * peak_mhz * 1e6 / 1e12
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
    prop_roof = None
    if "warm" in res:
        bf16_peak = peaks.get("bf16_tflops", 1590.0)
        prop_ms = res["warm"]["proposal_ms"]
        tc_flops = n * 2.0 * (49 * 144 * 32 + 25 * 288 * 32)
        prop_roof = {"bound": "tensor", "kernel": "k_prop_fwd", "achieved": tc_flops / (prop_ms / 1e3) / 1e12,
                     "peak": bf16_peak, "unit": "TFLOP/s", "frac": tc_flops / (prop_ms / 1e3) / 1e12 / bf16_peak,
                     "kernel_ms": prop_ms, "windows_per_s": n / (prop_ms / 1e3),
                     "peak_source": "bf16_tflops of measured MEASURED_PEAKS.json" if peaks else "fallback 1.59 PFLOP/s"}

    # e2e through the host-buffer C ABI (pinned host memory), plain arm: one
    # loc_fit_host_async call per block of frames (the whole stack for
    # one-method configurations), closed by loc_fit_host_wait
    e2e = None
    frames_pinned = torch.empty(frames_dev.shape, dtype=torch.int16, pin_memory=True)
    frames_pinned.copy_(frames_dev)
    frames_host = frames_pinned.numpy().view(np.uint16)
    if not args.no_e2e:
        import ctypes as C
        lib = L.lib()
        # one call per method block of a two-method configuration, else one
        # call for the whole stack (split into more calls, the single-method
        # stacks measured slower: each call pays its own solver tail, and
        # blocks under 10^5 candidates upload whole frames)
        blk = block if block > 0 else n_frames
        chunks = []
        fr_all = cands["frame"]
        for b0 in range(0, n_frames, blk):
            b1 = min(n_frames, b0 + blk)
            lo, hi = np.searchsorted(fr_all, b0), np.searchsorted(fr_all, b1)
            sub = cands[lo:hi].copy()
            sub["frame"] -= b0
            m = int(method_of(w, block, np.array([b0]))[0])
            pc = torch.empty(sub.nbytes, dtype=torch.uint8, pin_memory=True)
            pc.numpy()[...] = sub.view(np.uint8)
            ncol = lib.loc_output_columns(m)
            po = torch.empty((hi - lo, ncol), dtype=torch.float64, pin_memory=True)
            pf = torch.empty(hi - lo, dtype=torch.uint8, pin_memory=True)
            chunks.append((b0, b1, lo, hi, m, pc, po, pf))
        assert np.all(np.diff(fr_all) >= 0)
        # consecutive blocks go to the methods' contexts in turn (each with
        # its own streams and staging), so one block's fit overlaps the next
        # block's gather, copies and fit; each method's tuned launch shape is
        # passed explicitly, so the rows match the device path's bit for bit
        e_ctx = [p.eng for p in parts]
        e_eng = {k: e_ctx[k % len(e_ctx)] for k in range(len(chunks))}
        e_opts = {p.method: L.default_options(max_half_width=mh, precision=args.precision,
                                              **{k: tuned[p.method][k] for k in SHAPE_KEYS if p.method in tuned})
                  for p in parts}
        fb = frames_pinned.element_size() * size * size

        def e2e_step():
            for k, (b0, b1, lo, hi, m, pc, po, pf) in enumerate(chunks):
                rc = lib.loc_fit_host_async(e_eng[k].handle, C.c_void_p(frames_pinned.data_ptr() + b0 * fb), b1 - b0,
                                            size, size, C.c_void_p(pc.data_ptr()), hi - lo, m, w.w0, 1.0,
                                            C.byref(e_opts[m]), C.c_void_p(po.data_ptr()), C.c_void_p(pf.data_ptr()))
                if rc != 0:
                    raise RuntimeError(lib.loc_last_error().decode())

        def wait():
            for eng_m in e_ctx:
                if lib.loc_fit_host_wait(eng_m.handle) != 0:
                    raise RuntimeError(lib.loc_last_error().decode())

        def host_bytes():
            hb = [eng_m.host_bytes() for eng_m in e_ctx]
            return sum(h[0] for h in hb), sum(h[1] for h in hb)

        e_steps = args.e2e_steps or min(args.steps, 10)
        # two warm-up steps: the calls use two staging slots in turn, and a
        # slot's buffers are allocated at its first use
        e2e_step()
        e2e_step()
        wait()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        dstream = torch.cuda.default_stream()
        s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        hb0 = host_bytes()
        s2.record(dstream)
        for _ in range(e_steps):
            e2e_step()
        wait()
        e2.record(dstream)
        torch.cuda.synchronize()
        hb1 = host_bytes()
        _, e_ms, e_rate = DI.job_throughput(n * e_steps, s2.elapsed_time(e2))
        # bytes the library copied (its own count: with the ROI upload only the
        # candidates' ROIs cross PCIe, gathered on the host inside the calls)
        e2e = {"value": e_rate, "unit": UNIT, "h2d_bytes_per_step": int((hb1[0] - hb0[0]) // e_steps),
               "d2h_bytes_per_step": int((hb1[1] - hb0[1]) // e_steps), "arm": "plain",
               "frame_bytes_per_step": int(frames_dev.numel() * 2),
               "call": f"loc_fit_host_async per block of {blk} frames ({len(chunks)} calls per step, one context "
                       f"per method, pinned host buffers, uploads overlapping the previous call's fit, ROI upload "
                       f"where the candidates' ROIs are under half of the frames), loc_fit_host_wait at the end",
               "steps": e_steps, "ms_per_step": e_ms / e_steps}
        # the host-buffer path gives the device path's rows
        for b0, b1, lo, hi, m, pc, po, pf in chunks:
            p = next(q for q in parts if q.method == m)
            pos = np.searchsorted(p.idx, np.arange(lo, hi))
            o, f = p.out(torch, "plain")
            sel = torch.from_numpy(pos).cuda()
            assert np.array_equal(pf.numpy(), f[sel].cpu().numpy())
            # the block's calls number frames from the block's first frame
            assert np.array_equal(po.numpy()[:, 0] + b0, o[sel].cpu().numpy()[:, 0])
            assert np.array_equal(po.numpy()[:, 1:-2], o[sel].cpu().numpy()[:, 1:-2], equal_nan=True)
        log(f"[bench] e2e: {e_rate / 1e6:.2f} M fits/s")

    # CPU reference on a bounded sample of whole frames, and the accuracy of
    # every arm there
    cpu, accuracy = None, None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as O
        if O.ref_available():
            threads = os.cpu_count() or 1
            per_fit = calibrate_per_fit(frames_host, cands, methods, w.w0)
            chosen = sample_frames(n_frames, n / n_frames, args.ref_budget_repo * threads / per_fit, threads)
            sel = np.nonzero(np.isin(cands["frame"], chosen))[0]
            dt, ref, th = ref_fit_parallel(frames_host, cands[sel], methods[sel], w.w0, threads)
            cpu = {"value": len(sel) / dt, "unit": UNIT, "cores": th, "kind": "reference",
                   "sample": f"{len(sel)} candidates of {len(chosen)} whole frames spread through the stack; "
                             f"reference Localization.cpp FP64 ({REF_BUILD[False]}) + lmsder restatement, "
                             f"{th} host threads"}
            if O.ref_fast_available():
                # the same sample through the reference's release build: the
                # baseline's value (the strict build above gives the accuracy)
                dt_f, _, _ = ref_fit_parallel(frames_host, cands[sel], methods[sel], w.w0, threads, fast=True)
                cpu["strict_fits_per_s"] = cpu["value"]
                cpu["value"] = len(sel) / dt_f
                cpu["sample"] = cpu["sample"].replace(REF_BUILD[False], REF_BUILD[True] + "; the strict build's rate "
                                                      "is strict_fits_per_s")
            accuracy = {"sample_fits": int(len(sel)), "reference": "reference fitter (FP64) on the same candidates",
                        "classes": "converged fits beyond 1e-3 px: rounding_sensitive (the GPU's all-FP64 solve "
                                   "misses too) or fp32_only"}
            # the sample's candidates once more, all in FP64 on the GPU
            fp64 = {}
            for p in parts:
                idx_s = ref[p.method][0]
                sub = np.ascontiguousarray(cands[sel[idx_s]])
                d_sub = torch.from_numpy(sub.view(np.uint8)).cuda()
                o64 = torch.empty((len(sub), p.ncol), dtype=torch.float64, device="cuda")
                f64 = torch.empty(len(sub), dtype=torch.uint8, device="cuda")
                p.eng.fit_device(frames_dev.data_ptr(), n_frames, size, size, d_sub.data_ptr(), len(sub), p.method,
                                 w.w0, 1.0, o64.data_ptr(), f64.data_ptr(), stream.cuda_stream,
                                 L.default_options(max_half_width=mh, precision=1))
                p.eng.sync(stream.cuda_stream)
                fp64[p.method] = (o64.cpu().numpy(), f64.cpu().numpy())
            for arm in res:
                accuracy[arm] = {}
                for p in parts:
                    idx_s, rrows, rkept, rit = ref[p.method]
                    gidx = sel[idx_s]                     # global candidate index
                    pos = np.searchsorted(p.idx, gidx)    # row in the part
                    o, f = p.out(torch, arm)
                    t = torch.from_numpy(pos).cuda()
                    accuracy[arm][f"method_{p.method}"] = accuracy_report(o[t].cpu().numpy(), f[t].cpu().numpy(),
                                                                          rrows, rkept, rit, p.method,
                                                                          *fp64[p.method])

    next_rows = None
    if rank == 0 and not args.no_next_rows:
        p = parts[-1]
        o, f = p.out(torch, "plain")
        next_rows = measure_next_rows(L, torch, p.eng, frames_dev, frames_host, p, w.w0, o.cpu().numpy(),
                                      f.cpu().numpy(), peaks.get("hbm_gbs", 6650.0), peaks)
    if rank == 0:
        launches = sum(int(s["kernel_launches"]) for s in st.values())
        per_method = {m: {"fits": int(s["fits"]), "iterations_per_fit": s["iterations"] / max(s["fits"], 1),
                          "fits_fp64_rerun": int(s["fits_fp64_rerun"]),
                          "fp64_rerun_fraction": s["fits_fp64_rerun"] / max(s["fits"], 1),
                          "solver_ms": s["solver_ms"]} for m, s in st.items()}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision == 0 else "f64",
                "data": "synthetic (seeded emitters, GPU-rendered Poisson+read-noise frames)",
                "config": {"workload": CONFIGS[args.config]["label"], "config": args.config,
                           "frames_per_gpu": n_frames, "candidates_per_gpu": n,
                           "methods": {str(p.method): p.n for p in parts}, "parallelism": f"dp{world}",
                           "launch_shapes": {str(m): t for m, t in tuned.items()} or "library defaults",
                           "l2": f"inputs larger than L2 ({frames_dev.numel() * 2 / 1e9:.2f} GB frames)"},
                "value_arm": "plain", "plain_lm_fits_per_s": value,
                "plain": {"per_method": per_method, "solver_ms": k_ms},
                "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                             "frac": achieved / peak,
                             "traffic": TRAFFIC_PER_FIT["bytes"] * n if TRAFFIC_PER_FIT else None,
                             "traffic_note": (f"DRAM bytes per step of the plain solver chain, "
                                              f"{TRAFFIC_PER_FIT['bytes']:.0f} B per fit from "
                                              f"{TRAFFIC_PER_FIT['source']}") if TRAFFIC_PER_FIT else
                             "no ncu capture of the current solver chain",
                             "peak_source": "nominal FP32 (148 SM x 128 lanes x 2 x max SM clock); "
                                            "no measured FP32 peak in MEASURED_PEAKS.json",
                             "kernel": "k1_lm_fit + k3_flag_class + k2_finalize (plain arm, every ROI class and "
                                       "level)", "kernel_ms": k_ms, "flops_per_step": flops,
                             "kernel_ms_source": "step device time (method calls overlap)" if concurrent else
                             "solver stage events of the call"},
                "finder": finder, "stats": st, "clocks": clocks, "e2e": e2e, "cpu_baseline": cpu,
                "accuracy": accuracy, "next_rows": next_rows, "gpu_launches": launches * args.steps}
        if "warm" in res:
            sw = res["warm"]["stats"]
            line.update({"warm_start_lm_fits_per_s": res["warm"]["value"],
                         "warm_vs_plain": res["warm"]["value"] / value,
                         "warm_ms_per_step": res["warm"]["ms"] / args.steps,
                         "warm_start": {"per_method": {m: {
                             "fits_warm": int(s["fits_warm"]), "fits_cold_fallback": int(s["fits_fp64_rerun"]),
                             "iterations_per_fit": s["iterations"] / max(s["fits"], 1),
                             "plain_iterations_per_fit": st[m]["iterations"] / max(st[m]["fits"], 1)}
                             for m, s in sw.items()},
                             "proposal_ms": res["warm"]["proposal_ms"], "solver_ms": res["warm"]["solver_ms"],
                             "training": train_rep},
                         "proposal_roofline": prop_roof, "warm_clocks": res["warm"]["clocks"]})
        if "fp64" in res:
            line["precision_report"] = precision_report(res, accuracy, parts)
        if args.warm_study and "warm" in res:
            line["warm_study"] = warm_study(L, torch, parts, opts, res, frames_dev, n_frames, size, w, stream)
        print(json.dumps(line))
    for net in nets.values():
        net.close()
    for p in parts:
        p.eng.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def warm_study(L, torch, parts, opts, res, frames_dev, n_frames, size, w, stream):
    """Cold against warm starts: FP32 iteration histograms of the plain and
    the warm fits (from the solver's per-fit diagnostics), and, per
    warm-start re-run limit, the fits/s and the fraction of fits re-run from
    the reference start."""
    bins = [1, 2, 3, 4, 5, 6, 7, 8, 10, 12, 16, 20, 32, 64, 201]
    out = {"iteration_bins": bins, "histogram": {}, "limits": {}}
    for arm in ("plain", "warm"):
        hist = np.zeros(len(bins) - 1, dtype=np.int64)
        for p in parts:
            dg = torch.zeros((p.n, 8), dtype=torch.float32, device="cuda")
            o, f = p.out(torch, arm)
            opt = opts[arm][p.method]
            saved = opt.d_diag
            opt.d_diag = dg.data_ptr()
            p.eng.fit_device(frames_dev.data_ptr(), n_frames, size, size, p.d_cands.data_ptr(), p.n, p.method, w.w0,
                             1.0, o.data_ptr(), f.data_ptr(), stream.cuda_stream, opt)
            p.eng.sync(stream.cuda_stream)
            opt.d_diag = saved
            it = dg[:, 5].cpu().numpy()
            hist += np.histogram(it[it > 0], bins=bins)[0]
        out["histogram"][arm] = hist.tolist()
    for arm, lim in (("warm", 8), ("warm_limit12", 12), ("warm_limit16", 16)):
        if arm not in res:
            continue
        s = res[arm]["stats"]
        out["limits"][str(lim)] = {"fits_per_s": res[arm]["value"],
                                   "rerun_fraction": sum(v["fits_fp64_rerun"] for v in s.values()) /
                                   max(sum(v["fits"] for v in s.values()), 1)}
    return out


def precision_report(res, accuracy, parts):
    """The precision-stress comparison: the FP32 solver (compensated by its
    FP64 re-run of decision-sensitive fits) against the GPU FP64 solver and
    the CPU FP64 reference."""
    rep = {}
    for arm in ("plain", "fp64"):
        s = res[arm]["stats"]
        rep[arm] = {"fits_per_s": res[arm]["value"],
                    "fits_fp64_rerun": int(sum(v["fits_fp64_rerun"] for v in s.values())),
                    "fp64_rerun_fraction": sum(v["fits_fp64_rerun"] for v in s.values()) /
                    max(sum(v["fits"] for v in s.values()), 1),
                    "fp64_pivot_escalations": int(sum(v["fp64_escalations"] for v in s.values())),
                    "vs_cpu_reference": accuracy.get(arm) if accuracy else None}
    return rep


def measure_next_rows(L, torch, eng, frames_dev, frames_host, part, w0, rows_plain, flags_plain, hbm_peak, peaks):
    """Throughput of the path's neighbours on the same workload, outside the
    timed region: frame ingest (row-major float32 camera frames -> the
    uint16 stack, HBM-bound at 4 + 2 B per pixel), the MLEwG fit (method 6)
    against the reference's own MLEwG on one host core, and the positions
    text writer."""
    import tempfile

    from oracle import oracle as O
    out = {}
    nf = max(1, min(frames_dev.shape[0], (2000 * 256 * 256) // (frames_dev.shape[1] * frames_dev.shape[2])))
    src = (frames_dev[:nf].to(torch.int32) & 0xFFFF).to(torch.float32).transpose(1, 2).contiguous()
    dst, lossy = L.ingest_frames(src, row_major=True)
    assert lossy == 0 and torch.equal(dst, frames_dev[:nf])
    reps = 10
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        L.ingest_frames(src, row_major=True)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    gbs = src.numel() * 6 / (ms / 1e3) / 1e9
    out["ingest"] = {"kernel": "k_ingest_rm<float>", "frames": nf, "ms_per_call": ms, "frames_per_s": nf / (ms / 1e3),
                     "achieved_gbs": gbs, "peak_gbs": hbm_peak, "frac": gbs / hbm_peak,
                     "bytes_per_pixel": 6, "check": "lossless round trip of the uint16 stack",
                     "timing": "per call, including the call's host synchronisation for the lossy count",
                     "peak_source": "hbm_gbs of measured MEASURED_PEAKS.json" if peaks else "fallback 6.65 TB/s"}
    del src, dst
    k = min(100000, part.n)
    ncol6 = L.lib().loc_output_columns(6)
    o6 = torch.empty((k, ncol6), dtype=torch.float64, device="cuda")
    f6 = torch.empty(k, dtype=torch.uint8, device="cuda")
    opt6 = L.default_options(max_half_width=int(part.cands["half_width"].max()))
    stream = torch.cuda.current_stream().cuda_stream

    def fit6():
        eng.fit_device(frames_dev.data_ptr(), frames_dev.shape[0], frames_dev.shape[2], frames_dev.shape[1],
                       part.d_cands.data_ptr(), k, 6, w0, 1.0, o6.data_ptr(), f6.data_ptr(), stream, opt6)

    fit6()
    torch.cuda.synchronize()
    a.record()
    for _ in range(3):
        fit6()
    b.record()
    torch.cuda.synchronize()
    ms6 = a.elapsed_time(b) / 3
    mlewg = {"candidates": k, "ms_per_call": ms6, "fits_per_s": k / (ms6 / 1e3)}
    if O.ref_available():
        f0 = int(part.cands["frame"][0])
        sel = np.nonzero(part.cands["frame"][:k] == f0)[0]
        t = time.perf_counter()
        rout, rkept, _, _ = O.ref_fit(frames_host, np.ascontiguousarray(part.cands[sel]), 6, w0)
        dt = time.perf_counter() - t
        g = o6[torch.from_numpy(sel).cuda()].cpu().numpy()
        gk = f6[torch.from_numpy(sel).cuda()].cpu().numpy() == 0
        rk = rkept == 1
        same = (gk == rk) & (~gk | np.all(g[:, :8] == rout[:, :8], axis=1))
        mlewg["reference_one_core"] = {"fits_per_s": len(sel) / dt, "fits": int(len(sel)),
                                       "sample": f"the {len(sel)} candidates of frame {f0}"}
        mlewg["identical_to_reference"] = float(np.mean(same))
    out["mlewg"] = mlewg
    m = min(300000, len(rows_plain))
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "positions.txt")
        t = time.perf_counter()
        kept = L.write_positions(path, rows_plain[:m], flags_plain[:m], part.method, "bench")
        dt = time.perf_counter() - t
        size = os.path.getsize(path)
    out["writer"] = {"rows": m, "kept_rows_written": int(kept), "s": dt, "rows_per_s": m / dt,
                     "mb_per_s": size / dt / 1e6, "threads": os.cpu_count()}
    return out


if __name__ == "__main__":
    sys.exit(main())
