"""Learned start proposal: the network's kernels against the numpy oracle,
and what the trained network gains the fit.

CPU: the oracle's backward pass against finite differences of its forward
pass, and its BF16 rounding. GPU: the tcgen05 forward pass and the
CUDA-core backward pass against the oracle on the same windows and weights
(relative L2 error per weight tensor, tolerance below), training on the GPU
lowers the loss, and a trained network warm-starts the fit with fewer
solver iterations at the accuracy of the cold fit.
"""
import numpy as np
import pytest

import localizer_b200 as L
from oracle import oracle as O
from oracle import proposal_ref as R

# forward outputs and gradients: relative L2 error against the oracle, which
# rounds the same values to BF16; what remains is FP32 vs FP64 accumulation
# and the rare activation that rounds to the other side of a BF16 step
FWD_RTOL = 2e-3
GRAD_RTOL = 5e-3


def _labels(rng, n, nout):
    cols = {0: rng.uniform(200, 900, n), 1: rng.uniform(1.0, 2.2, n), 2: rng.uniform(-1, 1, n),
            3: rng.uniform(-1, 1, n), 4: rng.uniform(-0.3, 0.3, n), 5: rng.uniform(50, 200, n)}
    roles = R.roles(nout)
    return np.column_stack([cols[r] for r in roles]).astype(np.float32)


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    for nout in (5, 7):
        w = rng.normal(0, 0.3, R.weight_count(nout))
        win = rng.integers(50, 900, size=(4, 121)).astype(np.float64)
        lab = _labels(rng, 4, nout)
        lam = rng.uniform(0.5, 2.0, nout)
        _, g = R.loss_and_grad(w, win, lab, lam, nout, bf16_round=False)
        h = 1e-6
        for a, b in R.segments(nout).values():
            for i in rng.choice(np.arange(a, b), 3, replace=False):
                wp, wm = w.copy(), w.copy()
                wp[i] += h
                wm[i] -= h
                fd = (R.loss_and_grad(wp, win, lab, lam, nout, False)[0] -
                      R.loss_and_grad(wm, win, lab, lam, nout, False)[0]) / (2 * h)
                assert abs(fd - g[i]) <= 1e-3 * max(abs(fd), abs(g[i])) + 1e-6, (nout, i, fd, g[i])


def test_oracle_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0], dtype=np.float32)
    r = R.bf16(x)
    # 1 + 2^-8 is halfway between BF16 neighbours 1 and 1 + 2^-7: ties to even
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12 and r[4] == 0.0


@pytest.fixture(scope="module")
def gpu():
    import torch
    from localizer_b200 import proposal as P
    return torch, P


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.gpu
@pytest.mark.parametrize("method", [0, 7])
def test_forward_matches_oracle(gpu, method):
    torch, P = gpu
    net = P.Proposal(method, 0, seed=3)
    rois = P.synth_rois(700, elliptic=method == 7, seed=11)
    out, stat = net.forward(rois, with_stat=True)
    net.status()
    win = rois.cpu().numpy().view(np.uint16)
    ref, cache = R.forward(net.weights().astype(np.float64), win, net.nout)
    assert _rel(out.cpu().numpy(), ref) < FWD_RTOL
    st = stat.cpu().numpy()
    np.testing.assert_allclose(st[:, 0], cache["b0"], rtol=1e-5)
    np.testing.assert_allclose(st[:, 1], cache["s0"], rtol=1e-5)
    # gathered rows equal the same windows run in place
    idx = torch.tensor(np.random.default_rng(1).permutation(700)[:333].astype(np.int32), device="cuda")
    out_g = net.forward(rois, index=idx)
    np.testing.assert_allclose(out_g.cpu().numpy(), out.cpu().numpy()[idx.cpu().numpy()], rtol=0, atol=1e-6)
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("method", [0, 7])
def test_gradient_matches_oracle(gpu, method):
    torch, P = gpu
    net = P.Proposal(method, 0, seed=5)
    rng = np.random.default_rng(2)
    n = 500
    rois = P.synth_rois(n, elliptic=method == 7, seed=12)
    lab = _labels(rng, n, net.nout)
    lam = rng.uniform(0.5, 2.0, net.nout).astype(np.float32)
    g, loss = net.gradient(rois, torch.from_numpy(lab).cuda(), lam)
    net.status()
    win = rois.cpu().numpy().view(np.uint16)
    ref_loss, ref_g = R.loss_and_grad(net.weights().astype(np.float64), win, lab.astype(np.float64), lam, net.nout)
    assert abs(loss - ref_loss) <= 1e-3 * abs(ref_loss)
    gg = g.cpu().numpy()
    for name, (a, b) in R.segments(net.nout).items():
        assert _rel(gg[a:b], ref_g[a:b]) < GRAD_RTOL, name
    net.close()


@pytest.mark.gpu
def test_training_lowers_loss_and_warm_start_saves_iterations(gpu):
    torch, P = gpu
    from localizer_b200 import synth
    net, rep = P.train(method=0, n_rois=400_000, epochs=6, batch=2048, seed=21)
    assert rep["loss_last_epoch"] < 0.5 * rep["loss_initial"], rep
    assert rep["loss_last_epoch"] <= 1.05 * rep["loss_first_epoch"], rep
    assert rep["holdout_pos_median_px"] < 0.1, rep
    # warm start on the small golden-style workload: symmetric PSF, method 0
    w = synth.scaled(synth.workloads()["small"], 48, seed=4242)
    frames, _ = synth.make(w)
    cands = L.find_candidates(frames, 30.0, w.w0)
    eng = L.Engine(0)
    cold_rows, cold_flags = eng.fit_host(frames, cands, 0, w.w0)
    cold = eng.stats()
    opts = L.default_options(proposal=net.handle.value)
    warm_rows, warm_flags = eng.fit_host(frames, cands, 0, w.w0, options=opts)
    warm = eng.stats()
    net.status()
    assert warm["fits_warm"] > 0.5 * warm["fits"], warm
    # warm fits need fewer solver iterations than the reference start
    warm_its = warm["iterations"] / warm["fits"]
    cold_its = cold["iterations"] / cold["fits"]
    assert warm_its < 0.95 * cold_its, (warm_its, cold_its)
    # results against the FP64 oracle's cold fits
    ref, ref_flags, _, _ = O.fit(frames, cands, 0, w.w0, nthreads=8)
    kept_ref = ref_flags == 0
    kept = warm_flags == 0
    assert np.mean(kept == kept_ref) >= 0.998
    both = kept & kept_ref & (ref[:, -1] != 1)
    err = np.abs(warm_rows[both][:, 3:5] - ref[both][:, 3:5]).max(axis=1)
    assert np.mean(err < 1e-3) >= 0.995, np.mean(err < 1e-3)
    eng.close()
    net.close()
