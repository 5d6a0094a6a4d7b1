"""Learned preconditioner: the network's forward pass and weight gradients against the CPU
oracle (itself pinned by finite differences), the harvested training pairs against the
screened-kinetic relation they must satisfy, and what the trained network gains in the sweep.

Tolerances: the GPU computes in FP32 with the same bfloat16-rounded weights as the float64
oracle, so outputs agree to ~1e-6 of their scale (tested at 2e-5) and the weight gradients,
sums over ~1e5 points with FP32 atomics, to 2e-4 of the largest component."""
import os
import re

import time

import numpy as np
import pytest

from oracle import lpc_oracle as L
from rsdft_develop_b200 import api, synth
from tests import npref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# ---------------------------------------------------------------- CPU: the oracle itself
def test_weight_count_matches_header():
    h = open(os.path.join(ROOT, "include", "rsdft_b200.h")).read()
    n = int(re.search(r"#define RSDFT_LPC_NWEIGHTS (\d+)", h).group(1))
    assert n == L.NW == api.LPC_NWEIGHTS == 14688


def test_bf16_round_to_nearest_even():
    # halfway cases go to the even mantissa
    x = np.array([1.0, 1 + 2.0 ** -8, 1 + 3 * 2.0 ** -8, 1 + 2.0 ** -7 + 2.0 ** -9, -2.5], np.float32)
    want = np.array([1.0, 1.0, 1 + 2.0 ** -6, 1 + 2.0 ** -7, -2.5], np.float32)
    assert np.array_equal(L.bf16_round(x), want)
    # against a second formulation: 8 significant bits by frexp and round-half-even
    y = np.random.default_rng(9).normal(size=4096).astype(np.float32) * 10.0 ** np.arange(-3, 5).repeat(512)
    m, e = np.frexp(y.astype(np.float64))
    assert np.array_equal(L.bf16_round(y), np.ldexp(np.round(m * 256.0) / 256.0, e).astype(np.float32))


def test_oracle_gradient_matches_finite_differences():
    w = L.init_weights(3)
    rng = np.random.default_rng(0)
    x = rng.normal(size=(2, 10, 10, 10))
    t = 0.5 * rng.normal(size=(2, 10, 10, 10))
    _, g = L.loss_grad(w, x, t, 4)
    idx = [0, 5, 431, 532, 7344 + 777, 7344 + 6000, L.NW - 20, L.NW - 1]
    fd = L.fd_check(w, x, t, 4, idx, h=1e-4)
    assert np.max(np.abs(g[idx] - fd)) < 1e-6 * np.max(np.abs(fd))


def test_oracle_network_is_odd():
    w = L.init_weights(4)
    x = np.random.default_rng(1).normal(size=(1, 8, 8, 8))
    assert np.max(np.abs(L.forward(w, x, True) + L.forward(w, -x, True))) == 0.0


def test_screened_target_solves_shifted_kinetic():
    prob = synth.make_problem("t0")
    n1, n2, n3 = prob.n
    tsym = L.kinetic_symbol(prob.n, prob.h, synth.fd_lap_coef(prob.md), prob.md)
    g = np.random.default_rng(2).normal(size=(2, n3, n2, n1))
    y = L.screened_target(g, tsym, 2.5)
    # np_hpsi without V_loc and projectors applies the kinetic operator T alone
    ty = npref.np_hpsi(prob, y.reshape(2, -1), nonlocal_on=False, vloc_on=False)
    assert np.max(np.abs(ty + 2.5 * y.reshape(2, -1) - 2.5 * g.reshape(2, -1))) < 1e-10 * np.max(np.abs(g))


# ---------------------------------------------------------------- GPU: kernels vs oracle
@pytest.mark.gpu
@pytest.mark.parametrize("periodic,shape", [(False, (2, 12, 20, 16)), (True, (3, 16, 16, 16)), (True, (1, 8, 10, 24))])
def test_forward_matches_oracle(periodic, shape):
    w = L.init_weights(11)
    x = np.random.default_rng(5).normal(size=shape).astype(np.float32)
    with api.BandUpdate(synth.make_problem("t0"), precision=api.PREC_MIXED) as g:
        g.lpc_set_weights(w)
        assert np.array_equal(g.lpc_get_weights(), w)
        y = g.lpc_forward(x, periodic=periodic)
    ref = L.forward(w, x.astype(np.float64), periodic)
    assert np.max(np.abs(y - ref)) < 2e-5 * np.max(np.abs(ref))


@pytest.mark.gpu
@pytest.mark.parametrize("nb,n,margin", [(2, 12, 4), (5, 16, 4), (1, 10, 2)])
def test_loss_grad_matches_oracle(nb, n, margin):
    w = L.init_weights(12)
    rng = np.random.default_rng(6)
    x = rng.normal(size=(nb, n, n, n)).astype(np.float32)
    t = (0.5 * rng.normal(size=(nb, n, n, n))).astype(np.float32)
    with api.BandUpdate(synth.make_problem("t0"), precision=api.PREC_MIXED) as g:
        g.lpc_set_weights(w)
        loss, grad = g.lpc_loss_grad(x, t, margin)
    lref, gref = L.loss_grad(w, x.astype(np.float64), t.astype(np.float64), margin)
    assert abs(loss - lref) < 1e-5 * lref
    assert np.max(np.abs(grad - gref)) < 2e-4 * np.max(np.abs(gref))


@pytest.mark.gpu
def test_harvested_pairs_satisfy_screened_relation():
    prob = synth.make_problem("t0")
    sigma, pn = 2.5, 16
    with api.BandUpdate(prob, precision=api.PREC_MIXED) as g:
        g.random_wf(7)
        g.gram_schmidt()
        g.lpc_dataset(64, pn)
        added = g.lpc_harvest(40, sigma=sigma, iters=40, seed=3)
        assert added == 40
        assert g.lpc_status()[3] == 40
        x, t = g.lpc_dataset_get(0, 40, pn)
    # t = sigma (T + sigma)^-1 x: check (T + sigma) t = sigma x where the Md-deep stencil stays
    # inside the patch (the grid is 16^3, so a 16^3 patch is one periodic image: check it whole)
    cls = type("P", (), {})
    q = cls()
    q.n, q.md, q.kin, q.is_complex = (pn, pn, pn), prob.md, prob.kin, False
    tt = npref.np_hpsi(q, t.reshape(40, -1).astype(np.float64), nonlocal_on=False, vloc_on=False)
    lhs = tt + sigma * t.reshape(40, -1)
    assert np.max(np.abs(lhs - sigma * x.reshape(40, -1))) < 2e-4 * np.max(np.abs(sigma * x))
    assert np.all(np.isfinite(x)) and np.max(np.abs(x)) > 0.1


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c0", "t1"])
def test_tensor_core_inference_matches_fp32(name):
    """The tensor-core application (BF16 activations, FP32 accumulation in TMEM) against the
    FP32 CUDA-core one and against the oracle, on full periodic bands.  BF16 activations carry
    8 significant bits, so the outputs agree to ~1e-2 of their scale (tested at 3e-2)."""
    prob = synth.make_problem(name)
    w = L.init_weights(13)
    rng = np.random.default_rng(8)
    g = rng.normal(size=(3, prob.ng)).astype(np.float32)
    with api.BandUpdate(prob, precision=api.PREC_MIXED) as gpu:
        gpu.lpc_set_weights(w)
        gpu.lpc_inference(fp32=False)
        tc = gpu.lpc_precond(g)
        gpu.lpc_inference(fp32=True)
        f32 = gpu.lpc_precond(g)
    n1, n2, n3 = prob.n
    rms = np.sqrt(np.mean(g.astype(np.float64) ** 2, axis=1))
    ref = L.forward(w, (g / rms[:, None]).reshape(3, n3, n2, n1).astype(np.float64), True).reshape(3, -1) * rms[:, None]
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(f32 - ref)) < 2e-5 * scale
    assert np.max(np.abs(tc - ref)) < 3e-2 * scale
    assert np.max(np.abs(tc - f32)) > 1e-6 * scale  # BF16 activations: a distinct computation


def _sweeps_to(prob, pc, tol, weights=None, seed=21, maxsw=300):
    with api.BandUpdate(prob, precision=api.PREC_MIXED, pc_mode=pc) as g:
        if weights is not None:
            g.lpc_set_weights(weights)
        g.init_sweep(prob.nband - prob.nband // 8)
        g.random_wf(seed)
        g.gram_schmidt()
        g.synchronize()
        t0 = time.perf_counter()
        it, esp, res = g.calc_sweep(maxsw, tol)
        _sweeps_to.last_s = time.perf_counter() - t0
        st = g.lpc_status()
    return it, esp[0, 0], res[0, 0], st


@pytest.mark.gpu
def test_trained_network_gains_over_plain_preconditioner():
    """Train on pairs harvested from the plain solver, then solve from a new start: the learned
    preconditioner must need fewer sweeps than precond_hprsdft (and far fewer than CG without
    preconditioning), reach the same eigenvalues, and stay on the learned path (no fallback).
    Wall times of both solves are printed: per sweep the network costs more than the 7-point
    preconditioner, which is why precond_hprsdft stays the default."""
    prob = synth.make_problem("c0")
    tol = 1e-8
    with api.BandUpdate(prob, precision=api.PREC_MIXED, pc_mode=api.PC_HPRSDFT) as g:
        g.init_sweep(prob.nband - prob.nband // 8)
        g.random_wf(5)
        g.gram_schmidt()
        g.lpc_init(1)
        g.lpc_dataset(4000, 16)
        for sw in range(5):
            g.lpc_harvest(800, sigma=2.5, iters=30, seed=100 + sw)
            g.calc_sweep(2)
        losses = g.lpc_train(epochs=25, batch=32, lr=2e-3)
        w = g.lpc_get_weights()
    assert losses[-1] < 0.5 * losses[0]
    n_none, e_none, _, _ = _sweeps_to(prob, api.PC_NONE, tol)
    n_plain, e_plain, _, _ = _sweeps_to(prob, api.PC_HPRSDFT, tol)
    t_plain = _sweeps_to.last_s
    n_lpc, e_lpc, r_lpc, st = _sweeps_to(prob, api.PC_LEARNED, tol, weights=w)
    t_lpc = _sweeps_to.last_s
    print(f"sweeps to res {tol}: none {n_none}, precond_hprsdft {n_plain} ({t_plain:.3f} s), learned {n_lpc} "
          f"({t_lpc:.3f} s); loss {losses[0]:.3e} -> {losses[-1]:.3e}")
    mb = prob.nband - prob.nband // 8
    assert r_lpc[:mb].max() <= tol
    assert st[1] == api.PC_LEARNED and st[2] == 0
    assert n_lpc < n_plain
    assert n_lpc <= 0.5 * n_none
    assert np.max(np.abs(e_lpc[:mb] - e_plain[:mb])) < 1e-6
