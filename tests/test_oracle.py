"""Pins the CPU FP64 oracle (oracle/) before it is trusted as the GPU parity checker.

The reference ships no golden vectors for this path (no test suite; test_hpsi2 prints
timings only), so the oracle is pinned by:
  * exact known answers: the Md=6 FD rationals of src/fd_module.f90:18-54, the plane-wave
    dispersion of the periodic FD operator (real and k-shifted via zcoef_kin), and the
    eigenvalues of the dense kinetic matrix (d_construct_matrix_kinetic_sol);
  * a second, independent numpy formulation of every routine (tests/npref.py);
  * committed golden fixtures (tests/golden/, made by tests/golden/make_golden.py).
"""
import dataclasses
import os
from fractions import Fraction

import numpy as np
import pytest

from rsdft_develop_b200 import synth
from tests import npref

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _prob_novloc(name):
    p = synth.make_problem(name)
    return dataclasses.replace(p, vloc=np.zeros_like(p.vloc))


def test_fd_rationals_md6():
    lap = synth.fd_lap_coef(6)
    exact = [Fraction(-5369, 1800), Fraction(12, 7), Fraction(-15, 56), Fraction(10, 189),
             Fraction(-1, 112), Fraction(2, 1925), Fraction(-1, 16632)]
    for m, fr in enumerate(exact):
        assert lap[6 + m] == pytest.approx(float(fr), rel=1e-14, abs=1e-16)
        assert lap[6 - m] == lap[6 + m]
    assert abs(lap.sum()) < 1e-13


def test_fd_nabla_weights():
    nab = synth.fd_nab_coef(6)
    # antisymmetric first-derivative weights: sum_m m*w_m over m>0 with sign = 1/2
    s = sum(m * nab[6 + m] for m in range(1, 7))
    assert s == pytest.approx(0.5, rel=1e-13)
    # exact for polynomials: sum_m m^(2q+1) w_m = 0 for q = 1..5
    for q in range(1, 6):
        assert abs(sum(m ** (2 * q + 1) * nab[6 + m] for m in range(1, 7))) < 1e-9


@pytest.mark.parametrize("md", [4, 6])
def test_fd_laplacian_polynomial_exactness(md):
    lap = synth.fd_lap_coef(md)
    m = np.arange(-md, md + 1)
    assert np.sum(lap * m ** 2) == pytest.approx(2.0, rel=1e-12)
    for q in range(2, md + 1):
        assert abs(np.sum(lap * m.astype(float) ** (2 * q))) < 1e-8 * q ** (2 * q)


def test_oracle_plane_wave_dispersion(oracle_mod):
    prob = _prob_novloc("t0")
    o = oracle_mod.Oracle(prob, nonlocal_on=False)
    n = prob.n[0]
    idx = np.arange(prob.ng)
    i1, i2, i3 = idx % n, (idx // n) % n, idx // (n * n)
    for (m1, m2, m3) in [(0, 0, 0), (1, 0, 0), (2, 3, 1), (5, 7, 8)]:
        th = 2 * np.pi * (m1 * i1 + m2 * i2 + m3 * i3) / n
        psi = np.cos(th)
        h = o.hpsi(psi[None, :])[0]
        e = npref.dispersion(prob, m1, m2, m3).real
        assert np.allclose(h, e * psi, atol=1e-11 * max(1.0, abs(e)))
    # small-theta accuracy of the 12th-order stencil against 1/2 |G|^2
    e1 = npref.dispersion(prob, 1, 0, 0).real
    G = 2 * np.pi / prob.cfg.L
    assert e1 == pytest.approx(0.5 * G * G, rel=1e-9)


def test_oracle_kpoint_dispersion(oracle_mod):
    prob = dataclasses.replace(synth.make_problem("tk"), vloc=np.zeros(synth.make_problem("tk").ng))
    n = prob.n[0]
    idx = np.arange(prob.ng)
    i1, i2, i3 = idx % n, (idx // n) % n, idx // (n * n)
    for k in (0, 3, 7):
        o = oracle_mod.Oracle(prob, k=k, nonlocal_on=False)
        for (m1, m2, m3) in [(0, 0, 0), (1, 2, 0), (3, 1, 5)]:
            psi = np.exp(2j * np.pi * (m1 * i1 + m2 * i2 + m3 * i3) / n)
            h = o.hpsi(psi[None, :])[0]
            e = npref.dispersion(prob, m1, m2, m3, k)
            assert abs(e.imag) < 1e-12
            assert np.allclose(h, e.real * psi, atol=1e-10)
    # dispersion approximates 1/2 |k + G|^2 for small G
    kc = prob.kcart[7]
    G = 2 * np.pi / prob.cfg.L
    e = npref.dispersion(prob, 1, 0, 0, 7).real
    assert e == pytest.approx(0.5 * ((kc[0] + G) ** 2 + kc[1] ** 2 + kc[2] ** 2), rel=1e-6)


def test_oracle_dense_kinetic_matrix_eigenvalues(oracle_mod):
    cfg = synth.get_config("t0", n=8, natom=1, n_gauss=1)
    prob = dataclasses.replace(synth.make_problem(cfg), vloc=np.zeros(8 ** 3))
    o = oracle_mod.Oracle(prob, nonlocal_on=False)
    H = o.dense_kinetic()
    assert np.allclose(H, H.T, atol=1e-12)
    ev = np.linalg.eigvalsh(H)
    ana = sorted(npref.dispersion(prob, a, b, c).real for a in range(8) for b in range(8) for c in range(8))
    assert np.allclose(ev, ana, atol=1e-10)
    # the dense matrix and the stencil agree on a random vector
    x = np.random.default_rng(0).normal(size=(1, prob.ng))
    assert np.allclose(o.hpsi(x)[0], H @ x[0], atol=1e-11)


@pytest.mark.parametrize("name", ["t0", "t1", "c0"])
def test_oracle_hpsi_matches_numpy(oracle_mod, name):
    prob = synth.make_problem(name)
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(3, 3, prob.ng)
    a = o.hpsi(psi)
    b = npref.np_hpsi(prob, psi)
    assert np.max(np.abs(a - b)) < 1e-10 * np.max(np.abs(b))


def test_oracle_hpsi_complex_matches_numpy(oracle_mod):
    prob = synth.make_problem("tk")
    for k in (0, 5):
        o = oracle_mod.Oracle(prob, k=k)
        psi = synth.random_wavefunctions(4, 2, prob.ng, is_complex=True, kindex=k)
        a = o.hpsi(psi)
        b = npref.np_hpsi(prob, psi, k)
        assert np.max(np.abs(a - b)) < 1e-10 * np.max(np.abs(b))
        # Hermiticity: <a|H b> = conj(<b|H a>)
        ha = o.hpsi(psi[:1]); hb = o.hpsi(psi[1:2])
        assert abs(np.vdot(psi[0], hb[0]) - np.conj(np.vdot(psi[1], ha[0]))) < 1e-9 * abs(np.vdot(psi[0], hb[0]))


def test_oracle_reference_form_dij(oracle_mod):
    cfg = synth.get_config("t1", reference_form=True)
    prob = synth.make_problem(cfg)
    lm = set(zip(prob.lmap, prob.mmap))
    for (l1, l2) in prob.pairs:
        assert (prob.lmap[l1 - 1], prob.mmap[l1 - 1]) == (prob.lmap[l2 - 1], prob.mmap[l2 - 1])
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(5, 2, prob.ng)
    assert np.allclose(o.hpsi(psi), npref.np_hpsi(prob, psi), rtol=0, atol=1e-10 * 100)


def test_oracle_precond_matches_numpy(oracle_mod):
    prob = synth.make_problem("t0")
    o = oracle_mod.Oracle(prob)
    g = synth.random_wavefunctions(9, 2, prob.ng)
    a = o.precond(g)
    for b in range(2):
        assert np.allclose(a[b], npref.np_precond(prob, g[b]), atol=1e-11 * np.abs(a[b]).max())


def test_oracle_gram_schmidt_is_qr(oracle_mod):
    prob = synth.make_problem("c0")
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(11, prob.nband, prob.ng)
    q = o.gram_schmidt(psi)
    S = q @ q.T * prob.dV
    assert np.max(np.abs(S - np.eye(prob.nband))) < 1e-12
    # same Q as Cholesky QR: psi = R^T q with R upper triangular, positive diagonal
    R = np.linalg.cholesky(psi @ psi.T * prob.dV).T
    q2 = np.linalg.solve(R.T, psi)
    assert np.max(np.abs(q - q2)) < 1e-9 * np.abs(q).max()


def test_oracle_subspace_diag(oracle_mod):
    prob = synth.make_problem("t1")
    o = oracle_mod.Oracle(prob)
    psi = o.gram_schmidt(synth.random_wavefunctions(12, prob.nband, prob.ng))
    u, esp = o.subspace_diag(psi)
    H = psi @ npref.np_hpsi(prob, psi).T * prob.dV
    ev = np.linalg.eigvalsh(0.5 * (H + H.T))
    assert np.allclose(esp, ev, atol=1e-10)
    # rotated bands are orthonormal and diagonalise H in the subspace
    Hu = u @ npref.np_hpsi(prob, u).T * prob.dV
    assert np.allclose(Hu, np.diag(esp), atol=1e-9)


@pytest.mark.parametrize("name", ["t0", "tk"])
def test_oracle_cg_matches_numpy(oracle_mod, name):
    prob = synth.make_problem(name)
    o = oracle_mod.Oracle(prob, k=1 if prob.is_complex else 0)
    k = 1 if prob.is_complex else 0
    nb = int(prob.nband_k[k])
    psi = synth.random_wavefunctions(13, nb, prob.ng, is_complex=prob.is_complex, kindex=k)
    psi = o.gram_schmidt(psi)
    psi, _ = o.subspace_diag(psi)
    u, esp, res = o.cg(psi)
    for b in range(min(nb, 3)):
        x, E, r = npref.np_cg_band(prob, psi[b], k)
        assert E == pytest.approx(esp[b], rel=1e-10, abs=1e-12)
        assert r == pytest.approx(res[b], rel=1e-7, abs=1e-14)
        assert np.max(np.abs(x - u[b])) < 1e-8 * np.abs(x).max()


def test_oracle_sweep_converges(oracle_mod):
    prob = synth.make_problem("t0")
    o = oracle_mod.Oracle(prob)
    psi = o.gram_schmidt(synth.random_wavefunctions(1, prob.nband, prob.ng))
    psi, _ = o.subspace_diag(psi)
    u, esp, res = o.sweep(psi, 150)
    e2, r2 = o.residual(u)
    assert r2.max() < 1e-8
    # converged eigenvalues equal the lowest eigenvalues of the dense Hamiltonian
    H = npref.np_hpsi(prob, np.eye(prob.ng))
    ev = np.linalg.eigvalsh(0.5 * (H + H.T))
    assert np.allclose(np.sort(e2), ev[:prob.nband], atol=1e-8)


def test_golden_fixtures(oracle_mod):
    g = np.load(os.path.join(GOLDEN, "oracle_golden.npz"))
    prob = synth.make_problem("c0")
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(int(g["seed"]), 4, prob.ng)
    assert np.array_equal(psi[:, ::997].ravel(), g["psi_sample"])
    h = o.hpsi(psi)
    assert np.allclose(h[:, ::997].ravel(), g["hpsi_sample"], rtol=1e-12, atol=1e-12)
    assert np.allclose(np.sum(h * h, axis=1), g["hpsi_norm2"], rtol=1e-12)
    pt = synth.make_problem("t0")
    ot = oracle_mod.Oracle(pt)
    assert np.allclose(np.linalg.eigvalsh(0.5 * (lambda H: H + H.T)(npref.np_hpsi(pt, np.eye(pt.ng))))[:pt.nband],
                       g["t0_eigs"], atol=1e-10)


@pytest.mark.parametrize("iswitch", [1, 2])
@pytest.mark.parametrize("name,k", [("t0", 0), ("tk", 3)])
def test_oracle_cg_with_cggs_matches_numpy(oracle_mod, name, k, iswitch):
    """cggs (SWGS = 1, 2) inside the oracle's CG against the numpy restatement, bands in order."""
    prob = synth.make_problem(name)
    o = oracle_mod.Oracle(prob, k=k, cggs=iswitch)
    nb = int(prob.nband_k[k])
    psi = synth.random_wavefunctions(17, nb, prob.ng, is_complex=prob.is_complex, kindex=k)
    psi = oracle_mod.Oracle(prob, k=k).gram_schmidt(psi)
    u, e, r = o.cg(psi)
    u_np, e_np, r_np = npref.np_cg_cggs(prob, psi, iswitch, k)
    assert np.max(np.abs(e - e_np)) < 1e-10
    assert np.max(np.abs(u - u_np)) < 1e-8 * np.max(np.abs(u_np))
