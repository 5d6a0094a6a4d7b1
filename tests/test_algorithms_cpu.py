"""CPU checks of the two reformulations the GPU sweep uses (numpy, FP64):

* precond_hprsdft in s-step form: the mloop CG steps run on coefficient vectors in the basis
  v_i = B^i r0 (B = (A - c0 I) / c0), with every inner product taken from the moments
  mu_j = <r0|B^j r0>; the result must equal the recurrence form (tests/npref.py:np_precond,
  itself the restatement of src/conjugate_gradient/cgpc_hprsdft_module.f90:133-270).
  The coefficient recurrence below is the same arithmetic as the kernel k_pcs_sc (cg.cu).
* the fused Cholesky-Rayleigh-Ritz step: S = dV X^T X = R^T R, Hsub = R^-T (dV X^T H X) R^-1 =
  V diag(e) V^T, X <- X (R^-1 V), against Gram-Schmidt (Cholesky QR) followed by subspace
  diagonalisation on the orthonormalised block.
"""
import numpy as np
import pytest
import scipy.linalg as sla

from rsdft_develop_b200 import synth
from tests import npref


def _sstep_precond(prob, g, mloop):
    n1, n2, n3 = prob.n
    h = prob.h
    c0 = 3.0 / h ** 2
    c = -0.5 / h ** 2

    def offdiag(v):  # (A - c0 I) v
        x = v.reshape(n3, n2, n1)
        f = np.zeros_like(x)
        for ax in (2, 1, 0):
            f = f + c * (np.roll(x, 1, axis=ax) + np.roll(x, -1, axis=ax))
        return f.ravel()

    def A(v):
        return c0 * v + offdiag(v)

    r0 = g - A(g)
    mu0 = float(np.dot(r0, r0))
    if mu0 < 1e-24:
        return g.copy()
    basis = [r0]
    for _ in range(1, mloop):
        basis.append(offdiag(basis[-1]) / c0)
    nxt = offdiag(basis[-1]) / c0
    # moments mu_j = <r0 | B^j r0> from the basis, as the passes that build it gather them
    mu = np.zeros(2 * mloop)
    mu[0] = mu0
    for i in range(1, mloop):
        mu[2 * i - 1] = np.dot(basis[i - 1], basis[i])
        mu[2 * i] = np.dot(basis[i], basis[i])
    mu[2 * mloop - 1] = np.dot(basis[-1], nxt)
    # the CG recurrence on coefficients (k_pcs_sc)
    p = np.zeros(mloop + 1); p[0] = 1.0
    r = p.copy()
    xi = np.zeros(mloop + 1)
    rr1 = mu[0]
    for it in range(1, mloop + 1):
        f = np.zeros(mloop + 1)
        for j in range(it + 1):
            f[j] = c0 * ((p[j - 1] if j > 0 else 0.0) + (p[j] if j < it else 0.0))
        pAp = sum(p[a] * f[b] * mu[a + b] for a in range(it) for b in range(it + 1))
        rr0 = rr1
        al = rr0 / pAp
        xi[:it] += al * p[:it]
        if it == mloop:
            break
        r[: it + 1] -= al * f[: it + 1]
        rr1 = sum(r[a] * r[b] * mu[a + b] for a in range(it + 1) for b in range(it + 1))
        be = rr1 / rr0
        p[: it + 1] = r[: it + 1] + be * p[: it + 1]
    return g + sum(xi[i] * basis[i] for i in range(mloop))


@pytest.mark.parametrize("name", ["t0", "t1"])
@pytest.mark.parametrize("mloop", [1, 2, 3, 4])
def test_sstep_preconditioner_equals_recurrence(name, mloop):
    prob = synth.make_problem(name)
    g = synth.random_wavefunctions(41, 3, prob.ng)
    for b in range(3):
        ref = npref.np_precond(prob, g[b], mloop=mloop)
        out = _sstep_precond(prob, g[b], mloop)
        assert np.max(np.abs(out - ref)) < 1e-10 * np.max(np.abs(ref))


def test_sstep_preconditioner_zero_band():
    prob = synth.make_problem("t0")
    g = np.zeros(prob.ng)
    assert np.all(_sstep_precond(prob, g, 3) == 0.0)


def test_cholesky_rayleigh_ritz_equals_gs_then_sd():
    prob = synth.make_problem("t1")
    nb = prob.nband
    X = synth.random_wavefunctions(42, nb, prob.ng)  # [nb][ng]
    HX = npref.np_hpsi(prob, X)
    dV = prob.dV
    # fused: one rotation X (R^-1 V)
    S = dV * X @ X.T
    M = dV * X @ HX.T
    M = 0.5 * (M + M.T)
    R = np.linalg.cholesky(S).T  # S = R^T R, R upper
    Ri = sla.solve_triangular(R, np.eye(nb), lower=False)
    Hs = Ri.T @ M @ Ri
    e1, V = np.linalg.eigh(0.5 * (Hs + Hs.T))
    Y1 = (X.T @ (Ri @ V)).T
    # separate: Q = X R^-1 (Gram-Schmidt as Cholesky QR), then Rayleigh-Ritz on Q
    Q = (X.T @ Ri).T
    HQ = npref.np_hpsi(prob, Q)
    Hq = dV * Q @ HQ.T
    e2, W = np.linalg.eigh(0.5 * (Hq + Hq.T))
    Y2 = (Q.T @ W).T
    assert np.max(np.abs(e1 - e2)) < 1e-9 * np.max(np.abs(e2))
    # same Ritz vectors up to sign (non-degenerate spectrum of the random block)
    ov = np.abs(np.sum(Y1 * Y2, axis=1) * dV)
    assert np.max(np.abs(ov - 1.0)) < 1e-8
    assert np.max(np.abs(dV * Y1 @ Y1.T - np.eye(nb))) < 1e-9
