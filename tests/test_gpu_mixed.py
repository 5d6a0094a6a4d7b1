"""Mixed precision: split-BF16 (3-term) tensor-core GEMMs, FP32 stencils/CG, FP64 dense solves
and FP64 residuals.

Acceptance: the GEMMs stay within 5e-5 (overlaps, K up to 2.6e5) / 2e-5 (rotations) of
max|C| against cuBLAS DGEMM on the same FP32 inputs -- the tensor cores' FP32 accumulation
truncates, so the error grows with the number of accumulation steps; the mixed solver
reaches the same FP64 residual as the FP64 solver and, converged to res <= 1e-10, gives
eigenvalues within 1e-8 Ha of the FP64 oracle."""
import numpy as np
import pytest

from rsdft_develop_b200 import api, synth
from tests import npref

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,k,tol", [(256, 256, 262144, 5e-5), (100, 37, 1000, 5e-6), (384, 200, 70000, 5e-5)])
def test_gemm_x3_overlap_vs_dgemm(m, n, k, tol):
    with api.BandUpdate(synth.make_problem("t0")) as g:
        err = g.selftest_gemm(m, n, k, 0)
    assert err < tol


@pytest.mark.parametrize("m,k", [(256, 262144), (37, 1000), (1024, 50000)])
def test_gemm_x3_rotation_vs_dgemm(m, k):
    with api.BandUpdate(synth.make_problem("t0")) as g:
        err = g.selftest_gemm(m, m, k, 1)
    assert err < 2e-5


def test_mixed_gram_schmidt(oracle_mod):
    prob = synth.make_problem("c0")
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(61, prob.nband, prob.ng).astype(np.float32).astype(np.float64)
    ref = o.gram_schmidt(psi)
    with api.BandUpdate(prob, precision=api.PREC_MIXED) as g:
        g.set_wf(psi)
        g.gram_schmidt()
        q = g.get_wf()
    assert np.max(np.abs(q @ q.T * prob.dV - np.eye(prob.nband))) < 1e-5
    assert np.max(np.abs(q - ref)) < 1e-4 * np.max(np.abs(ref))


def test_mixed_subspace_diag(oracle_mod):
    prob = synth.make_problem("c0")
    o = oracle_mod.Oracle(prob)
    psi = o.gram_schmidt(synth.random_wavefunctions(62, prob.nband, prob.ng))
    psi = psi.astype(np.float32).astype(np.float64)
    _, e_ref = o.subspace_diag(psi)
    with api.BandUpdate(prob, precision=api.PREC_MIXED) as g:
        g.set_wf(psi)
        esp = g.subspace_diag()
    assert np.max(np.abs(esp - e_ref)) < 1e-5 * np.max(np.abs(e_ref))


def test_mixed_cg_tracks_fp64(oracle_mod):
    prob = synth.make_problem("c0")
    o = oracle_mod.Oracle(prob)
    psi = o.gram_schmidt(synth.random_wavefunctions(63, prob.nband, prob.ng))
    psi, _ = o.subspace_diag(psi)
    u_ref, e_ref, r_ref = o.cg(psi)
    with api.BandUpdate(prob, precision=api.PREC_MIXED) as g:
        g.set_wf(psi)
        esp, res = g.conjugate_gradient()
    assert np.max(np.abs(esp - e_ref)) < 1e-5


def test_mixed_solver_reaches_fp64_accuracy(oracle_mod):
    """At equal FP64 residual the mixed and FP64 solves are equally accurate; at res <= 1e-10
    the mixed eigenvalues are within 1e-8 Ha of the converged FP64 oracle."""
    prob = synth.make_problem("t0")
    o = oracle_mod.Oracle(prob)
    psi = o.gram_schmidt(synth.random_wavefunctions(64, prob.nband, prob.ng))
    psi, _ = o.subspace_diag(psi)
    u_ref, _, _ = o.sweep(psi, 300)
    e_ref, r_ref = o.residual(u_ref)
    errs = {}
    for prec in (api.PREC_FP64, api.PREC_MIXED):
        with api.BandUpdate(prob, precision=prec) as g:
            g.set_wf(psi)
            it, esp, res = g.calc_sweep(400, tol=1e-8)
            assert res.max() <= 1e-8, (prec, it, res.max())
            errs[prec] = np.max(np.abs(np.sort(esp[0, 0]) - np.sort(e_ref)))
    assert errs[api.PREC_MIXED] <= 3.0 * errs[api.PREC_FP64] + 1e-9, errs
    with api.BandUpdate(prob, precision=api.PREC_MIXED) as g:
        g.set_wf(psi)
        it, esp, res = g.calc_sweep(600, tol=1e-10)
        u = g.get_wf()
    assert res.max() <= 1e-10, (it, res.max())
    assert np.max(np.abs(np.sort(esp[0, 0]) - np.sort(e_ref))) < 1e-8
    assert npref.principal_angles(u, u_ref) < 5e-4
