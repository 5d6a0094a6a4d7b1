"""Mixed precision: split-BF16 tensor-core GEMMs (two terms in the overlap/Hsub sums, three in
the rotations), FP32 stencils/CG/preconditioner, FP64 dense solves and FP64 residuals.

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


@pytest.mark.parametrize("wide", [True, False])
@pytest.mark.parametrize("m,n,k,tol", [(256, 256, 262144, 5e-5), (100, 37, 1000, 5e-6), (384, 200, 70000, 5e-5),
                                      (300, 520, 4160, 5e-6)])
def test_gemm_x3_overlap_vs_dgemm(m, n, k, tol, wide):
    with api.BandUpdate(synth.make_problem("t0")) as g:
        g.gemm_terms(3, 3)
        g.gemm_tile(wide)
        err = g.selftest_gemm(m, n, k, 0)
    assert err < tol


@pytest.mark.parametrize("wide", [True, False])
@pytest.mark.parametrize("m,k", [(256, 262144), (37, 1000), (1024, 50000), (300, 4160)])
def test_gemm_x3_rotation_vs_dgemm(m, k, wide):
    with api.BandUpdate(synth.make_problem("t0")) as g:
        g.gemm_terms(3, 3)
        g.gemm_tile(wide)
        err = g.selftest_gemm(m, m, k, 1)
    assert err < 2e-5


@pytest.mark.parametrize("m,n,k", [(256, 256, 262144), (100, 37, 1000), (384, 200, 70000)])
def test_gemm_two_terms_overlap_vs_dgemm(m, n, k):
    """Two BF16 terms per value: each product is good to about 2^-16, but the rounding is
    unbiased, so over K terms the sum keeps the three-term error level set by the FP32
    accumulation (long sums) or stays within 2^-16 of max|C| (short ones)."""
    with api.BandUpdate(synth.make_problem("t0")) as g:
        g.gemm_terms(3, 3)
        e3 = g.selftest_gemm(m, n, k, 0)
        g.gemm_terms(2, 3)
        e2 = g.selftest_gemm(m, n, k, 0)
    assert e2 < max(2.0 * e3, 3e-5), (e2, e3)


def test_gemm_two_terms_rotation_vs_dgemm():
    with api.BandUpdate(synth.make_problem("t0")) as g:
        g.gemm_terms(3, 2)
        err = g.selftest_gemm(256, 256, 262144, 1)
    assert err < 5e-5


@pytest.mark.parametrize("tri", [0, 1, 2])
@pytest.mark.parametrize("wide", [True, False])
@pytest.mark.parametrize("m,k", [(512, 65536), (1024, 21824), (200, 4160)])
def test_fused_overlap_hsub_vs_dgemm(m, k, wide, tri):
    """[S | Hsub] in one contraction: full, S by triangle tiles (the default), or both by
    triangle tiles (tiles wholly above the diagonal are left out from nb = 256 / 512 bands on;
    nb = 200 has tiles straddling S and Hsub), against DGEMM on the guaranteed elements."""
    with api.BandUpdate(synth.make_problem("t0")) as g:
        g.gemm_terms(3, 3)
        g.gemm_tile(wide, tri)
        err = g.selftest_gemm(m, m, k, 2)
    assert err < 5e-5, err


def test_gemm_terms_argument_checked():
    with api.BandUpdate(synth.make_problem("t0")) as g:
        with pytest.raises(api.RsdftError):
            g.gemm_terms(1, 3)


@pytest.mark.parametrize("name,mloop", [("t0", 3), ("c0", 3), ("c0", 1), ("c0", 2), ("c0", 4)])
def test_mixed_precond_matches_oracle(oracle_mod, name, mloop):
    """precond_hprsdft on FP32 bands (the s-step evaluation of the mloop CG steps) against the
    FP64 oracle's recurrence on the same FP32-representable input: FP32-level agreement."""
    prob = synth.make_problem(name)
    o = oracle_mod.Oracle(prob, mloop=mloop)
    g = synth.random_wavefunctions(33, 5, prob.ng).astype(np.float32)
    ref = o.precond(g.astype(np.float64))
    with api.BandUpdate(prob, precision=api.PREC_MIXED, mloop=mloop) as gpu:
        out = gpu.precond_f32(g)
    assert np.max(np.abs(out - ref)) < 2e-5 * np.max(np.abs(ref))


def test_mixed_precond_zero_band(oracle_mod):
    """A zero band stays zero (the reference's rr < 1e-24 exit) next to a normal band."""
    prob = synth.make_problem("t0")
    o = oracle_mod.Oracle(prob)
    g = synth.random_wavefunctions(34, 2, prob.ng).astype(np.float32)
    g[0] = 0.0
    ref = o.precond(g.astype(np.float64))
    with api.BandUpdate(prob, precision=api.PREC_MIXED) as gpu:
        out = gpu.precond_f32(g)
    assert np.all(out[0] == 0.0)
    assert np.max(np.abs(out[1] - ref[1])) < 2e-5 * np.max(np.abs(ref[1]))


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


@pytest.mark.parametrize("terms", [(3, 3), (2, 3)])
def test_mixed_solver_reaches_fp64_accuracy(oracle_mod, terms):
    """At equal FP64 residual the mixed and FP64 solves are equally accurate; at res <= 1e-10
    the mixed eigenvalues are within 1e-8 Ha of the converged FP64 oracle, with three BF16
    terms in the rotations and two or three in the overlap/Hsub contractions.  (Two-term
    rotations write 2^-16-relative noise into every band each sweep; the residual then stalls
    near 5e-9, so they are not used.)"""
    prob = synth.make_problem("t0")
    o = oracle_mod.Oracle(prob)
    psi = o.gram_schmidt(synth.random_wavefunctions(64, prob.nband, prob.ng))
    psi, _ = o.subspace_diag(psi)
    u_ref, _, _ = o.sweep(psi, 300)
    e_ref, r_ref = o.residual(u_ref)
    errs = {}
    for prec in (api.PREC_FP64, api.PREC_MIXED):
        with api.BandUpdate(prob, precision=prec) as g:
            g.gemm_terms(*terms)
            g.set_wf(psi)
            it, esp, res = g.calc_sweep(400, tol=1e-8)
            assert res.max() <= 1e-8, (prec, it, res.max())
            errs[prec] = np.max(np.abs(np.sort(esp[0, 0]) - np.sort(e_ref)))
    assert errs[api.PREC_MIXED] <= 3.0 * errs[api.PREC_FP64] + 1e-9, errs
    with api.BandUpdate(prob, precision=api.PREC_MIXED) as g:
        g.gemm_terms(*terms)
        g.set_wf(psi)
        it, esp, res = g.calc_sweep(600, tol=1e-10)
        u = g.get_wf()
    assert res.max() <= 1e-10, (it, res.max())
    assert np.max(np.abs(np.sort(esp[0, 0]) - np.sort(e_ref))) < 1e-8
    assert npref.principal_angles(u, u_ref) < 5e-4
