"""CG / preconditioner / Gram-Schmidt / subspace-diag / sweep parity against the FP64 oracle.

Acceptance (the path's stated bar): eigenvalues within 1e-8 Ha of the oracle and the
converged subspace within 1e-6 principal-angle error; per-routine checks are tighter.
"""
import numpy as np
import pytest

from rsdft_develop_b200 import api, synth
from tests import npref

pytestmark = pytest.mark.gpu


def _start(o, prob, seed=31):
    psi = synth.random_wavefunctions(seed, prob.nband, prob.ng)
    psi = o.gram_schmidt(psi)
    psi, _ = o.subspace_diag(psi)
    return psi


@pytest.mark.parametrize("name", ["t0", "c0"])
def test_precond_matches_oracle(oracle_mod, name):
    prob = synth.make_problem(name)
    o = oracle_mod.Oracle(prob)
    g = synth.random_wavefunctions(32, 4, prob.ng)
    ref = o.precond(g)
    with api.BandUpdate(prob) as gpu:
        out = gpu.precond(g)
    assert np.max(np.abs(out - ref)) < 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("name,block", [("t0", 0), ("c0", 0), ("c0", 7)])
def test_cg_matches_oracle(oracle_mod, name, block):
    prob = synth.make_problem(name)
    o = oracle_mod.Oracle(prob)
    psi = _start(o, prob)
    u_ref, e_ref, r_ref = o.cg(psi)
    with api.BandUpdate(prob, cg_block=block) as g:
        g.set_wf(psi)
        esp, res = g.conjugate_gradient()
        u = g.get_wf()
    assert np.max(np.abs(esp - e_ref)) < 1e-10
    assert np.all(np.abs(res - r_ref) <= 1e-7 * np.abs(r_ref) + 1e-14)
    assert np.max(np.abs(u - u_ref)) < 1e-8 * np.max(np.abs(u_ref))


def test_gram_schmidt_matches_oracle(oracle_mod):
    prob = synth.make_problem("c0")
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(33, prob.nband, prob.ng)
    ref = o.gram_schmidt(psi)
    with api.BandUpdate(prob) as g:
        g.set_wf(psi)
        g.gram_schmidt()
        q = g.get_wf()
    assert np.max(np.abs(q @ q.T * prob.dV - np.eye(prob.nband))) < 1e-12
    assert np.max(np.abs(q - ref)) < 1e-9 * np.max(np.abs(ref))


def test_subspace_diag_matches_oracle(oracle_mod):
    prob = synth.make_problem("c0")
    o = oracle_mod.Oracle(prob)
    psi = o.gram_schmidt(synth.random_wavefunctions(34, prob.nband, prob.ng))
    u_ref, e_ref = o.subspace_diag(psi)
    with api.BandUpdate(prob) as g:
        g.set_wf(psi)
        esp = g.subspace_diag()
        u = g.get_wf()
    assert np.max(np.abs(esp - e_ref)) < 1e-10
    # eigenvector signs are arbitrary: compare |<u_ref|u>| = 1 band by band
    ov = np.abs(np.sum(u * u_ref, axis=1) * prob.dV)
    assert np.all(np.abs(ov - 1.0) < 1e-9)


def test_residual_matches_oracle(oracle_mod):
    prob = synth.make_problem("c0")
    o = oracle_mod.Oracle(prob)
    psi = _start(o, prob, 35)
    e_ref, r_ref = o.residual(psi)
    with api.BandUpdate(prob) as g:
        g.set_wf(psi)
        e, r = g.residual()
    assert np.max(np.abs(e - e_ref)) < 1e-11
    assert np.all(np.abs(r - r_ref) <= 1e-8 * r_ref + 1e-16)


def test_sweeps_track_oracle(oracle_mod):
    prob = synth.make_problem("c0")
    o = oracle_mod.Oracle(prob)
    psi = _start(o, prob, 36)
    u_ref, e_ref, _ = o.sweep(psi, 4)
    with api.BandUpdate(prob) as g:
        g.set_wf(psi)
        it, esp, res = g.calc_sweep(4)
        u = g.get_wf()
    e_o, _ = o.residual(u_ref)
    assert it == 4
    assert np.max(np.abs(esp[0, 0] - e_o)) < 1e-8
    assert npref.principal_angles(u, u_ref) < 1e-6


def test_converged_eigenvalues_and_subspace(oracle_mod):
    """Run both to residual <= 1e-8 and compare eigenvalues (1e-8 Ha) and subspace (1e-6 rad)."""
    prob = synth.make_problem("t0")
    o = oracle_mod.Oracle(prob)
    psi = _start(o, prob, 37)
    u_ref, _, _ = o.sweep(psi, 400)
    e_ref, r_ref = o.residual(u_ref)
    assert r_ref.max() < 1e-15
    with api.BandUpdate(prob) as g:
        g.set_wf(psi)
        it, esp, res = g.calc_sweep(600, tol=1e-15)
        u = g.get_wf()
    assert res.max() <= 1e-15
    assert np.max(np.abs(np.sort(esp[0, 0]) - np.sort(e_ref))) < 1e-8
    assert npref.principal_angles(u, u_ref) < 1e-6


@pytest.mark.parametrize("iswitch", [1, 2])
@pytest.mark.parametrize("name,k", [("c0", 0), ("tk", 5)])
def test_cg_with_cggs_matches_oracle(oracle_mod, name, k, iswitch):
    """SWGS = 1 / 2: the preconditioned gradients orthogonalised against the lower / all other
    bands inside conjugate_gradient (cggs, src/conjugate_gradient/cggs_module.f90), one band per
    CG block (MB_d = 1, the oracle's band order)."""
    prob = synth.make_problem(name)
    o = oracle_mod.Oracle(prob, k=k, cggs=iswitch)
    nb = int(prob.nband_k[k])
    psi = synth.random_wavefunctions(38, nb, prob.ng, is_complex=prob.is_complex, kindex=k)
    psi = oracle_mod.Oracle(prob, k=k).gram_schmidt(psi)
    u_ref, e_ref, r_ref = o.cg(psi)
    with api.BandUpdate(prob, cg_block=1) as g:
        g.cggs(iswitch)
        g.set_wf(psi, k=k + 1)
        esp, res = g.conjugate_gradient(k=k + 1)
        u = g.get_wf(k=k + 1)
    assert np.max(np.abs(esp - e_ref)) < 1e-10
    assert np.all(np.abs(res - r_ref) <= 1e-7 * np.abs(r_ref) + 1e-14)
    assert np.max(np.abs(u - u_ref)) < 1e-8 * np.max(np.abs(u_ref))


def test_cg_with_cggs_mixed_tracks_oracle(oracle_mod):
    """The same on FP32 bands (mixed precision): energies within 1e-5 Ha of the FP64 oracle."""
    prob = synth.make_problem("c0")
    o = oracle_mod.Oracle(prob, cggs=1)
    psi = oracle_mod.Oracle(prob).gram_schmidt(synth.random_wavefunctions(39, prob.nband, prob.ng))
    _, e_ref, _ = o.cg(psi)
    with api.BandUpdate(prob, precision=api.PREC_MIXED, cg_block=1) as g:
        g.cggs(1)
        g.set_wf(psi)
        esp, res = g.conjugate_gradient()
    assert np.max(np.abs(esp - e_ref)) < 1e-5
