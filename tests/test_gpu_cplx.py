"""complex16 (k-point) hpsi parity against the FP64 oracle (z_op_kinetic_sol + z_op_ps_nloc_mr)."""
import numpy as np
import pytest

from rsdft_develop_b200 import api, synth

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("k", [0, 3, 7])
def test_hpsi_complex_fp64(oracle_mod, k):
    prob = synth.make_problem("tk")
    o = oracle_mod.Oracle(prob, k=k)
    psi = synth.random_wavefunctions(41, 3, prob.ng, is_complex=True, kindex=k)
    with api.BandUpdate(prob) as g:
        out = g.hamiltonian(psi, k=k + 1)
    assert _rel(out, o.hpsi(psi)) < 1e-12


def test_hpsi_complex_fp32(oracle_mod):
    prob = synth.make_problem("tk")
    o = oracle_mod.Oracle(prob, k=5)
    psi = synth.random_wavefunctions(42, 2, prob.ng, is_complex=True, kindex=5)
    with api.BandUpdate(prob) as g:
        out = g.hamiltonian(psi, k=6, fp32=True)
    ref = o.hpsi(psi.astype(np.complex64).astype(np.complex128))
    assert _rel(out.astype(np.complex128), ref) < 2e-6


def test_hpsi_complex_c4_all_kpoints(oracle_mod):
    prob = synth.make_problem("c4")
    with api.BandUpdate(prob) as g:
        for k in range(prob.nk):
            o = oracle_mod.Oracle(prob, k=k)
            psi = synth.random_wavefunctions(43, 2, prob.ng, is_complex=True, kindex=k)
            assert _rel(g.hamiltonian(psi, k=k + 1), o.hpsi(psi)) < 1e-12


def _start_c(o, prob, k, seed=51):
    nb = int(prob.nband_k[k])
    psi = synth.random_wavefunctions(seed, nb, prob.ng, is_complex=True, kindex=k)
    psi = o.gram_schmidt(psi)
    psi, _ = o.subspace_diag(psi)
    return psi


def test_cg_complex_matches_oracle(oracle_mod):
    prob = synth.make_problem("tk")
    k = 2
    o = oracle_mod.Oracle(prob, k=k)
    psi = _start_c(o, prob, k)
    u_ref, e_ref, r_ref = o.cg(psi)
    with api.BandUpdate(prob) as g:
        g.set_wf(np.zeros((int(prob.nband_k[0]), prob.ng), np.complex128), k=1)
        g.set_wf(psi, k=k + 1)
        esp, res = g.conjugate_gradient(k=k + 1)
        u = g.get_wf(k=k + 1)
    assert np.max(np.abs(esp - e_ref)) < 1e-10
    assert np.all(np.abs(res - r_ref) <= 1e-7 * np.abs(r_ref) + 1e-14)
    assert np.max(np.abs(u - u_ref)) < 1e-8 * np.max(np.abs(u_ref))


def test_gs_sd_complex_match_oracle(oracle_mod):
    prob = synth.make_problem("tk")
    k = 4
    o = oracle_mod.Oracle(prob, k=k)
    nb = int(prob.nband_k[k])
    psi = synth.random_wavefunctions(52, nb, prob.ng, is_complex=True, kindex=k)
    q_ref = o.gram_schmidt(psi)
    u_ref, e_ref = o.subspace_diag(q_ref)
    with api.BandUpdate(prob) as g:
        g.set_wf(psi, k=k + 1)
        g.gram_schmidt(k=k + 1)
        q = g.get_wf(k=k + 1)
        esp = g.subspace_diag(k=k + 1)
    assert np.max(np.abs(q - q_ref)) < 1e-9 * np.max(np.abs(q_ref))
    assert np.max(np.abs(esp - e_ref)) < 1e-10


def test_sweep_complex_all_kpoints_converge(oracle_mod):
    """Every k-point converges to residual <= 1e-10 and matches the oracle's converged eigenvalues."""
    prob = synth.make_problem("tk")
    with api.BandUpdate(prob) as g:
        for k in range(prob.nk):
            o = oracle_mod.Oracle(prob, k=k)
            g.set_wf(_start_c(o, prob, k, 53 + k), k=k + 1)
        it, esp, res = g.calc_sweep(400, tol=1e-10)
    assert np.nanmax(res) <= 1e-10
    for k in (0, 7):
        o = oracle_mod.Oracle(prob, k=k)
        u_ref, _, _ = o.sweep(_start_c(o, prob, k, 53 + k), 200)
        e_ref, r_ref = o.residual(u_ref)
        nb = int(prob.nband_k[k])
        assert np.max(np.abs(np.sort(esp[0, k, :nb]) - np.sort(e_ref))) < 1e-8


def test_gs_sd_complex_mixed_match_oracle(oracle_mod):
    """Mixed precision, complex16: Gram-Schmidt and subspace diagonalisation through the
    split-BF16 tensor-core contractions (complex overlaps over the interleaved view, complex
    rotation as the real form of its matrix) against the FP64 oracle on FP32-rounded input."""
    prob = synth.make_problem("tk")
    k = 4
    o = oracle_mod.Oracle(prob, k=k)
    nb = int(prob.nband_k[k])
    psi = synth.random_wavefunctions(54, nb, prob.ng, is_complex=True, kindex=k)
    psi = psi.astype(np.complex64).astype(np.complex128)
    q_ref = o.gram_schmidt(psi)
    u_ref, e_ref = o.subspace_diag(q_ref)
    with api.BandUpdate(prob, precision=api.PREC_MIXED) as g:
        g.set_wf(psi, k=k + 1)
        g.gram_schmidt(k=k + 1)
        q = g.get_wf(k=k + 1)
        esp = g.subspace_diag(k=k + 1)
        u = g.get_wf(k=k + 1)
    assert np.max(np.abs(q.conj() @ q.T * prob.dV - np.eye(nb))) < 1e-5
    assert np.max(np.abs(q - q_ref)) < 1e-4 * np.max(np.abs(q_ref))
    assert np.max(np.abs(esp - e_ref)) < 1e-5 * np.max(np.abs(e_ref))
    # eigenvectors up to a phase: |<u_ref|u>| = 1 band by band
    ov = np.abs(np.sum(u_ref.conj() * u, axis=1) * prob.dV)
    assert np.all(np.abs(ov - 1.0) < 1e-4)


def test_sweep_complex_mixed_all_kpoints_converge(oracle_mod):
    """Mixed precision, complex16, all 8 k-points: residual <= 1e-8 and the eigenvalues of the
    first and last k-point within 1e-8 Ha of the oracle's converged ones."""
    prob = synth.make_problem("tk")
    with api.BandUpdate(prob, precision=api.PREC_MIXED) as g:
        for k in range(prob.nk):
            o = oracle_mod.Oracle(prob, k=k)
            g.set_wf(_start_c(o, prob, k, 55 + k), k=k + 1)
        it, esp, res = g.calc_sweep(400, tol=1e-8)
    assert np.nanmax(res) <= 1e-8
    for k in (0, 7):
        o = oracle_mod.Oracle(prob, k=k)
        u_ref, _, _ = o.sweep(_start_c(o, prob, k, 55 + k), 200)
        e_ref, r_ref = o.residual(u_ref)
        nb = int(prob.nband_k[k])
        assert np.max(np.abs(np.sort(esp[0, k, :nb]) - np.sort(e_ref))) < 1e-8
