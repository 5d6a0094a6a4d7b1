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
