"""Failure paths of the C ABI: each is provoked on the host side or by a bounded wait that is
told to give up, never by a GPU fault, and each leaves the context usable.

Reference convention: the reference stops (stop_program) or reports ierr < 0 from calc_sweep
(src/sweep_module.f90:192-240); the library returns a negative status instead.
"""
import numpy as np
import pytest

from rsdft_develop_b200 import api, synth

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_rank_deficient_bands_give_not_spd_and_context_recovers(oracle_mod):
    """A zero band makes the overlap matrix singular: gram_schmidt returns RSDFT_ERR_NOT_SPD (-4)
    before it touches the bands; good bands then orthonormalise as usual."""
    prob = synth.make_problem("t1")
    psi = synth.random_wavefunctions(31, prob.nband, prob.ng)
    bad = psi.copy()
    bad[3] = 0.0
    for prec in (api.PREC_FP64, api.PREC_MIXED):
        with api.BandUpdate(prob, precision=prec) as g:
            g.set_wf(bad)
            with pytest.raises(api.RsdftError) as e:
                g.gram_schmidt()
            assert e.value.code == -4, prec
            g.set_wf(psi)
            g.gram_schmidt()
            q = g.get_wf()
            s = q @ q.T * prob.dV
            assert np.max(np.abs(s - np.eye(prob.nband))) < (1e-10 if prec == api.PREC_FP64 else 1e-5)


def test_nonfinite_vloc_rejected_and_context_recovers(oracle_mod):
    """V_loc with a NaN is refused with RSDFT_ERR_NUMERIC (-9); the previous V_loc stays in use."""
    prob = synth.make_problem("t1")
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(32, 3, prob.ng)
    with api.BandUpdate(prob) as g:
        v = np.ascontiguousarray(prob.vloc, np.float64).copy()
        v[17] = np.nan
        with pytest.raises(api.RsdftError) as e:
            api._call(g.lib.rsdft_gpu_set_vloc, api._ptr(v), prob.ng, 1)
        assert e.value.code == -9
        assert _rel(g.hamiltonian(psi), o.hpsi(psi)) < 1e-12


def test_stencil_wait_timeout_returns_status_and_context_recovers(oracle_mod):
    """With the stencil's bounded waits told to give up at once, hamiltonian returns
    RSDFT_ERR_TIMEOUT (-6) (the kernel lets its own bulk copies land before it exits); with
    the default limit restored the next call is correct."""
    prob = synth.make_problem("c0")
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(33, 4, prob.ng)
    ref = o.hpsi(psi)
    with api.BandUpdate(prob) as g:
        g.wait_polls(0)
        with pytest.raises(api.RsdftError) as e:
            g.hamiltonian(psi)
        assert e.value.code == -6
        g.wait_polls(-1)
        assert _rel(g.hamiltonian(psi), ref) < 1e-12
        out32 = g.hamiltonian(psi, fp32=True).astype(np.float64)
        assert _rel(out32, o.hpsi(psi.astype(np.float32).astype(np.float64))) < 2e-6


def test_stalled_learned_preconditioner_falls_back_and_converges():
    """A network that stalls the solve (all weights zero: Pg = 0, so CG cannot move): the
    FP64-residual guard of calc_sweep switches CG to precond_hprsdft (fallback counter 1) and
    the solve still reaches the tolerance."""
    prob = synth.make_problem("c0")
    tol = 1e-8
    mb = prob.nband - prob.nband // 8
    with api.BandUpdate(prob, precision=api.PREC_MIXED, pc_mode=api.PC_LEARNED) as g:
        g.lpc_set_weights(np.zeros(api.LPC_NWEIGHTS, np.float32))
        g.init_sweep(mb)
        g.random_wf(9)
        g.gram_schmidt()
        it, esp, res = g.calc_sweep(400, tol)
        ready, pc_now, fallbacks, _ = g.lpc_status()
    assert ready == 1
    assert fallbacks >= 1 and pc_now == api.PC_HPRSDFT
    assert res[0, 0, :mb].max() <= tol and it < 400
