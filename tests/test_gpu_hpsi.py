"""hpsi parity: the CUDA library through the C ABI against the FP64 oracle.

Tolerances: FP64 path max|dH| <= 1e-12 max|H psi|; FP32 path (mixed precision hpsi) <= 2e-6.
"""
import dataclasses

import numpy as np
import pytest

from rsdft_develop_b200 import api, synth

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-6


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("name", ["t0", "t1", "c0", "c1", "c2", "c3"])
def test_hpsi_fp64_matches_oracle(oracle_mod, name):
    prob = synth.make_problem(name)
    o = oracle_mod.Oracle(prob)
    nb = {"c1": 3, "c3": 4}.get(name, 5)
    psi = synth.random_wavefunctions(21, nb, prob.ng)
    ref = o.hpsi(psi)
    with api.BandUpdate(prob) as g:
        out = g.hamiltonian(psi)
    assert _rel(out, ref) < TOL64


@pytest.mark.parametrize("name", ["t1", "c0", "c1", "c2", "c3"])
def test_hpsi_fp32_matches_oracle(oracle_mod, name):
    prob = synth.make_problem(name)
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(22, 4, prob.ng)
    ref = o.hpsi(psi.astype(np.float32).astype(np.float64))
    with api.BandUpdate(prob) as g:
        out = g.hamiltonian(psi, fp32=True)
    assert out.dtype == np.float32
    assert _rel(out.astype(np.float64), ref) < TOL32


@pytest.mark.parametrize("fp32", [False, True])
@pytest.mark.parametrize("name", ["t0", "t1", "c0", "c1", "c3"])
def test_hpsi_vloc_from_l2_matches_oracle(oracle_mod, name, fp32):
    """Stencil form 1: V_loc rows read from L2 by the consumer threads instead of staged with the
    plane (generic and compile-time row lengths, ragged last y-tiles)."""
    prob = synth.make_problem(name)
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(25, 5, prob.ng)
    if fp32:
        psi = psi.astype(np.float32).astype(np.float64)
    ref = o.hpsi(psi)
    with api.BandUpdate(prob) as g:
        g.stencil_form(True)
        out = g.hamiltonian(psi, fp32=fp32)
    assert _rel(out.astype(np.float64), ref) < (TOL32 if fp32 else TOL64)


@pytest.mark.parametrize("fp32", [False, True])
@pytest.mark.parametrize("name", ["t1", "c0", "c2"])
def test_hpsi_nonlocal_forms_agree(oracle_mod, name, fp32):
    """The nonlocal term added inside the streaming stencil and by the scatter kernel after it
    (the default) both match the oracle."""
    prob = synth.make_problem(name)
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(24, 6, prob.ng)
    if fp32:
        psi = psi.astype(np.float32).astype(np.float64)
    ref = o.hpsi(psi)
    outs = []
    with api.BandUpdate(prob) as g:
        for fused in (True, False):
            g.nl_form(fused)
            out = g.hamiltonian(psi, fp32=fp32)
            outs.append(out.astype(np.float64))
            assert _rel(outs[-1], ref) < (TOL32 if fp32 else TOL64), fused
    assert _rel(outs[0], outs[1]) < (TOL32 if fp32 else TOL64)


def test_hpsi_without_nonlocal(oracle_mod):
    prob = synth.make_problem("c0")
    o = oracle_mod.Oracle(prob, nonlocal_on=False)
    psi = synth.random_wavefunctions(23, 3, prob.ng)
    with api.BandUpdate(prob, nonlocal_on=False) as g:
        out = g.hamiltonian(psi)
    assert _rel(out, o.hpsi(psi)) < TOL64


def test_hpsi_kb_diagonal_form(oracle_mod):
    base = synth.make_problem("t1")
    rng = np.random.default_rng(5)
    pairs = np.stack([np.arange(1, base.nzlma + 1)] * 2, axis=1).astype(np.int32)
    iuv = rng.choice([-1.0, 1.0], size=base.nzlma)
    prob = dataclasses.replace(base, pairs=pairs, dij=iuv)
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(24, 3, prob.ng)
    with api.BandUpdate(prob) as g:
        out = g.hamiltonian(psi)
    assert _rel(out, o.hpsi(psi)) < TOL64


def test_hpsi_reference_form_dij_and_md4(oracle_mod):
    cfg = synth.get_config("t1", reference_form=True, md=4)
    prob = synth.make_problem(cfg)
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(25, 2, prob.ng)
    with api.BandUpdate(prob) as g:
        out = g.hamiltonian(psi)
    assert _rel(out, o.hpsi(psi)) < TOL64


def test_hpsi_single_band_and_odd_grid(oracle_mod):
    # N1 must be a multiple of 4; N2, N3 may be anything (partial y tiles, wrapped halos)
    cfg = synth.get_config("t0", n=20, h=0.42)
    prob = synth.make_problem(cfg)
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(26, 1, prob.ng)
    with api.BandUpdate(prob) as g:
        out = g.hamiltonian(psi)
        assert _rel(out, o.hpsi(psi)) < TOL64
        out32 = g.hamiltonian(psi, fp32=True)
        assert _rel(out32.astype(np.float64), o.hpsi(psi.astype(np.float32).astype(np.float64))) < TOL32


def test_hpsi_device_pointers(oracle_mod):
    torch = pytest.importorskip("torch")
    prob = synth.make_problem("c0")
    o = oracle_mod.Oracle(prob)
    psi = synth.random_wavefunctions(27, 4, prob.ng)
    with api.BandUpdate(prob) as g:
        x = torch.from_numpy(psi).cuda()
        y = torch.zeros_like(x)
        torch.cuda.synchronize()
        g.hamiltonian_device(x.data_ptr(), y.data_ptr(), 4)
        g.synchronize()
        out = y.cpu().numpy()
    assert _rel(out, o.hpsi(psi)) < TOL64


def test_random_wf_bit_identical():
    prob = synth.make_problem("c0")
    with api.BandUpdate(prob) as g:
        g.random_wf(77)
        dev = g.get_wf()
    host = synth.random_wavefunctions(77, prob.nband, prob.ng)
    assert np.array_equal(dev, host)


def test_bad_arguments_rejected():
    prob = synth.make_problem("t0")
    with api.BandUpdate(prob) as g:
        with pytest.raises(api.RsdftError) as e:
            api._call(g.lib.rsdft_gpu_hamiltonian_d, 9, 1, None, None, prob.ng, 1, 0)
        assert e.value.code == -1
        with pytest.raises(api.RsdftError):
            g.get_wf()  # nothing resident yet
