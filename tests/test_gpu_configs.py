"""Parity at the sizes of the benchmark configurations.

* C1 (64^3, 256 bands, real8): the plain FP64 GPU drop-in tracks the FP64 oracle over two
  CG -> GS -> SD sweeps from the same start: Ritz values within 1e-8 Ha, subspace within 1e-6 rad.
* C2 (96^3, 1024 bands, s+p+d projectors): the mixed-precision solve and the plain FP64 solve of
  the same input, both to max res <= 1e-8 over bands 1..mb_ref: eigenvalues within 1e-8 Ha; the
  subspace of the bands below the largest gap near mb_ref within 1e-4 rad (at res 1e-8 the
  angle of either solve to the exact subspace is bounded by ~sqrt(res)/gap, so two solves
  stopped at that tolerance cannot be compared more tightly).
* Mixed precision with the FP64 final polish (c0 and C1): the mixed solve to 1e-8, then
  rsdft_gpu_set_precision(FP64) and FP64 sweeps to 1e-12, against the FP64 solve to 1e-12:
  eigenvalues within 1e-8 Ha and subspace within 1e-6 rad.
* C4 grid (64^3, complex16, Bloch k-points) with a reduced band count: two sweeps of every
  k-point against the complex oracle at the first and last k-point.

Reference: calc_sweep (src/sweep_module.f90:158-167) over conjugate_gradient, gram_schmidt and
subspace_diag.  Starting states come from the library's seeded device generator, which is
bit-identical to synth.random_wavefunctions.
"""
import numpy as np
import pytest

from rsdft_develop_b200 import api, synth
from tests import npref

pytestmark = pytest.mark.gpu


def _device_psi(prob, seed, k=1):
    with api.BandUpdate(prob) as g:
        g.random_wf(seed, k=k)
        return g.get_wf(k=k)


def _start(o, psi):
    psi = o.gram_schmidt(psi)
    psi, _ = o.subspace_diag(psi)
    return psi


def _gap_index(esp, lo, hi):
    gaps = esp[lo:hi + 1] - esp[lo - 1:hi]
    return lo + int(np.argmax(gaps))


def test_c1_fp64_sweeps_track_oracle(oracle_mod):
    prob = synth.make_problem("c1")
    o = oracle_mod.Oracle(prob)
    psi = _start(o, _device_psi(prob, 71))
    u_ref, _, _ = o.sweep(psi, 2)
    e_ref, _ = o.residual(u_ref)
    with api.BandUpdate(prob) as g:
        g.set_wf(psi)
        it, esp, res = g.calc_sweep(2)
        u = g.get_wf()
    assert it == 2
    assert np.max(np.abs(esp[0, 0] - e_ref)) < 1e-8
    m = _gap_index(e_ref, 200, 240)
    assert npref.principal_angles(u[:m], u_ref[:m]) < 1e-6


def test_c2_mixed_solve_matches_fp64_solve():
    prob = synth.make_problem("c2")
    mb = prob.nband - prob.nband // 8
    out = {}
    for prec in (api.PREC_FP64, api.PREC_MIXED):
        with api.BandUpdate(prob, precision=prec) as g:
            g.init_sweep(mb)
            g.random_wf(72)
            g.gram_schmidt()
            it, esp, res = g.calc_sweep(400, tol=1e-8)
            assert res[0, 0, :mb].max() <= 1e-8, (prec, it)
            out[prec] = (esp[0, 0].copy(), g.get_wf(), it)
    e64, u64, it64 = out[api.PREC_FP64]
    e32, u32, it32 = out[api.PREC_MIXED]
    err = np.max(np.abs(e32[:mb] - e64[:mb]))
    m = _gap_index(e64, mb - 64, mb)
    ang = npref.principal_angles(u32[:m], u64[:m])
    print(f"c2: sweeps fp64 {it64}, mixed {it32}; eigenvalue error {err:.2e} Ha; angle {ang:.2e} rad "
          f"(bands 1..{m}, gap {e64[m] - e64[m - 1]:.2e} Ha)")
    assert err < 1e-8
    assert ang < 1e-4


@pytest.mark.parametrize("name", ["c0", "c1"])
def test_mixed_with_fp64_polish_matches_fp64_solve(name):
    prob = synth.make_problem(name)
    mb = prob.nband - prob.nband // 8
    tol = 1e-12
    with api.BandUpdate(prob, precision=api.PREC_FP64) as g:
        g.init_sweep(mb)
        g.random_wf(73)
        g.gram_schmidt()
        it64, esp, res = g.calc_sweep(600, tol=tol)
        assert res[0, 0, :mb].max() <= tol
        e64, u64 = esp[0, 0].copy(), g.get_wf()
    with api.BandUpdate(prob, precision=api.PREC_MIXED) as g:
        g.init_sweep(mb)
        g.random_wf(73)
        g.gram_schmidt()
        it32, _, res32 = g.calc_sweep(600, tol=1e-8)
        assert res32[0, 0, :mb].max() <= 1e-8
        g.set_precision(api.PREC_FP64)
        itp, esp, res = g.calc_sweep(600, tol=tol)
        assert res[0, 0, :mb].max() <= tol
        ep, up = esp[0, 0].copy(), g.get_wf()
    err = np.max(np.abs(ep[:mb] - e64[:mb]))
    m = _gap_index(e64, mb - min(32, mb // 4), mb)
    ang = npref.principal_angles(up[:m], u64[:m])
    print(f"{name}: fp64 {it64} sweeps; mixed {it32} + FP64 polish {itp} sweeps; eigenvalue error {err:.2e} Ha; "
          f"angle {ang:.2e} rad (bands 1..{m})")
    assert err < 1e-8
    assert ang < 1e-6


def test_c4_grid_two_kpoints_sweeps_track_oracle(oracle_mod):
    cfg = synth.get_config("c4", nband=32, nband_range=(24, 32))
    prob = synth.make_problem(cfg)
    starts = {}
    with api.BandUpdate(prob) as g:
        for k in range(prob.nk):
            o = oracle_mod.Oracle(prob, k=k)
            g.random_wf(74, k=k + 1)
            psi = _start(o, g.get_wf(k=k + 1))
            starts[k] = psi
            g.set_wf(psi, k=k + 1)
        it, esp, res = g.calc_sweep(2)
        us = {k: g.get_wf(k=k + 1) for k in (0, prob.nk - 1)}
    assert it == 2
    for k in (0, prob.nk - 1):
        o = oracle_mod.Oracle(prob, k=k)
        u_ref, _, _ = o.sweep(starts[k], 2)
        e_ref, _ = o.residual(u_ref)
        nb = int(prob.nband_k[k])
        assert np.max(np.abs(esp[0, k, :nb] - e_ref)) < 1e-8, k
        m = _gap_index(e_ref, nb - 8, nb - 1)
        assert npref.principal_angles(us[k][:m], u_ref[:m]) < 1e-6, k


def test_c4_grid_mixed_solve_matches_fp64_solve():
    """C4 grid (64^3, complex16, 8 Bloch k-points, uneven band counts, reduced): the mixed
    precision solve (FP32 bands, complex split-BF16 tensor-core contractions) and the plain FP64
    solve of the same input, both to max res <= 1e-8 over bands 1..nb_k - nb_k/8 of every
    k-point: eigenvalues within 1e-8 Ha."""
    cfg = synth.get_config("c4", nband=48, nband_range=(32, 48))
    prob = synth.make_problem(cfg)
    nbk = [int(x) for x in prob.nband_k]
    conv = [n - n // 8 for n in nbk]
    out = {}
    for prec in (api.PREC_FP64, api.PREC_MIXED):
        with api.BandUpdate(prob, precision=prec) as g:
            g.init_sweep(-1)
            for k in range(prob.nk):
                g.random_wf(75, k=k + 1)
                g.gram_schmidt(k=k + 1)
            it, esp, res = g.calc_sweep(400, tol=1e-8)
            for k in range(prob.nk):
                assert res[0, k, :conv[k]].max() <= 1e-8, (prec, k, it)
            out[prec] = (esp.copy(), it)
    e64, it64 = out[api.PREC_FP64]
    e32, it32 = out[api.PREC_MIXED]
    err = max(np.max(np.abs(e32[0, k, :conv[k]] - e64[0, k, :conv[k]])) for k in range(prob.nk))
    print(f"c4 grid, {nbk} bands: sweeps fp64 {it64}, mixed {it32}; eigenvalue error {err:.2e} Ha")
    assert err < 1e-8
