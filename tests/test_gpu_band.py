"""Band-structure driver (src/band_module.f90:47-361) on the GPU.

* Free-electron known answer: with V_loc = 0 and no projectors the Hamiltonian at k is the FD
  kinetic operator of zcoef_kin(k), whose eigenvalues are the plane-wave dispersion
  (tests/npref.dispersion, pinned against the oracle and the analytic 1/2 |k + G|^2 in
  test_oracle.py).  Along Gamma -> X -> M the driver's eigenvalues of bands 1..mb2 must equal the
  lowest dispersion values at every trajectory point within 1e-8 Ha.
* Full synthetic operator: at every point of a short trajectory the driver's eigenvalues equal
  the oracle's converged sweeps at the same k within 1e-7 Ha.
* The band_eigv text carries one block per trajectory point.
"""
import dataclasses

import numpy as np
import pytest

from rsdft_develop_b200 import band, synth
from tests import npref

pytestmark = pytest.mark.gpu

AK = [[0.0, 0.0, 0.0], [0.5, 0.0, 0.0], [0.5, 0.5, 0.0]]


def test_trajectory_points():
    t = band.k_trajectory(AK, [4, 2])
    assert t.shape == (7, 6)
    assert np.allclose(t[:, :3], [[0, 0, 0], [.125, 0, 0], [.25, 0, 0], [.375, 0, 0], [.5, 0, 0], [.5, .25, 0], [.5, .5, 0]])
    assert np.allclose(t[-1, 3:], 0.0)


def test_free_electron_bands_match_dispersion(tmp_path):
    cfg = synth.get_config("tk", nband=14)
    prob = band.trajectory_problem(cfg, AK, [3, 2])
    mb2 = 9
    path = str(tmp_path / "band_eigv")
    r = band.band_structure(cfg, AK, [3, 2], mb2, esp_conv_tol=1e-11, maxiter=400,
                            vloc=np.zeros(prob.ng), nonlocal_on=False, eigv_path=path)
    n = prob.n[0]
    ms = range(-n // 2, n // 2)
    for ik in range(prob.nk):
        ana = np.sort([npref.dispersion(prob, a, b, c, ik).real for a in ms for b in (-2, -1, 0, 1, 2)
                       for c in (-2, -1, 0, 1, 2)])[:mb2]
        assert np.max(np.abs(r.esp[ik] - ana)) < 1e-8, (ik, r.esp[ik], ana)
    text = open(path).read().split("\n")
    assert text[1].startswith(" Fermi_energy(hartree):")
    assert sum(1 for line in text if line.strip().endswith(" 1") and len(line.split()) == 6) == prob.nk


def test_synthetic_operator_bands_match_oracle(oracle_mod):
    cfg = synth.get_config("tk", nband=10)
    ak = [[0.0, 0.0, 0.0], [0.25, 0.25, 0.25]]
    mb2 = 6
    r = band.band_structure(cfg, ak, [2], mb2, esp_conv_tol=1e-11, maxiter=400)
    prob = band.trajectory_problem(cfg, ak, [2])
    for ik in range(prob.nk):
        o = oracle_mod.Oracle(prob, k=ik)
        psi = synth.random_wavefunctions(9, prob.nband, prob.ng, is_complex=True)
        psi = o.gram_schmidt(psi)
        u, _, _ = o.sweep(psi, 300)
        e, res = o.residual(u)
        e = np.sort(e)
        assert np.max(np.abs(r.esp[ik] - e[:mb2])) < 1e-7, (ik, r.esp[ik], e[:mb2])
