"""CPU checks of the SCF oracle (oracle/scf_oracle.py) and of the host side of the SCF driver.

* Hartree: a cosine density rho = cos(G.r) has V_H = 4 pi / |G|^2 cos(G.r) exactly.
* PZ81: both branches of the published correlation fit meet at rs = 1 (energy and potential),
  and the potential is d(rho eps_xc)/d rho (finite difference of the energy density).
* Methfessel-Paxton occupations: the product's calc_fermi_mp and the oracle's bisection give the
  same occupations and electron count for a gapped spectrum.
"""
import math

import numpy as np

from oracle import scf_oracle as so
from rsdft_develop_b200 import scf


def test_hartree_cosine_density():
    n, L = 16, 6.4
    x = np.arange(n) * (L / n)
    z3, y3, x3 = np.meshgrid(x, x, x, indexing="ij")
    G = 2 * math.pi / L * np.array([2, 1, 0])
    rho = np.cos(G[0] * x3 + G[1] * y3 + G[2] * z3).ravel()
    vh, _ = so.hartree(rho, n, L)
    assert np.allclose(vh, 4 * math.pi / float(G @ G) * rho, atol=1e-12)


def test_pz81_branches_and_potential():
    for pol in (0, 1):
        e_lo, v_lo = so.pz81_c(np.array([1.0 - 1e-12]), pol)
        e_hi, v_hi = so.pz81_c(np.array([1.0]), pol)
        assert abs(e_lo[0] - e_hi[0]) < 1e-4 and abs(v_lo[0] - v_hi[0]) < 2e-3
    rho = np.array([1e-3, 1e-2, 0.1, 1.0, 5.0])
    v, _, _ = so.lda_pz81(rho)
    h = 1e-6 * rho

    def edens(r):
        _, e, _ = so.lda_pz81(r)
        return e

    fd = np.array([(edens(np.array([r + d])) - edens(np.array([r - d]))) / (2 * d) for r, d in zip(rho, h)])
    assert np.allclose(v, fd, rtol=1e-6, atol=1e-9)


def test_mp_occupations_agree():
    rng = np.random.default_rng(3)
    esp = np.sort(rng.uniform(-1.0, 1.0, 20))
    esp[10:] += 0.3  # gap above band 10
    occ_p, ef_p = scf.calc_fermi_mp(esp[None, None, :], np.array([1.0]), 20.0)
    occ_o, ef_o = so.mp_occ(esp[None, None, :], [1.0], 20.0)
    assert abs(occ_p.sum() - 20.0) < 1e-9 and abs(occ_o.sum() - 20.0) < 1e-9
    assert np.allclose(occ_p, occ_o, atol=1e-9)
    assert np.allclose(occ_p[0, 0, :10], 2.0) and np.allclose(occ_p[0, 0, 10:], 0.0, atol=1e-12)
