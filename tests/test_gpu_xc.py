"""The device GGA-PBE potential (rsdft_gpu_xc_pbe) against the host restatement gga.pbe.

Both restate calc_GGAPBE96_2 (src/xc/xc_ggapbe96_2_module.f90:26-370); gga.pbe is the one the
O2 tests pin to the reference's logs.  Cases: the O2 sample's initial density (two spins, a
vacuum region where densities fall below the 1e-10 cut), its total density as one spin, and a
two-spin density with uneven spin channels and exact zeros.  V_xc to 1e-11 of its largest
value, E_x and E_c to 1e-12 relative.
"""
import os

import numpy as np
import pytest

from rsdft_develop_b200 import api, gga, pseudo, structure

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(__file__)


@pytest.fixture(scope="module")
def o2():
    pp = pseudo.load_npz(os.path.join(HERE, "golden", "o_pbe_rc15_psv.npz"))
    return structure.setup(structure.o2_molecule(pp))


def _compare(prob, rho):
    ns = rho.shape[0]
    v_ref, ex_ref, ec_ref = gga.pbe(rho, prob.n, (prob.h,) * 3, prob.dV, prob.md)
    with api.BandUpdate(prob, nspin=ns) as g:
        for _ in range(2):                      # the second call reuses the device buffers
            v, ex, ec = g.xc_pbe(rho)
            assert np.max(np.abs(v - v_ref)) <= 1e-11 * np.max(np.abs(v_ref)), np.max(np.abs(v - v_ref))
            assert abs(ex - ex_ref) <= 1e-12 * abs(ex_ref) and abs(ec - ec_ref) <= 1e-12 * abs(ec_ref)


def test_xc_pbe_two_spins_o2_initial_density(o2):
    _compare(o2.problem, o2.rho)


def test_xc_pbe_one_spin(o2):
    _compare(o2.problem, o2.rho.sum(axis=0, keepdims=True))


def test_xc_pbe_uneven_spins_with_zeros(o2):
    rng = np.random.default_rng(5)
    rho = o2.rho.copy()
    rho[1] *= np.exp(rng.normal(scale=0.3, size=rho.shape[1]))
    rho[:, ::7] = 0.0
    rho[1, ::11] = 0.0
    _compare(o2.problem, rho)
