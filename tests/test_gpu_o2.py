"""The CUDA band update on the reference's O2 sample operator, against the reference's own logs.

The operator (PBE, two spins, 48^3 grid, filtered KB projectors of O_PBE_RC1.5.psv, potential
of the initial density) is built on the host by rsdft_develop_b200.structure from the fixture
tests/golden/o_pbe_rc15_psv.npz; both spins run in one context (nspin = 2, Vloc per spin).  The
converged band energies must match the values the reference printed at scf_iter 1 in all eight
O2 logs (tests/golden/reference_logs.json): bands 1-5 to 1e-10 Ha, the pi* pair (bands 6-7,
logged before it had fully converged) to 3e-8 Ha.  FP64 directly; mixed precision after its FP64
polish, and within 1e-6 Ha before it; the complex16 build at Gamma in FP64.  The device density of
the FP64 bands with scf_iter 1's occupations matches that iteration's printed charges, spin
density sum and squared density change.
"""
import json
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


def _logs():
    return json.load(open(os.path.join(HERE, "golden", "reference_logs.json")))["o2"]


def _check(esp, tol15=1e-10, tol67=3e-8):
    for log in _logs():
        for s in (1, 2):
            col = 2 if s == 1 else 5
            ref = np.array([r[col] for r in log["esp_scf1"][:7]])
            got = esp[s - 1, 0, :7]
            assert np.max(np.abs(got[:5] - ref[:5])) < tol15, (s, log["source"], got[:5] - ref[:5])
            assert np.max(np.abs(got[5:7] - ref[5:7])) < tol67, (s, log["source"], got[5:7] - ref[5:7])


def _check_density(g, o2):
    """The device density of the converged bands with scf_iter 1's occupations (7 up, 5 down)
    against what that iteration prints (tolerances as in test_pseudo_cpu.py)."""
    occ = np.zeros((2, 1, o2.problem.nband))
    occ[0, 0, :7] = 1.0
    occ[1, 0, :5] = 1.0
    g.density(occ)
    rho = g.get_rho()[0]
    dV = o2.problem.dV
    vh, _ = gga.hartree_sphere(rho.sum(axis=0), o2.ggrid, dV)
    vxc, _, _ = gga.pbe(rho, o2.problem.n, (o2.problem.h,) * 3, dV)
    sq_v = np.sum((o2.vion[None, :] + vh[None, :] + vxc - o2.vloc) ** 2, axis=1) / rho.shape[1]
    sq_rho = np.sum((rho - o2.rho) ** 2, axis=1) / rho.shape[1]
    spin = float(np.sum(np.abs(rho[0] - rho[1]))) * dV
    for log in _logs():
        assert np.allclose(rho.sum(axis=1) * dV, log["charge_scf1"], atol=1e-11)
        assert abs(spin - log["sum_abs_spin_scf1"]) < 1e-7, (spin, log["sum_abs_spin_scf1"])
        assert np.allclose(sq_rho, log["sqerr_rho_scf1"], rtol=1e-5, atol=0), (sq_rho, log["sqerr_rho_scf1"])
        assert np.allclose(sq_v, log["sqerr_v_scf1"], rtol=1e-2, atol=0), (sq_v, log["sqerr_v_scf1"])


def _start(g, o2):
    g.set_vloc(o2.vloc[1], s=2)
    g.init_sweep(7)
    for s in (1, 2):
        g.random_wf(1, s=s)
        g.gram_schmidt(s=s)


def test_o2_fp64_band_energies_match_reference_logs(o2):
    with api.BandUpdate(o2.problem_for_spin(1), precision=api.PREC_FP64, nspin=2) as g:
        _start(g, o2)
        it, esp, res = g.calc_sweep(80, tol=1e-18)
        assert np.max(res[:, 0, :7]) <= 1e-18, (it, res[:, 0, :7])
        _check(esp)
        _check_density(g, o2)


def test_o2_complex16_build_band_energies_match_reference_logs():
    """The complex16 build at the Gamma point (the reference's complex16 O2 runs print the same
    energies): complex bands, projectors with unit phases."""
    pp = pseudo.load_npz(os.path.join(HERE, "golden", "o_pbe_rc15_psv.npz"))
    o2c = structure.setup(structure.o2_molecule(pp), complex16=True)
    assert o2c.problem.is_complex
    with api.BandUpdate(o2c.problem_for_spin(1), precision=api.PREC_FP64, nspin=2) as g:
        _start(g, o2c)
        it, esp, res = g.calc_sweep(80, tol=1e-18)
        assert np.max(res[:, 0, :7]) <= 1e-18, (it, res[:, 0, :7])
        _check(esp)


def test_o2_mixed_precision_then_fp64_polish(o2):
    with api.BandUpdate(o2.problem_for_spin(1), precision=api.PREC_MIXED, nspin=2) as g:
        _start(g, o2)
        it, esp, res = g.calc_sweep(80, tol=1e-9)
        assert np.max(res[:, 0, :7]) <= 1e-9, (it, res[:, 0, :7])
        _check(esp, tol15=1e-6, tol67=1e-6)
        g.set_precision(api.PREC_FP64)
        it2, esp, res = g.calc_sweep(40, tol=1e-18)
        assert np.max(res[:, 0, :7]) <= 1e-18, (it2, res[:, 0, :7])
        _check(esp)


def test_o2_scf_on_the_gpu_reaches_the_reference_state(o2):
    """The SCF loop for PSV structures (rsdft_develop_b200.scf_structure) with the CUDA band
    update, FP64: the converged energy terms, eigenvalues and spin-density sum of the reference's
    first O2 SCF cycle (tolerances of tests/test_scf_structure_cpu.py)."""
    from rsdft_develop_b200 import scf_structure
    from tests.test_scf_structure_cpu import check_against_logs
    import time
    bands = scf_structure.GpuBands(o2, precision=api.PREC_FP64)
    try:
        t0 = time.perf_counter()
        res = scf_structure.run_scf_structure(o2, bands, nsweep=10, diter=60)
        wall = time.perf_counter() - t0
    finally:
        bands.close()
    print(f"O2 SCF on the GPU: {res.iterations} iterations in {wall:.2f} s, total energy "
          f"{res.energies['total']:.10f} Ha")
    check_against_logs(res)
