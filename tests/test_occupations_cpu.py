"""Fermi-Dirac occupations and entropy (src/fermi_dirac_module.f90) beside the default
Methfessel-Paxton ones (calc_fermi_mp), on synthetic band energies and in the k-point SCF."""
import os

import numpy as np

from rsdft_develop_b200 import pseudo, scf, scf_structure, structure, synth

HERE = os.path.dirname(__file__)


def _bands(ns=1, nk=5, nb=8, seed=0, gap=0.0):
    rng = np.random.default_rng(seed)
    e = np.sort(rng.uniform(-0.5, 0.5, size=(ns, nk, nb)), axis=2)
    e[:, :, 4:] += gap
    w = rng.uniform(0.5, 1.5, nk)
    return e, w / w.sum()


def test_fermi_dirac_counts_electrons_and_orders_occupations():
    for ns in (1, 2):
        e, w = _bands(ns=ns)
        for ekbt in (1e-3, 1e-2, 0.05):
            occ, ef = scf.fermi_dirac(e, w, 7.3, ekbt)
            assert abs(occ.sum() - 7.3) < 1e-9
            f = occ / (w[None, :, None] * 2.0 / ns)
            order = np.argsort(e, axis=None)
            assert np.all(np.diff(f.ravel()[order]) <= 1e-9)        # non-increasing in energy
            assert np.all((f > -1e-9) & (f < 1 + 1e-9))


def test_fermi_dirac_at_small_temperature_is_the_mp_filling_of_a_gapped_spectrum():
    e, w = _bands(gap=0.3)
    occ_fd, ef_fd = scf.fermi_dirac(e, w, 8.0, 1e-4)
    occ_mp, _ = scf.calc_fermi_mp(e, w, 8.0, 1e-5, 5)
    assert np.max(np.abs(occ_fd - occ_mp)) < 1e-12
    assert e[:, :, 3].max() < ef_fd < e[:, :, 4].min()


def test_entropy_fd_formula():
    """S is taken of the weighted occupation occ ns / 2 (= f w_k), as the reference evaluates it:
    with weight 1 that is f, and a filled state of weight w < 1 still contributes S(w)."""
    occ = np.array([[[1.0, 0.5, 0.0]]]) * 2.0          # one k (weight 1), one spin: f = 1, 1/2, 0
    assert abs(scf.entropy_fd(0.01, occ) - 2.0 * 0.01 * np.log(2.0)) < 1e-15
    w = 0.25
    occ = np.array([[[2.0 * w]]])                        # one filled state of weight 1/4
    sw = -w * np.log(w) - (1 - w) * np.log(1 - w)
    assert abs(scf.entropy_fd(0.01, occ) - 2.0 * 0.01 * sw) < 1e-15


def test_si_scf_with_fermi_dirac_occupations():
    """The Si operator (2 x 2 x 2 mesh) with Fermi-Dirac occupations at kT = 1e-3 Ha converges to
    the Methfessel-Paxton state of the insulator: the conduction bands take ~e^-20 electrons."""
    from oracle import oracle as orc
    from tests.test_si_cpu import OracleBandsK
    orc.set_threads(4)
    pp = pseudo.load_npz(os.path.join(HERE, "golden", "si_pbe_tm_psv.npz"))
    kbb, w = synth.generate_bz((2, 2, 2))
    su = structure.setup(structure.si_crystal(pp, kbb, w, nband=8))
    out = {}
    for occ in ("mp", "fd"):
        res = scf_structure.run_scf_kpoints(su, OracleBandsK(su, orc), nsweep=8, diter=30, scf_conv=1e-14,
                                            occupations=occ, ekbt=1e-3 if occ == "fd" else 1e-5)
        assert res.converged, (occ, res.sqerr[-2:])
        out[occ] = res
    assert abs(out["fd"].energies["total"] - out["mp"].energies["total"]) < 1e-8
    assert abs(out["fd"].energies["entropy"] - scf.entropy_fd(1e-3, out["fd"].occ)) < 1e-15
    assert abs(out["fd"].energies["free"] - (out["fd"].energies["total"] - out["fd"].energies["entropy"])) < 1e-15
    assert abs(out["fd"].occ.sum() - 8.0) < 1e-9


def test_lda_pz81_against_the_oracle_and_its_spin_limits():
    """gga.lda_pz81 (calc_LDAPZ81 with spin) equals the oracle's unpolarised PZ81, two equal spin
    halves equal one spin, and V_xc is the derivative of E_xc in the polarised case."""
    from oracle import scf_oracle
    from rsdft_develop_b200 import gga
    rng = np.random.default_rng(0)
    rho = rng.uniform(0.0, 2.0, 4000) ** 3                 # rs on both sides of 1
    v, ex, ec = gga.lda_pz81(rho[None, :], 1.0)
    vo, exc_o, _ = scf_oracle.lda_pz81(rho)
    assert np.max(np.abs(v[0] - vo)) < 1e-13 and abs(ex + ec - exc_o) < 1e-10
    v2, ex2, ec2 = gga.lda_pz81(np.stack([rho / 2, rho / 2]), 1.0)
    assert np.max(np.abs(v2 - v)) < 1e-13 and abs(ex2 + ec2 - ex - ec) < 1e-10
    r = np.stack([rng.uniform(0.01, 1.0, 50), rng.uniform(0.01, 1.0, 50)])
    v, _, _ = gga.lda_pz81(r, 1.0)
    for s in (0, 1):
        d = np.zeros_like(r)
        d[s] = 1e-6 * r[s]
        ep = sum(gga.lda_pz81(r + d, 1.0)[1:])
        em = sum(gga.lda_pz81(r - d, 1.0)[1:])
        # E is a sum over points: dE/d(rho_s(i)) at every point at once via a common relative step
        assert abs((ep - em) / 2.0 - float(np.sum(v[s] * d[s]))) < 1e-9


def test_si_scf_with_lda():
    """XCtype LDAPZ81 (the reference's default) in the structure set-up and the k-point SCF."""
    from oracle import oracle as orc
    from tests.test_si_cpu import OracleBandsK
    import dataclasses
    orc.set_threads(4)
    pp = pseudo.load_npz(os.path.join(HERE, "golden", "si_pbe_tm_psv.npz"))
    kbb, w = synth.generate_bz((2, 2, 2))
    st = dataclasses.replace(structure.si_crystal(pp, kbb, w, nband=8), xc="LDAPZ81")
    su = structure.setup(st)
    res = scf_structure.run_scf_kpoints(su, OracleBandsK(su, orc), nsweep=8, diter=30, scf_conv=1e-14)
    assert res.converged
    pbe = structure.setup(structure.si_crystal(pp, kbb, w, nband=8))
    assert np.max(np.abs(su.vxc - pbe.vxc)) > 1e-3            # a different functional
    assert -8.0 < res.energies["total"] < -7.7


def test_fixed_moment_occupations():
    """calc_fermi_mp's fixed-moment branch: N/2 + dspn/2 electrons in spin 1 and N/2 - dspn/2 in
    spin 2, each to its own level; on a spectrum with a gap in each spin channel this is the
    integer filling the O2 loop uses (7 up, 5 down for 12 electrons and a moment of 2)."""
    rng = np.random.default_rng(7)
    e = np.sort(rng.uniform(-1.0, 0.0, size=(2, 1, 18)), axis=2)
    e[0, :, 7:] += 0.5
    e[1, :, 5:] += 0.5
    occ, (ef_up, ef_dn) = scf.calc_fermi_mp_fixed(e, np.array([1.0]), 12.0, 2.0)
    want = np.zeros((2, 1, 18))
    want[0, 0, :7] = 1.0
    want[1, 0, :5] = 1.0
    assert np.max(np.abs(occ - want)) < 1e-12
    assert e[0, 0, 6] < ef_up < e[0, 0, 7] and e[1, 0, 4] < ef_dn < e[1, 0, 5]
    e2, w2 = _bands(ns=2, nk=4)
    occ, _ = scf.calc_fermi_mp_fixed(e2, w2, 7.0, 1.0, 1e-2)
    assert abs(occ[0].sum() - 4.0) < 1e-10 and abs(occ[1].sum() - 3.0) < 1e-10
