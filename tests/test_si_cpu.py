"""The reference's Si sample (FCC cell, 12^3 grid, 63 k-points, PBE) against its own logs.

The set-up of rsdft_develop_b200.structure for a non-orthogonal cell on k-points (G sphere,
init_kinetic's metric and FD tables, analytic initial density, Ewald sum) must reproduce what
the reference printed; the oracle's complex16 band update on that operator (stencil with the
cross-derivative terms -ggg(4) D1 D2 - ggg(5) D2 D3 - ggg(6) D3 D1, projectors with the k phases
of prep_uvk_ps_nloc2) must reproduce the scf_iter 1 eigenvalues of every k-point; the k-point
SCF loop scf_structure.run_scf_kpoints must retrace the reference's iterations and land on the
converged energies, and the bands of
its potential along the band-structure trajectory on band_eigv (the total energy to 1e-9 Ha; it
lands within ~1e-14 Ha of the printed one).  Values come from the three
logs in tests/golden/reference_logs.json ("si", "si_band"; they agree to ~1e-8 Ha among
themselves in the kinetic / nonlocal split and to ~1e-9 Ha in the band energies).
"""
import dataclasses
import json
import math
import os

import numpy as np
import pytest

from rsdft_develop_b200 import pseudo, scf, scf_structure, structure, synth

HERE = os.path.dirname(__file__)


def _logs(key="si"):
    d = json.load(open(os.path.join(HERE, "golden", "reference_logs.json")))[key]
    assert len(d) >= 1
    return d


@pytest.fixture(scope="module")
def si():
    pp = pseudo.load_npz(os.path.join(HERE, "golden", "si_pbe_tm_psv.npz"))
    kbb, w = synth.generate_bz((5, 5, 5))
    return structure.setup(structure.si_crystal(pp, kbb, w))


def _oracle():
    from oracle import oracle as orc
    orc.set_threads(min(8, os.cpu_count() or 1))
    return orc


def test_si_pseudopotential_matches_reference_prints():
    pp = pseudo.load_npz(os.path.join(HERE, "golden", "si_pbe_tm_psv.npz"))
    for log in _logs():
        ps = log["psv"]
        assert pp.zps == ps["zps"] and pp.rad.size == ps["mr"] and abs(pp.rad[-1] - ps["r_end"]) < 1e-12
        assert list(pp.nrps) == ps["nrps"] and list(pp.lo) == ps["lo"]
        assert np.allclose(pp.rps, ps["rps"], rtol=1e-14) and np.allclose(pp.anorm, ps["anorm"], rtol=1e-14)
        assert np.allclose(pp.parloc, ps["parloc"], rtol=1e-14)


def test_si_setup_matches_reference_prints(si):
    st = si.structure
    gr = si.ggrid
    kin = si.problem.kin
    rho0 = pseudo.initial_density([(st.species[0][0], st.species[0][1])], st.n, st.avec)
    dV = si.problem.dV
    for log in _logs():
        assert abs(gr.ecut - log["ecut"]) < 1e-13 * log["ecut"] and abs(gr.gcut - log["gcut"]) < 1e-13 * log["gcut"]
        assert gr.ng == log["nggrid"] and gr.nmgl == log["nmgl"]
        assert np.allclose(kin["ggg"], log["ggg"], atol=1e-12)
        assert abs(kin["coef_lap0"] - log["lap_table"][0][2]) < 1e-12
        for row in log["lap_table"][1:]:
            assert np.allclose(kin["coef_lap"][:, row[0] - 1], row[2:], rtol=1e-13, atol=1e-15)
        for row in log["nab_table"]:
            assert np.allclose(kin["coef_nab"][:, row[0] - 1], row[2:], rtol=1e-13, atol=1e-15)
        raw, norm = log["initrho"]
        assert abs(rho0.sum() * dV - raw[1]) < 1e-9 and abs(rho0.min() - raw[2]) < 1e-10 and abs(rho0.max() - raw[3]) < 1e-10
        r = si.rho.sum(axis=0)
        assert abs(r.sum() * dV - norm[1]) < 1e-12 and abs(r.min() - norm[2]) < 1e-10 and abs(r.max() - norm[3]) < 1e-10
        assert abs(scf_structure.ewald_energy(st) - log["ewald"]) < 1e-12


def test_device_band_update_refuses_non_orthogonal_cells(si):
    """The CUDA stencil carries no cross-derivative terms: the host mirror refuses the FCC
    operator before it creates a library context."""
    from rsdft_develop_b200 import api
    with pytest.raises(NotImplementedError, match="non-orthogonal"):
        api.BandUpdate(si.problem)


def test_si_stencil_is_the_fd_symbol_of_the_fcc_metric(si):
    """A plane wave through the oracle's non-orthogonal k stencil (V = 0, no projectors) picks up
    coef_lap0 + k^2/2 + sum_d 2 (coef_lap cos + coef_nabk sin) + 4 sum_pairs ggg S_a S_b, and that
    symbol approaches |k + G|^2 / 2 as G -> 0."""
    orc = _oracle()
    prob = dataclasses.replace(si.problem, vloc=np.zeros(si.problem.ng))
    kin, n, md = prob.kin, prob.n, prob.md
    B = pseudo.reciprocal(si.structure.avec)
    i3, i2, i1 = np.meshgrid(*[np.arange(x) for x in n[::-1]], indexing="ij")
    for ik in (0, 20, 62):
        o = orc.Oracle(prob, k=ik, nonlocal_on=False)
        for m in (np.array([1, -2, 3]), np.array([0, 1, 0]), np.array([1, 1, -1])):
            psi = np.exp(2j * math.pi * (m[0] * i1 / n[0] + m[1] * i2 / n[1] + m[2] * i3 / n[2])).reshape(1, -1)
            th = 2.0 * math.pi * m / np.array(n)
            S = [sum(kin["coef_nab"][d, j - 1] * math.sin(j * th[d]) for j in range(1, md + 1)) for d in range(3)]
            sym = kin["coef_lap0"] + kin["const_k2"][ik]
            for d in range(3):
                for j in range(1, md + 1):
                    sym += 2.0 * (kin["coef_lap"][d, j - 1] * math.cos(j * th[d]) + kin["coef_nabk"][ik, d, j - 1] * math.sin(j * th[d]))
            g = kin["ggg"]
            sym += 4.0 * (g[3] * S[0] * S[1] + g[4] * S[1] * S[2] + g[5] * S[2] * S[0])
            assert np.max(np.abs(o.hpsi(psi) / psi - sym)) < 1e-12
            if np.abs(m).sum() == 1:
                kg = prob.kbb[ik] @ B + m @ B
                assert abs(sym - 0.5 * kg @ kg) < 1e-3 * (0.5 * kg @ kg)


def _converge(orc, prob, k, nband, nsweep, seed=1):
    o = orc.Oracle(prob, k=k)
    psi = o.gram_schmidt(synth.random_wavefunctions(seed + k, nband, prob.ng).astype(np.complex128))
    psi, _, _ = o.sweep(psi, nsweep)
    return o, psi


def test_si_oracle_eigenvalues_match_scf_iter1(si):
    """Bands 1-8 of the operator of the initial density at eight of the 63 k-points: within
    1e-9 Ha plus twice the change the reference printed beside each value (its own convergence
    estimate), and never above the printed value by more than 1e-12 (the printed values are
    upper bounds of partly converged Ritz values)."""
    orc = _oracle()
    prob = si.problem
    for k in (0, 1, 6, 19, 33, 44, 57, 62):
        o, psi = _converge(orc, prob, k, si.structure.nband, 30)
        e, res = o.residual(psi)
        assert np.max(res[:8]) < 1e-16, res[:8]
        for log in _logs():
            rows = [r for r in log["esp_scf1"] if r[0] == k + 1][:8]
            ref = np.array([r[2] for r in rows])
            err = np.array([abs(r[3]) for r in rows])
            assert np.all(np.abs(e[:8] - ref) <= 1e-9 + 2.0 * err), (k, e[:8] - ref, err)
            assert np.all(e[:8] <= ref + 1e-12), (k, e[:8] - ref)


class OracleBandsK:
    """The oracle's FP64 complex16 band update for every (k, s) behind run_scf_kpoints' interface."""

    def __init__(self, su, orc, seed=1, klist=None):
        self.su, self.orc = su, orc
        p = su.problem
        self.klist = list(range(p.nk)) if klist is None else list(klist)
        self.ns, self.nk = su.structure.nspin, len(self.klist)
        self.v = su.vloc.copy()
        self.psi = {}
        for s in range(self.ns):
            for j, k in enumerate(self.klist):
                o = orc.Oracle(p, k=k)
                self.psi[s, j] = o.gram_schmidt(
                    synth.random_wavefunctions(seed + k, su.structure.nband, p.ng).astype(np.complex128))

    def set_vloc(self, v):
        self.v = v.copy()

    def sweep(self, n, diag_first=False):
        esp = np.zeros((self.ns, self.nk, self.su.structure.nband))
        for s in range(self.ns):
            pr = dataclasses.replace(self.su.problem, vloc=np.ascontiguousarray(self.v[s]))
            for j, k in enumerate(self.klist):
                o = self.orc.Oracle(pr, k=k)
                if diag_first:
                    self.psi[s, j], _ = o.subspace_diag(self.psi[s, j])
                self.psi[s, j], _, _ = o.sweep(self.psi[s, j], n)
                esp[s, j], _ = o.residual(self.psi[s, j])
        return esp

    def bands(self, s, k):
        p = self.psi[s, k]
        return p / np.sqrt(np.sum(np.abs(p) ** 2, axis=1) * self.su.problem.dV)[:, None]

    def density(self, occ):
        return np.array([sum(np.sum(occ[s, k][:, None] * np.abs(self.bands(s, k)) ** 2, axis=0)
                             for k in range(self.nk)) for s in range(self.ns)])


@pytest.fixture(scope="module")
def si_scf(si):
    orc = _oracle()
    bands = OracleBandsK(si, orc)
    res = scf_structure.run_scf_kpoints(si, bands, nsweep=10, diter=40, scf_conv=1e-15)
    return res, bands


def test_si_scf_reaches_the_reference_state(si, si_scf):
    """The total energy is stationary at the fixed point and must agree to 1e-9 Ha (it agrees to
    ~1e-13).  The separate terms are first order in the density: the reference stops when its
    last step still moves the density by 6e-9 rms per point and V_loc by 3e-8 Ha rms (it prints
    |rho - rho0|^2 = 3.8e-17, |Vloc - Vloc0|^2 = 9.4e-16), which leaves its ion-local and
    nonlocal terms uncertain at the 1e-7 Ha level; they agree to 6e-7 Ha (the kinetic, Hartree
    and exchange-correlation terms to ~5e-8), the eigenvalues of the last iteration to 1e-7 Ha."""
    res, _ = si_scf
    assert res.converged, (res.iterations, res.sqerr[-3:])
    evb = float(np.max(res.esp[0, :, 3]))
    ecb = float(np.min(res.esp[0, :, 4]))
    assert evb < res.energies["fermi"] < ecb
    for log in _logs():
        ref = log["energies"]
        assert abs(res.energies["total"] - ref["total"]) < 1e-9, (res.energies["total"], ref["total"])
        assert abs(res.energies["harris"] - ref["harris"]) < 1e-9, (res.energies["harris"], ref["harris"])
        assert abs(res.energies["ewald"] - ref["ewald"]) < 1e-12
        for key in ("kinetic", "hartree", "xc", "exchange", "correlation", "ion_local", "local", "nonlocal",
                    "sum_eigen"):
            assert abs(res.energies[key] - ref[key]) < 6e-7, (key, res.energies[key], ref[key], log["source"])
        last = np.array([r[2] for r in log["esp_last"]]).reshape(63, 9)[:, :8]
        assert np.max(np.abs(res.esp[0, :, :8] - last)) < 1e-7
        # the printed entropy is entropy_fd of the weighted occupations at EKBT 1e-5 (nonzero for
        # an insulator: S is taken of f w_k), and Free Energy = Etot - entropy
        ent = scf.entropy_fd(1e-5, res.occ)
        assert abs(ent - ref["entropy"]) < 1e-12, (ent, ref["entropy"])
        assert abs(res.energies["total"] - ent - ref["free"]) < 1e-9


def test_si_scf_follows_the_reference_iterations(si_scf):
    """The loop runs the reference's order (Rayleigh-Ritz on the new potential, one sweep,
    occupations, density, potential, calc_sqerr, IMIX = 10 Pulay with its beta search) and
    retraces its printed squared changes of V_loc: the first to its 6 printed digits (it only
    depends on the initial-density operator), the next three within 5 % (they depend on the
    partly converged bands of 10 sweeps from random starts), the jump when the Pulay history
    fills within 25 %, and reaches the reference's stop (<= 1e-15) within two iterations of its
    15."""
    res, _ = si_scf
    ours = [h[0] for h in res.sqerr]
    for log in _logs():
        ref = log["sqerr_v"]
        assert abs(ours[0] - ref[0]) <= 1e-5 * ref[0], (ours[0], ref[0])
        for i in (1, 2, 3):
            assert abs(ours[i] - ref[i]) <= 0.05 * ref[i], (i, ours[i], ref[i])
        assert abs(ours[4] - ref[4]) <= 0.25 * ref[4], (ours[4], ref[4])
        n_ours = next(i + 1 for i, v in enumerate(ours) if v <= 1e-15)
        assert abs(n_ours - log["iterations"]) <= 2, (n_ours, log["iterations"])


def test_si_band_structure_of_the_converged_potential(si, si_scf):
    """Bands 1-12 at six points of the band_eigv trajectory (Gamma, X, L and between) with the
    converged SCF potential, against the band energies the reference wrote.  The reference stops
    its band sweeps once no eigenvalue changes by more than esp_conv_tol = 1e-7 Ha per sweep, so
    its values are upper bounds within 1e-6 Ha; ours (residual < 1e-16) must lie below them up to
    1e-7 Ha, the eigenvalue agreement of the two converged SCF potentials."""
    orc = _oracle()
    res, bands = si_scf
    traj = _logs("si_band")[0]
    pick = [0, 10, 20, 25, 35, 45]
    kbb = np.array([traj["kpoints"][i] for i in pick])
    st = dataclasses.replace(si.structure, kbb=kbb, wbz=np.full(len(pick), 1.0 / len(pick)), nband=16)
    su = structure.setup(st)
    prob = dataclasses.replace(su.problem, vloc=np.ascontiguousarray(bands.v[0]))
    for j, i in enumerate(pick):
        o, psi = _converge(orc, prob, j, 16, 40)
        e, res = o.residual(psi)
        assert np.max(res[:12]) < 1e-16, res[:12]
        for t in _logs("si_band"):
            assert np.allclose(t["kpoints"][i], kbb[j], atol=1e-12)
            d = e[:12] - np.array(t["esp"][i])
            assert np.all(d < 1e-7) and np.all(d > -1e-6), (i, d)


def test_si_gamma_real8_operator_matches_the_complex16_one(si):
    """The real8 build at Gamma (real bands, the real stencil path with the cross terms, projectors
    without phases) gives the Gamma eigenvalues of the complex16 k-point set."""
    orc = _oracle()
    pp = pseudo.load_npz(os.path.join(HERE, "golden", "si_pbe_tm_psv.npz"))
    st = structure.si_crystal(pp)
    su = structure.setup(st)
    assert not su.problem.is_complex and abs(su.problem.kin["ggg"][3] + 0.5) < 1e-12
    prob = dataclasses.replace(su.problem, vloc=np.ascontiguousarray(si.vloc[0]))
    o = orc.Oracle(prob)
    psi = o.gram_schmidt(synth.random_wavefunctions(3, 16, prob.ng))
    psi, _, _ = o.sweep(psi, 30)
    e_r, res = o.residual(psi)
    assert np.max(res[:8]) < 1e-16
    oc, psic = _converge(orc, si.problem, 0, 16, 30)
    e_c, _ = oc.residual(psic)
    assert np.max(np.abs(e_r[:8] - e_c[:8])) < 1e-11, e_r[:8] - e_c[:8]


def test_si_two_spin_scf_equals_the_one_spin_scf():
    """nspin = 2 with no initial moment (the initial density split in halves, occupations
    Methfessel-Paxton over both spins) converges to the spin-unpolarised state: equal spin
    densities, the one-spin total energy and eigenvalues (2 x 2 x 2 mesh, 8 bands)."""
    orc = _oracle()
    pp = pseudo.load_npz(os.path.join(HERE, "golden", "si_pbe_tm_psv.npz"))
    kbb, w = synth.generate_bz((2, 2, 2))
    out = []
    for ns in (1, 2):
        st = dataclasses.replace(structure.si_crystal(pp, kbb, w, nband=8), nspin=ns)
        su = structure.setup(st)
        res = scf_structure.run_scf_kpoints(su, OracleBandsK(su, orc), nsweep=8, diter=30, scf_conv=1e-14)
        assert res.converged, (ns, res.sqerr[-2:])
        out.append(res)
    one, two = out
    assert np.max(np.abs(two.rho[0] - two.rho[1])) < 1e-9
    assert abs(two.energies["total"] - one.energies["total"]) < 1e-9
    assert np.max(np.abs(two.esp[0] - one.esp[0])) < 1e-8 and np.max(np.abs(two.esp[1] - one.esp[0])) < 1e-8


def test_si_other_mixing_schemes_reach_the_pulay_state():
    """IMIX = 20 (Broyden of the density), 11 (Pulay of the potential) and 30 (Pulay of the
    density's Fourier coefficients with the Kerker weights) converge the Si
    operator on the 2 x 2 x 2 mesh to the state of the default IMIX = 10 (Pulay of the density):
    the same total energy and eigenvalues (bands 1-6; the top two of the eight carried bands
    converge slowest in a one-sweep-per-iteration SCF)."""
    orc = _oracle()
    pp = pseudo.load_npz(os.path.join(HERE, "golden", "si_pbe_tm_psv.npz"))
    kbb, w = synth.generate_bz((2, 2, 2))
    su = structure.setup(structure.si_crystal(pp, kbb, w, nband=8))
    out = {}
    for imix in (10, 20, 11, 30):
        res = scf_structure.run_scf_kpoints(su, OracleBandsK(su, orc), nsweep=8, diter=40, scf_conv=1e-14,
                                            imix=imix)
        assert res.converged, (imix, res.sqerr[-2:])
        out[imix] = res
    for imix in (20, 11, 30):
        assert abs(out[imix].energies["total"] - out[10].energies["total"]) < 1e-10, imix
        assert np.max(np.abs(out[imix].esp[:, :, :6] - out[10].esp[:, :, :6])) < 1e-7, imix
