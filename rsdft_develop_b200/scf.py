"""SCF outer loop over the C ABI: the caller of the band update.

Reference: calc_scf (src/scf_module.f90:85-563) with its defaults: XCtype LDAPZ81, IMIX = 10
(Pulay mixing of the density, MMIX = 4, BETA = 1.1 with the beta search of perform_mixing),
Methfessel-Paxton occupations of order KINTEG = 5 with EKBT = 1e-5 (calc_fermi_mp,
src/fermi_module.f90:108-262, ff0 :284-302, get_ef :305-345), Ndiag = 1.  One SCF iteration:

  per (k, s): subspace_diag, then conjugate_gradient -> gram_schmidt -> subspace_diag (one sweep)
  calc_fermi -> occ;  calc_density;  calc_hartree + calc_xc -> Vloc of the new density
  calc_sqerr of (Vloc, rho) against the last mixed pair -> converged when
      max sqerr(Vloc) <= scf_conv[0] or max sqerr(rho) <= scf_conv[1]
  otherwise perform_mixing (rho <- Pulay mix), normalize_density, Hartree + XC -> Vloc

The band update, density, Poisson solve, XC, potential update and the mixing vector operations
run on the GPU (csrc/scf.cu and the band-update kernels); the occupations (a bisection over
band energies) and the 4 x 4 Pulay system are host work, as in the reference.  Synthetic inputs:
V_ion is the configuration's Gaussian V_loc; the start is the uniform density of nelec electrons.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import api, synth


def _mp_factors(kinteg: int) -> np.ndarray:
    """A_n = (-1)^n / (n! 4^n sqrt(pi)), the Methfessel-Paxton coefficients (prep_ff0)."""
    return np.array([(-1) ** n / (math.factorial(n) * 4 ** n * math.sqrt(math.pi)) for n in range(1, kinteg + 1)])


def ff0(kinteg: int, x: np.ndarray) -> np.ndarray:
    """Methfessel-Paxton occupation of order kinteg at x = (e - ef) / ekbt (fermi_module ff0)."""
    x = np.asarray(x, dtype=np.float64)
    erf = np.vectorize(math.erf)
    f = 0.5 * (1.0 - erf(x))
    if kinteg <= 0:
        return f
    fac = _mp_factors(kinteg)
    hp0 = np.ones_like(x)
    hp1 = 2.0 * x
    ff = fac[0] * hp1
    for i in range(2, kinteg + 1):
        hp2 = 2.0 * x * hp1 - 2.0 * (2 * i - 3) * hp0
        hp3 = 2.0 * x * hp2 - 2.0 * (2 * i - 2) * hp1
        ff = ff + fac[i - 1] * hp3
        hp0, hp1 = hp2, hp3
    return f + ff * np.exp(-x * x)


def _get_ef(nelec: float, esp: np.ndarray, wbz: np.ndarray, msp: int) -> float:
    """Initial Fermi level: fill levels in increasing order (fermi_module get_ef)."""
    ns, nk, nb = esp.shape
    order = np.argsort(esp, axis=None, kind="stable")
    e1 = float(esp.min())
    count = 0.0
    for flat in order:
        s, k, n = np.unravel_index(flat, esp.shape)
        e2 = float(esp[s, k, n])
        for _ in range(2 // msp):
            count += float(wbz[k])
            if abs(count - nelec) < 1e-10:
                return e2
            if count > nelec:
                return 0.5 * (e1 + e2)
        e1 = e2
    return float(esp.max())


def calc_fermi_mp(esp: np.ndarray, wbz: np.ndarray, nelec: float, ekbt: float = 1e-5, kinteg: int = 5):
    """Occupations occ(s, k, n) (weights wbz(k) and 2/MSP included) and the Fermi level
    (calc_fermi_mp, spin-unpolarised or MSP = 2 with the total electron count)."""
    ns = esp.shape[0]
    oc0 = 2.0 / ns
    w = np.asarray(wbz)[None, :, None]

    def nel(ef):
        return float(np.sum(ff0(kinteg, (esp - ef) / ekbt) * w * oc0))

    ef = _get_ef(nelec, esp, np.asarray(wbz), ns)
    mergin = 0.0004
    for loop in range(1, 1000001):
        ef1, ef2 = ef - loop * mergin, ef + loop * mergin
        if (nelec - nel(ef1)) * (nelec - nel(ef2)) <= 0.0:
            break
    ef0 = 1e10
    occ = None
    for _ in range(1000000):
        ef = 0.5 * (ef1 + ef2)
        if ef == ef0:
            break
        occ = ff0(kinteg, (esp - ef) / ekbt) * w * oc0
        d = float(occ.sum()) - nelec
        if d > 1e-12:
            ef2 = ef
        elif d < -1e-12:
            ef1 = ef
        else:
            break
        ef0 = ef
    return occ, ef


def calc_fermi_mp_fixed(esp: np.ndarray, wbz: np.ndarray, nelec: float, dspn: float, ekbt: float = 1e-5,
                        kinteg: int = 5):
    """The fixed-moment branch of calc_fermi_mp (src/fermi_module.f90:187-238, iterations up to
    NFIXED with two spins): each spin s has its own Fermi level for N_s = Nelectron / 2 +- Ndspin
    / 2 electrons (+ for spin 1), found by the same bracket-and-bisect search; occupations carry
    the k weights (one electron per state).  Returns (occ (2, nk, nb), (ef_up, ef_down))."""
    esp = np.asarray(esp, np.float64)
    if esp.shape[0] != 2:
        raise ValueError("a fixed moment needs two spins")
    occ = np.zeros_like(esp)
    efs = []
    for s in range(2):
        zne = 0.5 * nelec + (1.0 if s == 0 else -1.0) * 0.5 * dspn
        e = esp[s:s + 1]
        w = np.asarray(wbz, np.float64)[None, :, None]

        def nel(ef):
            return float(np.sum(ff0(kinteg, (e - ef) / ekbt) * w))

        ef = _get_ef(zne, e, np.asarray(wbz), 2)
        for loop in range(1, 1000001):
            ef1, ef2 = ef - loop * 0.0004, ef + loop * 0.0004
            if (zne - nel(ef1)) * (zne - nel(ef2)) <= 0.0:
                break
        for _ in range(1000000):
            ef = 0.5 * (ef1 + ef2)
            o = ff0(kinteg, (e - ef) / ekbt) * w
            d = float(o.sum()) - zne
            if d > 1e-12:
                ef2 = ef
            elif d < -1e-12:
                ef1 = ef
            else:
                break
            if 0.5 * (ef1 + ef2) in (ef1, ef2):      # the bracket cannot shrink further
                break
        occ[s] = o[0]
        efs.append(ef)
    return occ, tuple(efs)


def fermi_dirac(esp: np.ndarray, wbz: np.ndarray, nelec: float, ekbt: float):
    """Fermi-Dirac occupations occ(s, k, n) (weights and 2/nspin included) and the Fermi level:
    fermi_dirac without the fixed-spin branch (src/fermi_dirac_module.f90:11-250): bisection of
    the level on the bands mb1.. (100 cycles, tolerance 1e-10 on the electron count, the upper
    bound raised by min(100 ekbt, 0.1)); if it does not settle, the lowest band is taken as
    filled and the search repeats on the bands above; f = 1 / (exp(x) + 1) with x = (e - ef) /
    ekbt cut at |x| > 36.9 (a step function for ekbt < 1e-10); the remaining electron-count
    error is added to the highest occupied band of every (k, s)."""
    esp = np.asarray(esp, np.float64)
    ns, nk, nb = esp.shape
    w = np.asarray(wbz, np.float64)[None, :, None] * (2.0 / ns)
    eps, big = 1e-10, 36.9

    def ff(e, ef):
        if ekbt < eps:
            return np.where(e - ef > 0.0, 0.0, np.where(e - ef < 0.0, 1.0, 0.5))
        x = (e - ef) / ekbt
        with np.errstate(over="ignore"):
            return np.where(x > big, 0.0, np.where(x < -big, 1.0, 1.0 / (np.exp(np.clip(x, -big, big)) + 1.0)))

    if abs(2 * nb - nelec) < eps:
        return np.ones_like(esp) * w, float(esp.max())
    for mb1 in range(nb):
        sub = esp[:, :, mb1:]
        ef1, ef2 = float(sub.min()), float(sub.max())
        if ef1 == ef2:
            ef1, ef2 = ef1 - 0.01, ef2 + 0.01
        ef2 += min(ekbt * 1e2, 0.1)
        zne = nelec - 2.0 * mb1
        found = False
        for _ in range(100):
            ef = 0.5 * (ef1 + ef2)
            f = ff(sub, ef)
            n = float(np.sum(f * w))
            if n - zne > eps:
                ef2 = ef
            elif n - zne < -eps:
                ef1 = ef
            else:
                found = True
                break
        if found:
            occ = np.zeros_like(esp)
            occ[:, :, :mb1] = np.broadcast_to(w, (ns, nk, mb1))
            occ[:, :, mb1:] = f * w
            err = nelec - float(occ.sum())
            if abs(err) > 0.0:
                for s in range(ns):
                    for k in range(nk):
                        pos = np.nonzero(occ[s, k, mb1:] > 0.0)[0]
                        if pos.size:
                            occ[s, k, mb1 + pos[-1]] += err / (nk * ns)
            return occ, ef
    raise RuntimeError("fermi_dirac: the Fermi level did not settle (the reference stops with FERMI(1))")


def entropy_fd(ekbt: float, occ: np.ndarray) -> float:
    """entropy_fd (src/fermi_dirac_module.f90:330-351) as the reference evaluates it on the
    weighted occupations: sum over (s, k, n) of (2 / ns) ekbt S(f) with f = occ ns / 2 and
    S(f) = -f ln f - (1 - f) ln(1 - f)."""
    ns = occ.shape[0]
    f = occ * (ns / 2.0)
    g = 1.0 - f
    with np.errstate(divide="ignore", invalid="ignore"):
        sf = -np.where(f > 0.0, f * np.log(np.where(f > 0.0, f, 1.0)), 0.0) \
             - np.where(g > 0.0, g * np.log(np.where(g > 0.0, g, 1.0)), 0.0)
    return float(np.sum((2.0 / ns) * ekbt * sf))


@dataclasses.dataclass
class ScfResult:
    iterations: int
    converged: bool
    esp: np.ndarray           # (nspin, nk, mb) band energies of the last iteration
    occ: np.ndarray           # (nspin, nk, mb)
    efermi: float
    sqerr: list               # per iteration: sqerr of (Vloc, rho)
    energies: list            # per iteration: [E_band, E_H, E_xc, int rho Vxc, charge]
    betas: list               # beta taken by each mixing step
    esp_hist: list            # per iteration: band energies of spin 1, k-point 1


def run_scf(prob: synth.Problem, nelec: float, precision: int = api.PREC_FP64, nsweep: int = 5,
            diter: int = 50, scf_conv=(1e-12, 0.0), mmix: int = 4, beta: float = 1.1, ekbt: float = 1e-5,
            kinteg: int = 5, seed: int = 1, ctx: api.BandUpdate | None = None) -> ScfResult:
    """calc_scf on the GPU for the synthetic operator of prob (its V_loc is V_ion)."""
    own = ctx is None
    g = ctx or api.BandUpdate(prob, precision=precision)
    try:
        nk = prob.nk
        wbz = np.full(nk, 1.0 / nk)
        g.set_vion(prob.vloc)
        vol = prob.ng * prob.dV
        g.set_rho(np.full(prob.ng, nelec / vol))
        g.potential()
        for k in range(nk):
            g.random_wf(seed, k=k + 1)
            g.gram_schmidt(k=k + 1)
        if nsweep > 0:
            g.calc_sweep(nsweep)
        g.init_mixing(mmix, beta)
        sq_hist, e_hist, b_hist, esp_hist = [], [], [], []
        conv = False
        it = 0
        esp = occ = None
        ef = 0.0
        for it in range(1, diter + 1):
            for k in range(nk):
                g.subspace_diag(k=k + 1)
            _, e, _ = g.calc_sweep(1)
            esp = e[:, :, :]
            esp_hist.append(esp[0, 0].copy())
            occ, ef = calc_fermi_mp(esp, wbz, nelec, ekbt, kinteg)
            g.density(occ)
            ene = g.potential()
            e_band = float(np.sum(occ * esp))
            e_hist.append([e_band, *ene.tolist()])
            sq = g.sqerr()
            sq_hist.append(sq.tolist())
            ns = len(sq) // 2
            if (sq[:ns].max() <= scf_conv[0]) or (sq[ns:].max() <= scf_conv[1]):
                conv = True
                break
            b_hist.append(g.mix_density())
            g.normalize_density(nelec)
            g.potential()
        return ScfResult(iterations=it, converged=conv, esp=esp, occ=occ, efermi=ef, sqerr=sq_hist,
                         energies=e_hist, betas=b_hist, esp_hist=esp_hist)
    finally:
        if own:
            g.close()
