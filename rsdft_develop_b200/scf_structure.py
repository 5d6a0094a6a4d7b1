"""SCF loop for structures read from pseudopotential files (PBE or LDA PZ81, one or two spins,
Gamma or k-points).

The reference's calc_scf (src/scf_module.f90:85-563) around the band update, for the operators
rsdft_develop_b200.structure builds: per iteration (optionally after a Rayleigh-Ritz step on the
new potential, the reference's order) one sweep of every spin on the current V_loc,
occupations, the density of the new bands, V_out = V_ion + V_H + V_xc of that density,
calc_sqerr of (V_out, rho_out) against the previous iteration's pair
(src/sqerr_module.f90:38-103) as the convergence test, then mixing (ReferenceMixer restates the
reference's perform_mixing: simple, Pulay, Broyden or G-space Pulay, of the density or the
potential), renormalisation per spin, and V_loc of the mixed density for the next iteration.  Occupations
are the fixed-moment filling of the reference's first NFIXED iterations (src/fermi_module.f90):
the lowest N_s bands of spin s, N_s = (Nelectron +- Ndspin) / 2 (the reference's O2 sample keeps
that filling to convergence: its occupations print 1 / 0).  Energies follow calc_total_energy
(src/total_energy_module.f90:60-340): Etot = E_kin + E_ion + E_nl + E_H + E_xc + E_ewald, with
E_kin + E_nl = sum occ e - E_loc and E_loc = int rho_out V_loc of the potential the last sweep
used (the reference evaluates it after calc_density, before the potential is updated).

run_scf_kpoints is the same loop for crystals sampled on k-points (the reference's Si sample):
Methfessel-Paxton (calc_fermi_mp, EKBT 1e-5, KINTEG 5 by default) or Fermi-Dirac occupations on
the k weights, the density summed over k (and over ranks when the k-points are split), the
nonlocal energy with the k phases of the projectors.  Both loops report the Harris-Foulkes
energy, and to_vrho / restart_setup write and read the reference's vrho restart file.

The band update runs behind a small interface (set_vloc, sweep, density, bands, and optionally
xc): GpuBands drives the library's CUDA path through the C ABI (band update, density and the
PBE potential on the device); the tests drive the CPU oracle through the same loop.  The
Hartree solve on the cut-off sphere, the mixing and the energies are host work, as in the
reference.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import api, gga, pseudo, scf, structure, vrho


# ----------------------------------------------------------------------------
# ion-ion energy
# ----------------------------------------------------------------------------
def ewald_energy(st: structure.Structure, eta: float | None = None, tol: float = 1e-14) -> float:
    """Ewald energy of the ions (point charges Zps at the atoms, neutralising background) in the
    cell, the quantity calc_ewald returns (src/ewald_module.f90:69-420):
    1/2 sum'_{i,j,L} Z_i Z_j erfc(sqrt(eta) r) / r + (2 pi / V) sum_{G != 0} |S(G)|^2
    exp(-G^2 / 4 eta) / G^2 - sqrt(eta / pi) sum Z_i^2 - pi Q^2 / (2 eta V)."""
    if not st.orthorhombic:
        return _ewald_lattice(st, eta, tol)
    L = np.array(st.lengths, dtype=np.float64)
    vol = float(np.prod(L))
    pos, z = [], []
    for pp, p in st.species:
        for a in np.asarray(p, np.float64).reshape(-1, 3):
            pos.append(a * L)
            z.append(pp.zps)
    pos = np.array(pos)
    z = np.array(z)
    if eta is None:
        eta = math.pi / vol ** (2.0 / 3.0)
    se = math.sqrt(eta)
    # real space: images until erfc(sqrt(eta) r) < tol
    rcut = 1.0
    while math.erfc(se * rcut) > tol:
        rcut += 0.5
    nimg = [int(math.ceil(rcut / L[d])) + 1 for d in range(3)]
    er = 0.0
    rng = [np.arange(-n, n + 1) for n in nimg]
    sh = np.stack(np.meshgrid(*rng, indexing="ij"), axis=-1).reshape(-1, 3) * L
    for i in range(len(z)):
        for j in range(len(z)):
            d = pos[i] - pos[j] + sh
            r = np.sqrt(np.sum(d * d, axis=1))
            keep = (r > 1e-12) & (r < rcut)
            er += 0.5 * z[i] * z[j] * sum(math.erfc(se * x) / x for x in r[keep])
    # reciprocal space: until exp(-G^2 / 4 eta) < tol
    gmax = 2.0 * se * math.sqrt(-math.log(tol))
    b = 2.0 * math.pi / L
    ng = [int(math.ceil(gmax / b[d])) + 1 for d in range(3)]
    m = np.stack(np.meshgrid(*[np.arange(-n, n + 1) for n in ng], indexing="ij"), axis=-1).reshape(-1, 3)
    g = m * b
    g2 = np.sum(g * g, axis=1)
    keep = (g2 > 0) & (g2 <= gmax * gmax)
    g, g2 = g[keep], g2[keep]
    ph = g @ pos.T
    s = (np.cos(ph) * z).sum(axis=1) + 1j * (np.sin(ph) * z).sum(axis=1)
    eg = 2.0 * math.pi / vol * float(np.sum(np.abs(s) ** 2 * np.exp(-g2 / (4.0 * eta)) / g2))
    q = float(z.sum())
    return er + eg - se / math.sqrt(math.pi) * float(np.sum(z * z)) - math.pi * q * q / (2.0 * eta * vol)


def _ewald_lattice(st: structure.Structure, eta: float | None, tol: float) -> float:
    """ewald_energy for lattice vectors (rows of st.avec): lattice translations and reciprocal
    vectors as integer combinations, each range wide enough for the real- and reciprocal-space
    cut-offs along the normal of every pair of cell faces."""
    A = st.avec
    vol = st.volume
    B = 2.0 * math.pi / float(np.dot(A[0], np.cross(A[1], A[2]))) * np.array(
        [np.cross(A[1], A[2]), np.cross(A[2], A[0]), np.cross(A[0], A[1])])
    pos, z = [], []
    for pp, p in st.species:
        for a in np.asarray(p, np.float64).reshape(-1, 3):
            pos.append(a @ A)
            z.append(pp.zps)
    pos = np.array(pos)
    z = np.array(z)
    if eta is None:
        eta = math.pi / vol ** (2.0 / 3.0)
    se = math.sqrt(eta)
    rcut = 1.0
    while math.erfc(se * rcut) > tol:
        rcut += 0.5
    # |n_d| <= rcut |b_d| / (2 pi) + 1 covers every translation shorter than rcut (+ the atoms' spread)
    nimg = [int(math.ceil(rcut * float(np.linalg.norm(B[d])) / (2.0 * math.pi))) + 2 for d in range(3)]
    m = np.stack(np.meshgrid(*[np.arange(-x, x + 1) for x in nimg], indexing="ij"), axis=-1).reshape(-1, 3)
    sh = m @ A
    er = 0.0
    for i in range(len(z)):
        for j in range(len(z)):
            d = pos[i] - pos[j] + sh
            r = np.sqrt(np.sum(d * d, axis=1))
            keep = (r > 1e-12) & (r < rcut)
            er += 0.5 * z[i] * z[j] * sum(math.erfc(se * x) / x for x in r[keep])
    gmax = 2.0 * se * math.sqrt(-math.log(tol))
    ng = [int(math.ceil(gmax * float(np.linalg.norm(A[d])) / (2.0 * math.pi))) + 1 for d in range(3)]
    m = np.stack(np.meshgrid(*[np.arange(-x, x + 1) for x in ng], indexing="ij"), axis=-1).reshape(-1, 3)
    g = m @ B
    g2 = np.sum(g * g, axis=1)
    keep = (g2 > 0) & (g2 <= gmax * gmax)
    g, g2 = g[keep], g2[keep]
    ph = g @ pos.T
    sg = (np.cos(ph) * z).sum(axis=1) + 1j * (np.sin(ph) * z).sum(axis=1)
    eg = 2.0 * math.pi / vol * float(np.sum(np.abs(sg) ** 2 * np.exp(-g2 / (4.0 * eta)) / g2))
    q = float(z.sum())
    return er + eg - se / math.sqrt(math.pi) * float(np.sum(z * z)) - math.pi * q * q / (2.0 * eta * vol)


# ----------------------------------------------------------------------------
# host pieces
# ----------------------------------------------------------------------------
def potential(su: structure.Setup, rho: np.ndarray, xc=None):
    """V_loc(s) = V_ion + V_H + V_xc^PBE(s) of rho (nspin, ng), and the energy pieces.  xc: a
    callable rho -> (V_xc, E_x, E_c) (the device PBE of GpuBands); the host PBE otherwise."""
    st = su.structure
    dV = su.problem.dV
    h = (su.problem.h,) * 3
    vh, eh = gga.hartree_sphere(rho.sum(axis=0), su.ggrid, dV)
    if xc is not None:
        vxc, ex, ec = xc(rho)
    else:
        vxc, ex, ec = structure.host_xc(st.xc, rho, su.problem.n, h, dV, st.md, su.bmat)
    v = su.vion[None, :] + vh[None, :] + vxc
    return v, {"hartree": eh, "xc": ex + ec, "exchange": ex, "correlation": ec,
               "ion_local": float(np.sum(rho.sum(axis=0) * su.vion)) * dV,
               "local": float(np.sum(rho * v)) * dV}


class Pulay:
    """Pulay (DIIS) mixing of the density vector (both spins together), history mmix, step beta:
    rho_in' = sum_i c_i (rho_in,i + beta (rho_out,i - rho_in,i)) with sum c_i = 1 minimising
    |sum_i c_i (rho_out,i - rho_in,i)|."""

    def __init__(self, mmix: int = 4, beta: float = 0.5):
        self.mmix, self.beta = mmix, beta
        self.xin, self.res = [], []

    def mix(self, rin: np.ndarray, rout: np.ndarray) -> np.ndarray:
        self.xin.append(rin.ravel().copy())
        self.res.append((rout - rin).ravel().copy())
        self.xin, self.res = self.xin[-self.mmix:], self.res[-self.mmix:]
        n = len(self.res)
        A = np.array([[float(np.dot(a, b)) for b in self.res] for a in self.res])
        A += 1e-14 * np.trace(A) * np.eye(n)
        c = np.linalg.solve(A, np.ones(n))
        c /= c.sum()
        x = sum(ci * xi for ci, xi in zip(c, self.xin))
        r = sum(ci * ri for ci, ri in zip(c, self.res))
        return (x + self.beta * r).reshape(rin.shape)


def _kerker_weights(n: tuple, bb: np.ndarray):
    """(wq, wq2) on the FFT box, shape (n3, n2, n1): the reference's G index of box point i is
    i - N, or i where that falls below -(N - 1) / 2 (get_Kerker_weights)."""
    idx = []
    for N in n:
        i = np.arange(N)
        j = i - N
        idx.append(np.where(j < -((N - 1) // 2), i, j))
    j1, j2, j3 = idx
    J3, J2, J1 = np.meshgrid(j3, j2, j1, indexing="ij")
    g = [J1 * bb[c, 0] + J2 * bb[c, 1] + J3 * bb[c, 2] for c in range(3)]
    gg = g[0] ** 2 + g[1] ** 2 + g[2] ** 2
    nz = gg[gg > 0.0]
    gmin, gmax = float(nz.min()), float(nz.max())
    b1 = 19.0 * gmin * gmax / (gmax - 20.0 * gmin)
    b2 = ((1.5 * 0.529177) ** 2) ** 2
    with np.errstate(divide="ignore", invalid="ignore"):
        wq = np.where(gg == 0.0, 1.0, (gg + b1) / np.where(gg == 0.0, 1.0, gg))
        wq2 = np.where(gg == 0.0, 1.0, gg / (gg + b2))
    return wq, wq2


class ReferenceMixer:
    """perform_mixing (src/mixing/mixing_module.f90:145-290) for the density-mixing choices of
    IMIX: 0-9 simple mixing (simple_mixing :381-387), 10-19 Pulay (pulay_mixing,
    src/mixing/mixing_pulay_module.f90:29-111; the reference's default IMIX = 10 with MMIX = 4,
    BETA = 1.1), 20-29 Broyden (broyden_mixing, src/mixing/mixing_broyden_module.f90:11-188).

    Pulay: the history holds (input, output) density pairs; while fewer than mmix pairs exist a
    step is linear, x_in + beta (x_out - x_in); then x = sum_i c_i x_in,i + beta sum_i c_i
    (x_out,i - x_in,i) with sum_i c_i = 1 minimising |sum_i c_i (x_out,i - x_in,i)|.  Broyden:
    Johnson's modified Broyden step over the same history, residual weights 1/|F_k| (at most 1)
    and w_0 = beta.  Simple: (1 - beta) x_old + beta x_out.  BETA > 1 asks for a search: the
    first call takes beta = 0.05; later calls try beta = 1, 1/2, 1/4, ... (at most 11 tries, the
    last with the beta of the smallest change) while the squared change of the mixed density
    from the previous mixed one exceeds half of the previous change.  Even IMIX mixes the density
    (the result is made non-negative, chk_chrg), odd IMIX the potential V_loc (the SCF loop then
    takes the mixed potential as the next input).  IMIX 30-39 runs the Pulay step on the Fourier
    coefficients (pulay_g_mixing :124-205, get_Kerker_weights :275-337): residual products
    weighted by (|G|^2 + q1) / |G|^2 and updates damped by |G|^2 / (|G|^2 + q2), with q1 = 19
    |G|min^2 |G|max^2 / (|G|max^2 - 20 |G|min^2) over the FFT box and q2 = (1.5 x 0.529177)^4
    (BMIX squared twice, as the reference does); it needs grid = (n, bb) with bb the reciprocal
    vectors as columns."""

    def __init__(self, rho0: np.ndarray, mmix: int = 4, beta: float = 1.1, imix: int = 10, grid=None):
        if not 0 <= imix <= 39:
            raise NotImplementedError(f"IMIX {imix}: simple 0-9, Pulay 10-19, Broyden 20-29 or G-space Pulay 30-39")
        self.scheme = ("simple", "pulay", "broyden", "pulay_g")[imix // 10]
        self.potential = imix % 2 == 1
        self.mmix, self.beta = max(1, int(mmix)), float(beta)
        shape = rho0.shape
        if self.scheme == "pulay_g":
            if grid is None:
                raise ValueError("IMIX 30-39 needs grid = (n, bb)")
            self.n = tuple(grid[0])
            self.wq, self.wq2 = _kerker_weights(self.n, np.asarray(grid[1], np.float64))
            rho0 = self._fft(rho0)
            shape = rho0.shape
        self.xin = np.zeros((self.mmix,) + shape, rho0.dtype)
        self.xou = np.zeros((self.mmix,) + shape, rho0.dtype)
        self.xin[-1] = rho0
        self.count = 0
        self.xold = (self._ifft(rho0) if self.scheme == "pulay_g" else rho0).copy()
        self.dif0 = np.zeros(shape[0])
        self.betas = []

    def _fft(self, x: np.ndarray) -> np.ndarray:
        n1, n2, n3 = self.n
        return np.fft.fftn(x.reshape(-1, n3, n2, n1), axes=(1, 2, 3))

    def _ifft(self, z: np.ndarray) -> np.ndarray:
        return np.fft.ifftn(z, axes=(1, 2, 3)).real.reshape(z.shape[0], -1)

    def _pulay_g(self, f: np.ndarray, beta: float) -> np.ndarray:
        m = self.mmix
        self.xou[-1] = self._fft(f)
        self.count += 1
        m0 = min(self.count, m)
        if m == 1 or m0 < m:
            self.xin[:-1] = self.xin[1:].copy()
            self.xou[:-1] = self.xou[1:].copy()
            self.xin[-1] = self.xin[-1] + beta * self.wq2 * (self.xou[-1] - self.xin[-1])
            return self._ifft(self.xin[-1])
        r = (self.xou[m - m0:] - self.xin[m - m0:]).reshape(m0, -1)
        w = np.broadcast_to(self.wq, self.xin.shape[1:]).reshape(-1)
        a = (np.conj(r) * w) @ r.T
        try:
            c = np.linalg.solve(a, np.ones(m0, complex))
        except np.linalg.LinAlgError:
            c = np.linalg.lstsq(a, np.ones(m0, complex), rcond=None)[0]
        if not np.isfinite(c.sum()) or c.sum() == 0.0:
            c = np.zeros(m0, complex)
            c[-1] = 1.0
        c /= c.sum()
        x = np.tensordot(c, self.xin[m - m0:], axes=1)
        y = np.tensordot(c, self.xou[m - m0:], axes=1)
        self.xin[:-1] = self.xin[1:].copy()
        self.xou[:-1] = self.xou[1:].copy()
        self.xin[-1] = x + beta * self.wq2 * (y - x)
        return self._ifft(self.xin[-1])

    def _pulay(self, f: np.ndarray, beta: float) -> np.ndarray:
        m = self.mmix
        self.xou[-1] = f
        self.count += 1
        m0 = min(self.count, m)
        if m == 1 or m0 < m:
            self.xin[:-1] = self.xin[1:].copy()
            self.xou[:-1] = self.xou[1:].copy()
            self.xin[-1] = self.xin[-1] + beta * (self.xou[-1] - self.xin[-1])
            return self.xin[-1].copy()
        r = (self.xou[m - m0:] - self.xin[m - m0:]).reshape(m0, -1)
        a = r @ r.T
        try:
            c = np.linalg.solve(a, np.ones(m0))
        except np.linalg.LinAlgError:            # residuals linearly dependent (e.g. converged)
            c = np.linalg.lstsq(a, np.ones(m0), rcond=None)[0]
        if not np.isfinite(c.sum()) or c.sum() == 0.0:
            c = np.zeros(m0)
            c[-1] = 1.0
        c /= c.sum()
        x = np.tensordot(c, self.xin[m - m0:], axes=1)
        y = np.tensordot(c, self.xou[m - m0:], axes=1)
        self.xin[:-1] = self.xin[1:].copy()
        self.xou[:-1] = self.xou[1:].copy()
        self.xin[-1] = x + beta * (y - x)
        return self.xin[-1].copy()

    def _broyden(self, f: np.ndarray, alpha: float) -> np.ndarray:
        m = self.mmix
        self.xou[-1] = f
        self.count += 1
        m0 = min(self.count, m)
        if m == 1 or m0 == 1:
            self.xin[:-1] = self.xin[-1]
            self.xou[:-1] = self.xou[-1]
            self.xin[-1] = (1.0 - alpha) * self.xin[-1] + alpha * self.xou[-1]
            return self.xin[-1].copy()
        if m0 < m:                                # the history moves to the first m0 slots
            self.xin[:m0 - 1] = self.xin[1:m0].copy()
            self.xou[:m0 - 1] = self.xou[1:m0].copy()
            self.xin[m0 - 1] = self.xin[-1]
            self.xou[m0 - 1] = self.xou[-1]
        xin, xou = self.xin[:m0].reshape(m0, -1), self.xou[:m0].reshape(m0, -1)
        F = xou - xin
        w = np.ones(m0)
        nf = np.sum(F * F, axis=1)
        pos = nf > 0.0
        w[pos] = np.minimum(1.0, 1.0 / np.sqrt(nf[pos]))
        dF = F[1:] - F[:-1]
        nrm = 1.0 / np.sqrt(np.sum(dF * dF, axis=1))
        dF *= nrm[:, None]
        dX = (xin[1:] - xin[:-1]) * nrm[:, None]
        u = alpha * dF + dX
        wk = w[:-1]
        cm = wk * (dF @ F[-1])
        a = np.outer(wk, wk) * (dF @ dF.T) + alpha * alpha * np.eye(m0 - 1)
        gamma = cm @ np.linalg.inv(a)
        xnew = xin[-1] + alpha * F[-1] - (wk * gamma) @ u
        if m0 == m:
            self.xin[:-1] = self.xin[1:].copy()
            self.xou[:-1] = self.xou[1:].copy()
        self.xin[-1] = xnew.reshape(f.shape)
        return self.xin[-1].copy()

    def _step(self, f: np.ndarray, beta: float) -> np.ndarray:
        if self.scheme == "pulay":
            return self._pulay(f, beta)
        if self.scheme == "pulay_g":
            return self._pulay_g(f, beta)
        if self.scheme == "broyden":
            return self._broyden(f, beta)
        return (1.0 - beta) * self.xold + beta * f

    def mix(self, rho_out: np.ndarray) -> np.ndarray:
        ng = rho_out.shape[1]
        bak = (self.xin.copy(), self.xou.copy(), self.count)
        beta = beta_min = self.beta
        dif_min = np.full(rho_out.shape[0], 1e10)
        max_loop = 1
        if beta > 1.0:
            if np.all(self.dif0 == 0.0):
                beta = 0.05
            else:
                max_loop, beta = 11, 1.0
        h = dif1 = None
        for loop in range(1, max_loop + 1):
            h = self._step(rho_out.copy(), beta)
            dif1 = np.sum((h - self.xold) ** 2, axis=1) / ng
            safe = np.where(self.dif0 != 0.0, self.dif0, 1.0)
            diff = np.where(self.dif0 != 0.0, dif1 / safe, 0.0)
            if np.all(dif1 < dif_min):
                beta_min, dif_min = beta, dif1
            if loop < max_loop:
                if np.any(diff > 0.5):
                    self.xin, self.xou, self.count = bak[0].copy(), bak[1].copy(), bak[2]
                    beta *= 0.5
                else:
                    break
                if loop == max_loop - 1:
                    beta = beta_min
        self.betas.append(beta)
        self.dif0 = dif1
        if not self.potential:
            h = np.abs(h)
        self.xold = h.copy()
        return h


def nonlocal_energy(su: structure.Setup, psi: np.ndarray, occ: np.ndarray) -> float:
    """sum_n occ_n sum_lma iuV(lma) (dV sum_j uV(j, lma) psi_n(JJP(j, lma)))^2 for one spin."""
    ps = su.projectors
    dV = su.problem.dV
    e = 0.0
    for p in range(ps.nzlma):
        m = int(ps.mjj[p])
        idx = ps.jjp[p, :m] - 1
        c = dV * (psi[:, idx] @ ps.uv[p, :m])
        e += float(ps.iuv[p]) * float(np.sum(occ * c * c))
    return e


# ----------------------------------------------------------------------------
# the band update behind the loop
# ----------------------------------------------------------------------------
class GpuBands:
    """The library's CUDA band update (all spins in one context) for the SCF loop."""

    def __init__(self, su: structure.Setup, precision: int = api.PREC_FP64, seed: int = 1):
        self.su = su
        self.ns = su.structure.nspin
        self.g = api.BandUpdate(su.problem_for_spin(1), precision=precision, nspin=self.ns)
        for s in range(2, self.ns + 1):
            self.g.set_vloc(su.vloc[s - 1], s=s)
        for s in range(1, self.ns + 1):
            self.g.random_wf(seed + s - 1, s=s)
            self.g.gram_schmidt(s=s)

    def set_vloc(self, v: np.ndarray):
        for s in range(self.ns):
            self.g.set_vloc(v[s], s=s + 1)

    def sweep(self, n: int, diag_first: bool = False) -> np.ndarray:
        if diag_first:
            for s in range(1, self.ns + 1):
                self.g.subspace_diag(s=s)
        _, esp, _ = self.g.calc_sweep(n)
        return esp[:, 0, :].copy()

    def density(self, occ: np.ndarray) -> np.ndarray:
        self.g.density(occ[:, None, :])
        return self.g.get_rho()[0]

    def xc(self, rho: np.ndarray):
        """PBE V_xc and (E_x, E_c) of rho on the device (rsdft_gpu_xc_pbe)."""
        return self.g.xc_pbe(rho)

    def bands(self, s: int) -> np.ndarray:
        return self.g.get_wf(s=s + 1)

    def close(self):
        self.g.close()


@dataclasses.dataclass
class StructureScf:
    iterations: int
    converged: bool
    esp: np.ndarray               # (nspin, nband) of the last sweep
    occ: np.ndarray
    rho: np.ndarray               # output density of the last iteration
    sqerr: list                   # per iteration: sqerr of V_out (per spin) + of rho_out (per spin)
    energies: dict
    vloc: np.ndarray | None = None  # (nspin, ng) the potential of the last sweep


def to_vrho(su: structure.Setup, res: StructureScf) -> vrho.Vrho:
    """What write_data (OC = 2, 3, ...) saves at the end of an SCF: the output density, the
    potential of the last sweep, and V_H, V_xc of the output density (src/scf_module.f90 leaves
    Vloc un-updated on exit and recomputes V_H, V_xc at the top of each iteration)."""
    st = su.structure
    vh, _ = gga.hartree_sphere(res.rho.sum(axis=0), su.ggrid, su.problem.dV)
    vxc, _, _ = structure.host_xc(st.xc, res.rho, su.problem.n, (su.problem.h,) * 3, su.problem.dV, st.md, su.bmat)
    atoms = np.concatenate([np.asarray(p, np.float64).reshape(-1, 3) for _, p in st.species])
    ki = np.concatenate([np.full(len(np.asarray(p).reshape(-1, 3)), e + 1, np.int32)
                         for e, (_, p) in enumerate(st.species)])
    zn = np.array([int(round(pp.zelement)) for pp, _ in st.species], np.int32)
    return vrho.Vrho(n=tuple(su.problem.n), rho=res.rho.copy(), vloc=np.asarray(res.vloc).copy(), vh=vh,
                     vxc=vxc, efermi=float(res.energies.get("fermi", 0.0)), aa=st.avec, atoms=atoms,
                     ki_atom=ki, zn_atom=zn)


def restart_setup(su: structure.Setup, v: vrho.Vrho) -> structure.Setup:
    """su with the density and potential of a vrho file (read_data with IC = 2, 3, ...): the SCF
    starts from them instead of the initial density."""
    if tuple(v.n) != tuple(su.problem.n) or v.rho.shape != su.rho.shape:
        raise ValueError("vrho: grid or spin count differs from the structure's")
    return dataclasses.replace(su, rho=v.rho.copy(), vloc=v.vloc.copy(),
                               problem=dataclasses.replace(su.problem, vloc=np.ascontiguousarray(v.vloc[0])))


def _harris(e_sum: float, ene_in: dict, st: structure.Structure) -> float:
    """Harris-Foulkes energy of the last iteration (calc_with_rhoIN_total_energy,
    src/total_energy_module.f90:345-346): sum occ e - int rho_in V_in + E_H[rho_in] +
    E_xc[rho_in] + int rho_in V_ion + E_ewald, with rho_in the density V_in was built from."""
    return (e_sum - ene_in["local"] + ene_in["hartree"] + ene_in["xc"] + ene_in["ion_local"]
            + ewald_energy(st))


def run_scf_structure(su: structure.Setup, bands, nsweep: int = 10, diter: int = 100, scf_conv: float = 1e-11,
                      mmix: int = 1, beta: float = 0.5, mixing: str = "pulay", diag_first: bool = False,
                      imix: int = 10) -> StructureScf:
    """calc_scf for su with the band update `bands` (GpuBands or a test adapter): nsweep sweeps on
    the potential of the initial density, then up to diter iterations until the squared change
    of V_out (mean over the grid, every spin) is <= scf_conv.  Mixing "pulay": the Pulay class,
    linear with step beta for mmix = 1 (the default); "reference": ReferenceMixer with IMIX =
    imix, MMIX = mmix, BETA = beta (the reference's defaults are 10, 4 and 1.1).  diag_first: a Rayleigh-Ritz step
    of every spin on the new potential before each iteration's sweep, the reference's order
    (bands.sweep(n, True)).  On the reference's O2 sample the reference order and mixing reach
    scf_conv = 1e-15 (24 iterations with the oracle band update); linear mixing without the
    leading Rayleigh-Ritz step levels off near 1e-12, where PBE's potential near the vacuum
    follows the density tails around the 1e-10 cut, with energies converged to ~1e-8."""
    st = su.structure
    ns, nb = st.nspin, st.nband
    dV = su.problem.dV
    nel = np.asarray(su.nelectron_spin)
    if np.any(np.abs(nel - np.round(nel)) > 1e-12):
        raise NotImplementedError("fixed-moment filling needs integer electrons per spin")
    nocc = [int(round(x)) for x in (nel if ns == 2 else nel / 2.0)]
    occ = np.zeros((ns, nb))
    for s in range(ns):
        occ[s, :nocc[s]] = 1.0 if ns == 2 else 2.0
    xc = getattr(bands, "xc", None) if structure.is_pbe(st.xc) else None   # the device kernel is PBE
    bands.set_vloc(su.vloc)
    v_cur = su.vloc
    if nsweep > 0:
        bands.sweep(nsweep)
    rho_in = su.rho.copy()
    prev = (su.vloc.copy(), su.rho.copy())
    if mixing == "pulay":
        mixer = Pulay(mmix, beta)
    elif mixing == "reference":
        mixer = ReferenceMixer(su.vloc if imix % 2 else su.rho, mmix, beta, imix,
                               grid=(su.problem.n, pseudo.reciprocal(su.structure.avec).T))
    else:
        raise ValueError(f"mixing {mixing!r}: 'pulay' or 'reference'")
    vmix = mixing == "reference" and imix % 2 == 1
    ene_in = None if vmix else potential(su, su.rho, xc)[1]
    hist = []
    conv = False
    esp = rho_out = ene = None
    it = 0
    for it in range(1, diter + 1):
        esp = bands.sweep(1, True) if diag_first else bands.sweep(1)
        rho_out = bands.density(occ)
        v_out, ene = potential(su, rho_out, xc)
        sq = [float(np.mean((v_out[s] - prev[0][s]) ** 2)) for s in range(ns)] + \
             [float(np.mean((rho_out[s] - prev[1][s]) ** 2)) for s in range(ns)]
        hist.append(sq)
        prev = (v_out, rho_out)
        if max(sq[:ns]) <= scf_conv:
            conv = True
            break
        if vmix:
            v_in = mixer.mix(v_out)
        else:
            rho_in = mixer.mix(rho_in, rho_out) if mixing == "pulay" else mixer.mix(rho_out)
            for s in range(ns):
                rho_in[s] *= (occ[s].sum()) / (float(rho_in[s].sum()) * dV)
            v_in, ene_in = potential(su, rho_in, xc)
        bands.set_vloc(v_in)
        v_cur = v_in
    e_sum = float(np.sum(occ * esp))
    e_nl = sum(nonlocal_energy(su, bands.bands(s), occ[s]) for s in range(ns))
    ene = dict(ene)
    ene["local"] = float(np.sum(rho_out * v_cur)) * dV
    if ene_in is not None:
        ene["harris"] = _harris(e_sum, ene_in, st)
    ene["sum_eigen"] = e_sum
    ene["nonlocal"] = e_nl
    ene["kinetic"] = e_sum - ene["local"] - e_nl
    ene["ewald"] = ewald_energy(st)
    ene["total"] = (ene["kinetic"] + ene["ion_local"] + e_nl + ene["hartree"] + ene["xc"] + ene["ewald"])
    ene["spin_abs"] = float(np.sum(np.abs(rho_out[0] - rho_out[-1]))) * dV if ns == 2 else 0.0
    return StructureScf(iterations=it, converged=conv, esp=esp, occ=occ, rho=rho_out, sqerr=hist, energies=ene,
                        vloc=np.array(v_cur))


# ----------------------------------------------------------------------------
# crystals on k-points
# ----------------------------------------------------------------------------
def nonlocal_energy_k(su: structure.Setup, psi: np.ndarray, occ: np.ndarray, k: int) -> float:
    """sum_n occ_n sum_lma iuV(lma) |dV sum_j conj(uVk(j, lma, k)) psi_n(JJP(j, lma))|^2 for the
    bands psi (nb, ng) of k-point k (0-based) of one spin."""
    prob = su.problem
    dV = prob.dV
    e = 0.0
    for p in range(prob.nzlma):
        m = int(prob.mjj[p])
        idx = prob.jjp[p, :m] - 1
        c = dV * (psi[:, idx] @ np.conj(prob.uvk[k, p, :m]))
        e += float(prob.dij[p]) * float(np.sum(occ * np.abs(c) ** 2))
    return e


def run_scf_kpoints(su: structure.Setup, bands, nsweep: int = 10, diter: int = 100, scf_conv: float = 1e-15,
                    mixing: str = "reference", mmix: int = 4, beta: float = 1.1, ekbt: float = 1e-5,
                    kinteg: int = 5, diag_first: bool = True, kgroup=None, imix: int = 10,
                    occupations: str = "mp", nfixed: int = 0) -> StructureScf:
    """calc_scf for a structure set up on k-points (su.structure.kbb / wbz) with the band update
    `bands`: set_vloc(v (nspin, ng)), sweep(n, diag_first) -> esp (nspin, nk, nband),
    density(occ (nspin, nk, nband), weights included) -> rho (nspin, ng), bands(s, k) ->
    (nband, ng).  nsweep sweeps on the potential of the initial density, then per iteration, in
    the reference's order (src/scf_module.f90:200-460): a Rayleigh-Ritz step of every (k, s) on
    the new potential (subspace_diag, unless diag_first is False) and one sweep,
    Methfessel-Paxton occupations, the output density and potential, calc_sqerr's test of V_out
    against the previous iteration (mean over the grid <= scf_conv), mixing of the density and
    renormalisation per spin.  mixing "reference": ReferenceMixer (IMIX = imix, MMIX = mmix,
    BETA = beta, the reference's defaults 10, 4 and 1.1); "linear": x_in + beta (x_out - x_in).

    occupations "mp": Methfessel-Paxton of order kinteg (calc_fermi_mp, the reference's
    default; with two spins the first nfixed iterations keep the moment Ndspin of the
    structure, each spin filled to its own level); "fd": Fermi-Dirac (fermi_dirac, MP_VERSION -1) with its entropy term, the free
    energy E - TS in energies["free"].

    kgroup: a kparallel.KpointGroup when the k-points are split over ranks; `bands` then holds
    the k-points kgroup.klist only (its sweep returns those, its density sums over those, its
    bands(s, j) takes the local index j), the eigenvalues are gathered for the occupations and
    the density and band-energy sums are added over the ranks; every rank returns the same
    result."""
    from .kparallel import KpointGroup
    if occupations not in ("mp", "fd"):
        raise ValueError(f"occupations {occupations!r}: 'mp' or 'fd'")
    st = su.structure
    kg = kgroup if kgroup is not None else KpointGroup(su.problem.nk, local=True)
    kl = kg.klist
    ns = st.nspin
    dV = su.problem.dV
    wbz = np.asarray(st.wbz, np.float64)
    nel = st.nelectron
    bands.set_vloc(su.vloc)
    v_cur = su.vloc
    if nsweep > 0:
        bands.sweep(nsweep, False)
    rho_in = su.rho.copy()
    prev = (su.vloc.copy(), su.rho.copy())
    if mixing == "reference":
        mixer = ReferenceMixer(su.vloc if imix % 2 else su.rho, mmix, beta, imix,
                               grid=(su.problem.n, pseudo.reciprocal(su.structure.avec).T))
    elif mixing == "linear":
        mixer = None
    else:
        raise ValueError(f"mixing {mixing!r}: 'reference' or 'linear'")
    vmix = mixing == "reference" and imix % 2 == 1
    ene_in = None if vmix else potential(su, su.rho)[1]
    hist = []
    conv = False
    esp = occ = rho_out = ene = None
    ef = 0.0
    it = 0
    for it in range(1, diter + 1):
        esp = kg.gather_esp(bands.sweep(1, diag_first))
        if occupations == "fd":
            occ, ef = scf.fermi_dirac(esp, wbz, nel, ekbt)
        elif ns == 2 and it <= nfixed:
            occ, efs = scf.calc_fermi_mp_fixed(esp, wbz, nel, st.ndspin, ekbt, kinteg)
            ef = max(efs)
        else:
            occ, ef = scf.calc_fermi_mp(esp, wbz, nel, ekbt, kinteg)
        rho_out = kg.sum(bands.density(occ[:, kl[0]:kl[-1] + 1]))
        v_out, ene = potential(su, rho_out)
        sq = [float(np.mean((v_out[s] - prev[0][s]) ** 2)) for s in range(ns)] + \
             [float(np.mean((rho_out[s] - prev[1][s]) ** 2)) for s in range(ns)]
        hist.append(sq)
        prev = (v_out, rho_out)
        if max(sq[:ns]) <= scf_conv:
            conv = True
            break
        if vmix:
            v_in = mixer.mix(v_out)
        else:
            rho_in = mixer.mix(rho_out) if mixer is not None else rho_in + beta * (rho_out - rho_in)
            for s in range(ns):
                rho_in[s] *= float(occ[s].sum()) / (float(rho_in[s].sum()) * dV)
            v_in, ene_in = potential(su, rho_in)
        bands.set_vloc(v_in)
        v_cur = v_in
    e_sum = float(np.sum(occ * esp))
    e_nl = kg.sum(sum(nonlocal_energy_k(su, bands.bands(s, j), occ[s, k], k)
                      for s in range(ns) for j, k in enumerate(kl)))
    ene = dict(ene)
    ene["local"] = float(np.sum(rho_out * v_cur)) * dV
    ene["sum_eigen"] = e_sum
    ene["nonlocal"] = e_nl
    ene["kinetic"] = e_sum - ene["local"] - e_nl
    ene["ewald"] = ewald_energy(st)
    ene["total"] = (ene["kinetic"] + ene["ion_local"] + e_nl + ene["hartree"] + ene["xc"] + ene["ewald"])
    ene["fermi"] = float(ef)
    if ene_in is not None:
        ene["harris"] = _harris(e_sum, ene_in, st)
    if occupations == "fd":
        ene["entropy"] = scf.entropy_fd(ekbt, occ)
        ene["free"] = ene["total"] - ene["entropy"]
    return StructureScf(iterations=it, converged=conv, esp=esp, occ=occ, rho=rho_out, sqerr=hist, energies=ene,
                        vloc=np.array(v_cur))
