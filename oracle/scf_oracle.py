"""CPU FP64 restatement of the SCF outer loop around the oracle's band update.

TEST INFRASTRUCTURE ONLY: used by tests/ as the checker of the library's SCF pieces
(csrc/scf.cu) and of rsdft_develop_b200/scf.py; the product never imports it.

Restated from the reference (numpy, written independently of the library's code):
  calc_density          src/density_module.f90: rho(:,s) = sum_{k,n} occ(n,k,s) |unk|^2
  calc_hartree (FFT)    V_H(G) = 4 pi rho(G) / |G|^2, G != 0; V_H(0) = 0
  calc_LDAPZ81          src/xc/xc_ldapz81_module.f90 (Perdew-Zunger 1981)
  calc_fermi_mp         src/fermi_module.f90:108-262 (Methfessel-Paxton, KINTEG = 5, EKBT)
  init/perform_mixing   src/mixing/mixing_module.f90:70-298, pulay_mixing
                        src/mixing/mixing_pulay_module.f90:29-111 (IMIX = 10)
  calc_scf order        src/scf_module.f90:85-563
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from oracle import oracle as orc


def density(psis, occ):
    """psis[k]: (nb, ng) bands of spin 1 (one spin channel); occ (1, nk, nb)."""
    rho = np.zeros(psis[0].shape[1])
    for k, psi in enumerate(psis):
        w = occ[0, k, :psi.shape[0]]
        rho += np.einsum("n,ni->i", w, (psi.conj() * psi).real)
    return rho


def hartree(rho, n, L):
    """Periodic Poisson solve on the n^3 grid of a cubic cell of side L; returns (V_H, E_H / dV)."""
    r3 = rho.reshape(n, n, n)                     # [z][y][x]
    f = np.fft.rfftn(r3)
    m = np.fft.fftfreq(n, d=1.0 / n)
    mx = np.arange(n // 2 + 1)
    g = 2.0 * math.pi / L
    G2 = (g * m[:, None, None]) ** 2 + (g * m[None, :, None]) ** 2 + (g * mx[None, None, :]) ** 2
    fac = np.zeros_like(G2)
    fac[G2 > 0] = 4.0 * math.pi / G2[G2 > 0]
    vh = np.fft.irfftn(f * fac, s=r3.shape, axes=(0, 1, 2)).reshape(-1)
    return vh, 0.5 * float(np.dot(rho, vh))


def pz81_c(rs, pol):
    """Perdew-Zunger 1981 correlation energy per electron and potential (unpolarised pol = 0,
    polarised pol = 1), both branches of the published fit."""
    gam, b1, b2 = [(-0.1423, 1.0529, 0.3334), (-0.0843, 1.3981, 0.2611)][pol]
    A, B, C, D = [(0.0311, -0.048, 0.002, -0.0116), (0.01555, -0.0269, 0.0007, -0.0048)][pol]
    rs = np.asarray(rs, dtype=np.float64)
    ec = np.empty_like(rs)
    vc = np.empty_like(rs)
    hi = rs >= 1.0
    sq = np.sqrt(rs[hi])
    den = 1.0 + b1 * sq + b2 * rs[hi]
    ec[hi] = gam / den
    vc[hi] = ec[hi] * (1.0 + 7.0 / 6.0 * b1 * sq + 4.0 / 3.0 * b2 * rs[hi]) / den
    lo = ~hi
    lr = np.log(rs[lo])
    ec[lo] = A * lr + B + C * rs[lo] * lr + D * rs[lo]
    vc[lo] = A * lr + (B - A / 3.0) + 2.0 / 3.0 * C * rs[lo] * lr + (2.0 * D - C) / 3.0 * rs[lo]
    return ec, vc


def lda_pz81(rho):
    """Spin-unpolarised LDA: (V_xc, sum rho eps_xc, sum rho V_xc) on the grid."""
    r = np.maximum(rho, 0.0)
    pos = r > 0
    ex = np.zeros_like(r)
    ex[pos] = -0.75 * np.cbrt(3.0 / math.pi * r[pos])
    vx = 4.0 / 3.0 * ex
    ec = np.zeros_like(r)
    vc = np.zeros_like(r)
    rs = np.cbrt(3.0 / (4.0 * math.pi * r[pos]))
    ec[pos], vc[pos] = pz81_c(rs, 0)
    v = vx + vc
    return v, float(np.sum(r * (ex + ec))), float(np.sum(rho * v))


def mp_occ(esp, wbz, nelec, ekbt=1e-5, kinteg=5):
    """Methfessel-Paxton occupations (spin-unpolarised), bisection on the Fermi level."""
    fac = [(-1) ** n / (math.factorial(n) * 4 ** n * math.sqrt(math.pi)) for n in range(1, kinteg + 1)]

    def ff(x):
        f = 0.5 * np.array([math.erfc(v) for v in x.ravel()]).reshape(x.shape)
        h0, h1 = np.ones_like(x), 2.0 * x
        s = fac[0] * h1
        for i in range(2, kinteg + 1):
            h2 = 2.0 * x * h1 - 2.0 * (2 * i - 3) * h0
            h3 = 2.0 * x * h2 - 2.0 * (2 * i - 2) * h1
            s = s + fac[i - 1] * h3
            h0, h1 = h2, h3
        return f + s * np.exp(-x * x)

    w = np.asarray(wbz)[None, :, None] * 2.0
    srt = np.sort(esp.ravel())
    nocc = nelec / 2.0
    i = int(round(nocc))
    ef = 0.5 * (srt[i - 1] + srt[min(i, srt.size - 1)]) if abs(nocc - i) < 1e-12 else srt[int(nocc)]
    lo, hi = ef - 1.0, ef + 1.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        n = float(np.sum(ff((esp - mid) / ekbt) * w))
        if abs(n - nelec) <= 1e-12:
            break
        if n > nelec:
            hi = mid
        else:
            lo = mid
    return ff((esp - mid) / ekbt) * w, mid


@dataclasses.dataclass
class Mixer:
    """init_mixing / perform_mixing (IMIX = 10) state."""
    mmix: int
    beta: float
    xin: list
    xou: list
    xold_f: np.ndarray
    xold_g: np.ndarray
    count: int = 0
    dif0: float = 0.0

    @classmethod
    def init(cls, rho, vloc, mmix=4, beta=1.1):
        z = np.zeros_like(rho)
        xin = [z.copy() for _ in range(mmix)]
        xin[-1] = rho.copy()
        return cls(mmix, beta, xin, [z.copy() for _ in range(mmix)], rho.copy(), vloc.copy())

    def _pulay(self, h, beta):
        mm = self.mmix
        self.xou[-1] = h.copy()
        self.count += 1
        m0 = min(self.count, mm)
        if mm == 1 or m0 < mm:
            for i in range(1, mm):
                self.xin[i - 1] = self.xin[i].copy()
                self.xou[i - 1] = self.xou[i].copy()
            self.xin[-1] = self.xin[-1] + beta * (self.xou[-1] - self.xin[-1])
            return self.xin[-1].copy()
        idx = list(range(mm - m0, mm))
        R = [self.xou[i] - self.xin[i] for i in idx]
        A = np.array([[float(np.dot(a, b)) for b in R] for a in R])
        b = np.linalg.solve(A, np.ones(m0))
        b /= b.sum()
        X = sum(bi * self.xin[i] for bi, i in zip(b, idx))
        Y = sum(bi * self.xou[i] for bi, i in zip(b, idx))
        for i in range(max(1, mm - m0), mm):
            self.xin[i - 1] = self.xin[i].copy()
            self.xou[i - 1] = self.xou[i].copy()
        self.xin[-1] = X + beta * (Y - X)
        return self.xin[-1].copy()

    def mix(self, rho, vloc):
        ml = rho.size
        bak_in = [x.copy() for x in self.xin]
        bak_ou = [x.copy() for x in self.xou]
        cnt = self.count
        beta, beta_min, dif_min = self.beta, self.beta, 1e10
        max_loop = 1
        if beta > 1.0:
            if self.dif0 == 0.0:
                beta = 0.05
            else:
                max_loop, beta = 11, 1.0
        h = rho.copy()
        dif1 = 0.0
        for loop in range(1, max_loop + 1):
            h = self._pulay(rho.copy(), beta)
            dif1 = float(np.sum((h - self.xold_f) ** 2)) / ml
            diff = dif1 / self.dif0 if self.dif0 != 0.0 else 0.0
            if dif1 < dif_min:
                beta_min, dif_min = beta, dif1
            if loop < max_loop:
                if diff > 0.5:
                    self.xin = [x.copy() for x in bak_in]
                    self.xou = [x.copy() for x in bak_ou]
                    self.count = cnt
                    beta *= 0.5
                else:
                    break
                if loop == max_loop - 1:
                    beta = beta_min
        self.dif0 = dif1
        self.xold_f = h.copy()
        self.xold_g = vloc.copy()
        return h, beta


def run_scf(prob, nelec, nsweep=5, diter=50, scf_conv=(1e-12, 0.0), mmix=4, beta=1.1, seed=1, psi0=None):
    """calc_scf with the oracle's band update (one k-point, spin-unpolarised)."""
    from rsdft_develop_b200 import synth  # synthetic input generator (shared test input)
    n = prob.n[0]
    L = n * prob.h
    vion = prob.vloc.copy()
    rho = np.full(prob.ng, nelec / (prob.ng * prob.dV))

    def pot(r):
        vh, eh = hartree(r, n, L)
        vxc, exc, rvxc = lda_pz81(r)
        return vion + vh + vxc, [eh * prob.dV, exc * prob.dV, rvxc * prob.dV, float(r.sum()) * prob.dV]

    vloc, _ = pot(rho)
    psi = psi0 if psi0 is not None else synth.random_wavefunctions(seed, prob.nband, prob.ng)
    o = orc.Oracle(dataclasses.replace(prob, vloc=vloc))
    psi = o.gram_schmidt(psi)
    if nsweep > 0:
        psi, _, _ = o.sweep(psi, nsweep)
    mixer = Mixer.init(rho, vloc, mmix, beta)
    hist = dict(esp=[], sqerr=[], energies=[], betas=[], rho=[])
    for it in range(1, diter + 1):
        o = orc.Oracle(dataclasses.replace(prob, vloc=vloc))
        psi, _ = o.subspace_diag(psi)
        psi, esp, _ = o.sweep(psi, 1)
        esp, _ = o.residual(psi)
        occ, ef = mp_occ(esp[None, None, :], [1.0], nelec)
        rho = density([psi], occ)
        vloc_out, ene = pot(rho)
        sq = [float(np.sum((vloc_out - mixer.xold_g) ** 2)) / rho.size, float(np.sum((rho - mixer.xold_f) ** 2)) / rho.size]
        hist["esp"].append(esp.copy())
        hist["sqerr"].append(sq)
        hist["energies"].append([float(np.sum(occ[0, 0] * esp)), *ene])
        hist["rho"].append(rho.copy())
        if sq[0] <= scf_conv[0] or sq[1] <= scf_conv[1]:
            break
        rho, b = mixer.mix(rho, vloc_out)
        hist["betas"].append(b)
        rho *= nelec / (float(rho.sum()) * prob.dV)
        vloc, _ = pot(rho)
    return hist
