"""GGA-PBE exchange-correlation and the cut-off-sphere Hartree potential on the real-space grid.

Host-side potential pieces for structures read from pseudopotential files (the reference's
samples use PBE with spin polarisation).  Restated from the reference:

  calc_GGAPBE96_2        src/xc/xc_ggapbe96_2_module.f90:26-370 (PBE exchange and correlation
                         with mu = 0.21951, kappa = 0.804, beta = 3 mu / pi^2; densities below
                         1e-10 skipped; the gradient is that of the total density in both the
                         exchange and correlation terms, as the reference computes it)
  construct_gradient16   src/kinetic/gradient_module.f90:92-175 (central FD gradient of order Md)
  calc_abc_gradient_org  src/kinetic/gradient_module.f90:349-438 (the divergence term)
  calc_hartree_sol_fftw  src/hartree/hartree_sol_fftw_module.f90:24-110 (4 pi rho(G) / G^2 over
                         the cut-off sphere, G = 0 left out)
"""
from __future__ import annotations

import math

import numpy as np
import scipy.fft

from .synth import fd_nab_coef


def _fd_derivative(f3: np.ndarray, axis: int, nab: np.ndarray, md: int) -> np.ndarray:
    """sum_m nab(m) (f(i + m) - f(i - m)) along one axis of a periodic (z, y, x) array."""
    g = np.zeros_like(f3)
    for m in range(1, md + 1):
        g += nab[md + m] * (np.roll(f3, -m, axis=axis) - np.roll(f3, m, axis=axis))
    return g


def grid_metric(cell, n: tuple) -> np.ndarray:
    """b(:, j) = |a_j| b_j / (2 pi H_j) of calc_GGAPBE96_2 (src/xc/xc_ggapbe96_2_module.f90:70-73)
    as the columns of a 3 x 3 array: the Cartesian gradient is sum_j b(:, j) D_j f with D_j the
    unscaled FD derivative along grid axis j.  cell: three lattice vectors (rows, bohr)."""
    A = np.asarray(cell, np.float64)
    vol = float(np.dot(A[0], np.cross(A[1], A[2])))
    B = 2.0 * math.pi / vol * np.array([np.cross(A[1], A[2]), np.cross(A[2], A[0]), np.cross(A[0], A[1])])
    out = np.zeros((3, 3))
    for j in range(3):
        aj = float(np.sqrt(np.sum(A[j] ** 2)))
        out[:, j] = aj * B[j] / (2.0 * math.pi * (aj / n[j]))
    return out


def gradient(f: np.ndarray, n: tuple, h: tuple, md: int = 6, bmat: np.ndarray | None = None):
    """(gx, gy, gz) of a grid function (x fastest) by the reference's FD nabla; bmat (grid_metric)
    for a non-orthogonal cell, else the grid spacings h of an orthorhombic one."""
    nab = fd_nab_coef(md)
    f3 = f.reshape(n[2], n[1], n[0])
    if bmat is not None:
        d = [_fd_derivative(f3, 2 - j, nab, md).reshape(-1) for j in range(3)]
        return tuple(bmat[c, 0] * d[0] + bmat[c, 1] * d[1] + bmat[c, 2] * d[2] for c in range(3))
    gx = _fd_derivative(f3, 2, nab, md) / h[0]
    gy = _fd_derivative(f3, 1, nab, md) / h[1]
    gz = _fd_derivative(f3, 0, nab, md) / h[2]
    return gx.reshape(-1), gy.reshape(-1), gz.reshape(-1)


def _divergence_term(rx, ry, rz, n, h, md, bmat=None):
    """sum_j D_j (f_j) with the FD nabla, as calc_PBE_x/c apply it: f_j = sum_c r_c b(c, j)
    (r_j / h_j in an orthorhombic cell), unscaled FD derivative."""
    nab = fd_nab_coef(md)
    out = np.zeros(rx.size)
    if bmat is not None:
        for j in range(3):
            f3 = (rx * bmat[0, j] + ry * bmat[1, j] + rz * bmat[2, j]).reshape(n[2], n[1], n[0])
            out += _fd_derivative(f3, 2 - j, nab, md).reshape(-1)
        return out
    for axis3, r, hj in ((2, rx, h[0]), (1, ry, h[1]), (0, rz, h[2])):
        f3 = (r / hj).reshape(n[2], n[1], n[0])
        out += _fd_derivative(f3, axis3, nab, md).reshape(-1)
    return out


def pbe(rho: np.ndarray, n: tuple, h: tuple, dV: float, md: int = 6, mu: float = 0.21951, kp: float = 0.804,
        bmat: np.ndarray | None = None):
    """calc_GGAPBE96_2 for rho of shape (nspin, ng): returns (vxc (nspin, ng), Ex, Ec).  bmat:
    grid_metric of a non-orthogonal cell (h is then unused)."""
    rho = np.atleast_2d(np.asarray(rho, np.float64))
    ns = rho.shape[0]
    beta = mu * 3.0 / math.pi ** 2
    gx, gy, gz = gradient(rho.sum(axis=0), n, h, md, bmat)
    gg = gx * gx + gy * gy + gz * gz
    pi = math.pi
    # exchange, per spin with trho = 2 rho_s (spin scaling), the gradient of the total density
    vx = np.zeros_like(rho)
    factor = 2.0 if ns == 2 else 1.0
    ex_sum = 0.0
    rt = np.zeros(rho.shape[1])      # kept across spins where a spin's density is below 1e-10
    for s in range(ns):
        trho = factor * rho[s]
        ok = trho > 1e-10
        t = np.where(ok, trho, 1.0)
        kf = np.cbrt(3.0 * pi * pi * t)
        ex_lda = -3.0 / (4.0 * pi) * kf
        vx_lda = -kf / pi
        den = 4.0 * kp * (t * kf) ** 2 + mu * gg
        Fx = 1.0 + kp - 4.0 * kp * kp * (t * kf) ** 2 / den
        ex_sum += float(np.sum(np.where(ok, t * ex_lda * Fx, 0.0)))
        v = Fx * vx_lda + 24.0 * pi * kp * kp * mu * t ** 3 * gg / den ** 2
        rt = np.where(ok, -18.0 * pi * kp * kp * mu * t ** 4 / den ** 2, rt)
        vx[s] = np.where(ok, v, 0.0) - _divergence_term(rt * gx, rt * gy, rt * gz, n, h, md, bmat)
    Ex = ex_sum / factor * dV
    # correlation (PW92 local part + PBE H)
    A00, A01, A02 = 0.031091, 0.015545, 0.016887
    alp10, alp11, alp12 = 0.21370, 0.20548, 0.11125
    bt10, bt11, bt12 = 7.5957, 1.41189e1, 1.0357e1
    bt20, bt21, bt22 = 3.5876, 6.1977, 3.6231
    bt30, bt31, bt32 = 1.6382, 3.3662, 0.88026
    bt40, bt41, bt42 = 0.49294, 0.62517, 0.49671
    const1 = 2.0 ** (4.0 / 3.0) - 2.0
    const2 = 9.0 * (2.0 ** (1.0 / 3.0) - 1.0) / 4.0
    fac = 1.0 if ns == 2 else 0.5
    C2 = (1.0 - math.log(2.0)) / pi ** 2
    C1 = beta / C2
    rhoa = rho[0] * fac
    rhob = rho[ns - 1] * fac
    trho_all = rhoa + rhob
    ok = trho_all > 1e-10
    trho = np.where(ok, trho_all, 1.0)
    zeta = np.clip((rhoa - rhob) / trho, -1.0, 1.0)
    fz = ((1.0 + zeta) ** (4.0 / 3.0) + (1.0 - zeta) ** (4.0 / 3.0) - 2.0) * const1
    kf = np.cbrt(3.0 * pi * pi * trho)
    rs = np.cbrt(3.0 / (4.0 * pi) / trho)
    rssq = np.sqrt(rs)

    def g_pw(A, alp, b1, b2, b3, b4):
        q = b1 * rssq + b2 * rs + b3 * rs * rssq + b4 * rs * rs
        e = -2.0 * A * (1.0 + alp * rs) * np.log(1.0 + 1.0 / (2.0 * A * q))
        de = alp * e / (1.0 + alp * rs) + A * (1.0 + alp * rs) / rssq * (
            b1 + 2.0 * b2 * rssq + 3.0 * b3 * rs + 4.0 * b4 * rs * rssq) / (2.0 * A * q * q + q)
        return e, de

    ec_U, deU_drs = g_pw(A00, alp10, bt10, bt20, bt30, bt40)
    ec_P, deP_drs = g_pw(A01, alp11, bt11, bt21, bt31, bt41)
    alpc, dac_drs = g_pw(A02, alp12, bt12, bt22, bt32, bt42)
    z4 = zeta ** 4
    ec_lda = ec_U - alpc * fz * const2 * (1.0 - z4) + (ec_P - ec_U) * fz * z4
    phi = 0.5 * ((1.0 + zeta) ** (2.0 / 3.0) + (1.0 - zeta) ** (2.0 / 3.0))
    T = pi * gg / (16.0 * phi ** 2 * kf * trho ** 2)
    A = C1 / (np.exp(-ec_lda / (C2 * phi ** 3)) - 1.0)
    AT = A * T
    Hs = C2 * phi ** 3 * np.log(1.0 + C1 * T * (1.0 + AT) / (1.0 + AT + AT ** 2))
    Ec = float(np.sum(np.where(ok, trho * (ec_lda + Hs), 0.0))) * dV
    drs_dn = -4.0 * pi * rs ** 4 / 9.0
    deU_dn, deP_dn, dac_dn = deU_drs * drs_dn, deP_drs * drs_dn, dac_drs * drs_dn
    dfz_dz = 4.0 / 3.0 * ((1.0 + zeta) ** (1.0 / 3.0) - (1.0 - zeta) ** (1.0 / 3.0)) * const1
    dec_dz = (-alpc * dfz_dz * const2 * (1.0 - z4) + 4.0 * alpc * fz * const2 * zeta ** 3
              + (ec_P - ec_U) * (dfz_dz * z4 + fz * 4.0 * zeta ** 3))
    with np.errstate(divide="ignore", invalid="ignore"):
        dphi_dz = np.where(np.abs(zeta) == 1.0, 0.0,
                           ((1.0 + zeta) ** (-1.0 / 3.0) - (1.0 - zeta) ** (-1.0 / 3.0)) / 3.0)
    tmp = 1.0 + AT + AT ** 2
    dH_dA = -phi ** 3 * C1 * C2 * A * T ** 3 * (2.0 + AT) / (tmp ** 2 + C1 * T * (1.0 + AT) * tmp)
    dH_dT = phi ** 3 * C1 * C2 * (1.0 + 2.0 * AT) / (tmp ** 2 + C1 * T * (1.0 + AT) * tmp)
    dH_dphi = 3.0 * Hs / phi
    dz_dn = [2.0 * rhob / trho ** 2, -2.0 * rhoa / trho ** 2]
    vc = np.zeros_like(rho)
    for s in range(ns):
        dz = dz_dn[0] if s == 0 else dz_dn[1]
        if ns == 1:
            dz = dz_dn[1]            # dz_dn(1) is overwritten by dz_dn(size_global) for one spin
        dec_dn = (deU_dn - dac_dn * fz * const2 * (1.0 - z4) + (deP_dn - deU_dn) * fz * z4 + dec_dz * dz)
        dA_dn = A * (C1 + A) / (C1 * C2 * phi ** 3) * (dec_dn - 3.0 * ec_lda / phi * dphi_dz * dz)
        v = (ec_lda + Hs + trho * dec_dn + trho * dH_dA * dA_dn
             + dH_dT * (-7.0 / 3.0 * T - trho * 2.0 * T / phi * dphi_dz * dz) + trho * dH_dphi * dphi_dz * dz)
        vc[s] = np.where(ok, v, 0.0)
    rt = np.where(ok, dH_dT * pi / (8.0 * kf * trho * phi ** 2), 0.0)
    div = _divergence_term(rt * gx, rt * gy, rt * gz, n, h, md, bmat)
    vc -= div[None, :]
    return vx + vc, Ex, Ec


def lda_pz81(rho: np.ndarray, dV: float):
    """calc_LDAPZ81 (src/xc/xc_ldapz81_module.f90:17-219) for rho of shape (nspin, ng): Slater
    exchange per spin (scaled by 2^(1/3) for two spins; non-positive densities skipped) and the
    Perdew-Zunger 1981 correlation with the von Barth-Hedin interpolation
    f(zeta) = ((1 + zeta)^(4/3) + (1 - zeta)^(4/3) - 2) / (2^(4/3) - 2) between its unpolarised
    and polarised fits (|rho_s| used, one spin split in halves).  Returns (vxc (nspin, ng), Ex,
    Ec) with the energies integrated over the cell."""
    rho = np.atleast_2d(np.asarray(rho, np.float64))
    ns = rho.shape[0]
    cnst = 2.0 ** (1.0 / 3.0) if ns == 2 else 1.0
    vx = np.zeros_like(rho)
    ex_sum = 0.0
    for s in range(ns):
        pos = rho[s] > 0.0
        exd = -cnst * 0.75 * np.cbrt(3.0 / math.pi * rho[s][pos])
        ex_sum += float(np.sum(rho[s][pos] * exd))
        vx[s][pos] = 4.0 / 3.0 * exd
    gam, b1, b2 = (-0.1423, -0.0843), (1.0529, 1.3981), (0.3334, 0.2611)
    A, B, C, D = (0.0311, 0.01555), (-0.048, -0.0269), (0.002, 0.0007), (-0.0116, -0.0048)
    fac = 0.5 if ns == 1 else 1.0
    ra, rb = np.abs(rho[0] * fac), np.abs(rho[-1] * fac)
    tr = ra + rb
    ok = tr > 0.0
    t = np.where(ok, tr, 1.0)
    rs = np.cbrt(3.0 / (4.0 * math.pi) / t)
    hi = rs >= 1.0
    sq = np.sqrt(rs)
    lnr = np.log(rs)
    ecd, mu = [], []
    for p in (0, 1):
        den = 1.0 + b1[p] * sq + b2[p] * rs
        e_hi = gam[p] / den
        m_hi = e_hi + e_hi / 3.0 * (0.5 * b1[p] / sq + b2[p]) / (1.0 / rs + b1[p] / sq + b2[p])
        e_lo = A[p] * lnr + B[p] + C[p] * rs * lnr + D[p] * rs
        m_lo = e_lo - (A[p] + C[p] * rs * (1.0 + lnr) + rs * D[p]) / 3.0
        ecd.append(np.where(hi, e_hi, e_lo))
        mu.append(np.where(hi, m_hi, m_lo))
    c0 = 1.0 / (2.0 ** (4.0 / 3.0) - 2.0)
    f = c0 * ((2.0 * ra) ** (4.0 / 3.0) + (2.0 * rb) ** (4.0 / 3.0) - 2.0 * t ** (4.0 / 3.0)) / t ** (4.0 / 3.0)
    ec_sum = float(np.sum(np.where(ok, t * (ecd[0] + (ecd[1] - ecd[0]) * f), 0.0)))
    g = c0 * 4.0 / 3.0 * 2.0 * (np.cbrt(2.0 * ra) - np.cbrt(2.0 * rb)) / t ** (4.0 / 3.0)
    dfa, dfb = g * rb, -g * ra
    base = mu[0] + (mu[1] - mu[0]) * f
    vc = np.zeros_like(rho)
    vc[0] = np.where(ok, base + (ecd[1] - ecd[0]) * dfa, 0.0)
    vc[-1] = np.where(ok, base + (ecd[1] - ecd[0]) * dfb, 0.0)
    return vx + vc, ex_sum * dV, ec_sum * dV


def _hartree_kernel(gr) -> np.ndarray:
    """4 pi / |G|^2 on the sphere's points of the half spectrum (x axis 0..N1/2), G = 0 and the
    points outside the sphere 0; cached on gr.  The sphere is symmetric under G -> -G, so the
    half spectrum carries the whole filter of a real density."""
    ker = getattr(gr, "_vh_kernel", None)
    if ker is None:
        n1, n2, n3 = gr.n
        ker = np.zeros((n3, n2, n1 // 2 + 1))
        i1 = np.mod(gr.llg[:, 0], n1)
        keep = np.any(gr.llg != 0, axis=1) & (i1 <= n1 // 2)
        ker[np.mod(gr.llg[keep, 2], n3), np.mod(gr.llg[keep, 1], n2), i1[keep]] = 4.0 * math.pi / gr.g2[keep]
        gr._vh_kernel = ker
    return ker


def hartree_sphere(rho_total: np.ndarray, gr, dV: float):
    """calc_hartree_sol_fftw: V_H(G) = 4 pi rho(G) / |G|^2 on the cut-off sphere of gr (a
    pseudo.GGrid), G = 0 excluded; returns (V_H, E_H = dV/2 sum rho V_H).  Real-to-complex
    transforms on all host threads."""
    n1, n2, n3 = gr.n
    f = scipy.fft.rfftn(rho_total.reshape(n3, n2, n1), workers=-1)
    vh = scipy.fft.irfftn(f * _hartree_kernel(gr), s=(n3, n2, n1), workers=-1).reshape(-1)
    return vh, 0.5 * dV * float(np.dot(rho_total, vh))
