"""Independent numpy formulations used to pin the C++ oracle (test helper, CPU only).

These restate the same reference formulas a second way (whole-array rolls and dense
projector matrices instead of the reference's padded-array loops), so a mistake in one
formulation shows up as a disagreement with the other.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla


def np_hpsi(prob, psi, k=0, nonlocal_on=True, vloc_on=True):
    n1, n2, n3 = prob.n
    md = prob.md
    kin = prob.kin
    psi = np.atleast_2d(psi)
    nb = psi.shape[0]
    x = psi.reshape(nb, n3, n2, n1)
    v = prob.vloc.reshape(n3, n2, n1) if vloc_on else 0.0
    out = (kin["coef_lap0"] + kin["const_k2"][k] + v) * x
    axes = (3, 2, 1)
    for m in range(1, md + 1):
        for d, ax in enumerate(axes):
            xp = np.roll(x, -m, axis=ax)  # x[i+m]
            xm = np.roll(x, m, axis=ax)   # x[i-m]
            if prob.is_complex:
                zc = kin["zcoef_kin"][k, d, md + m]
                out = out + zc * xp + np.conj(zc) * xm
            else:
                out = out + kin["coef_lap"][d, m - 1] * (xp + xm)
    out = out.reshape(nb, -1)
    if nonlocal_on and prob.nzlma > 0:
        U, D = dense_projectors(prob, k)
        out = out + (U @ (D @ (prob.dV * (U.conj().T @ psi.T)))).T
    return out


def dense_projectors(prob, k=0):
    ng = prob.ng
    dt = np.complex128 if prob.is_complex else np.float64
    U = np.zeros((ng, prob.nzlma), dtype=dt)
    for p in range(prob.nzlma):
        m = prob.mjj[p]
        np.add.at(U[:, p], prob.jjp[p, :m] - 1, prob.uvk[k][p, :m])
    D = np.zeros((prob.nzlma, prob.nzlma))
    for (l1, l2), d in zip(prob.pairs, prob.dij):
        D[l1 - 1, l2 - 1] += d
    return U, D


def np_precond(prob, g, mloop=3):
    """precond_hprsdft (src/conjugate_gradient/cgpc_hprsdft_module.f90:133-270), one band."""
    n1, n2, n3 = prob.n
    h = prob.h
    c0 = 3.0 / h ** 2
    c = -0.5 / h ** 2

    def A(v):
        x = v.reshape(n3, n2, n1)
        f = c0 * x
        for ax in (2, 1, 0):
            f = f + c * (np.roll(x, 1, axis=ax) + np.roll(x, -1, axis=ax))
        return f.ravel()

    pg = g.copy()
    r = g - A(g)
    p = r.copy()
    rr1 = float(np.vdot(r, r).real)
    if rr1 < 1e-24:
        return pg
    for it in range(1, mloop + 1):
        f = A(p)
        pAp = float(np.vdot(p, f).real)
        rr0 = rr1
        a = rr0 / pAp
        pg = pg + a * p
        if it == mloop:
            break
        r = r - a * f
        rr1 = float(np.vdot(r, r).real)
        p = r + (rr1 / rr0) * p
    return pg


def np_cg_band(prob, x, k=0, ncg=3, mloop=3, others=()):
    """One band of d/z_conjugate_gradient_1 (src/conjugate_gradient/cg_module.f90:112-754).
    others: bands the preconditioned gradient is orthogonalised against after every
    preconditioner call (cggs, src/conjugate_gradient/cggs_module.f90), classical Gram-Schmidt."""
    dV = prob.dV
    cpx = prob.is_complex
    gfac, c1sq = (-1.0, 1.0) if cpx else (-2.0, 4.0)
    x = x.copy()
    hx = np_hpsi(prob, x, k)[0]
    E = float(np.vdot(x, hx).real) * dV
    E1 = 1e10
    g = gfac * (hx - E * x)
    rb = float(np.vdot(g, g).real) * dV
    gkgk = 0.0
    p = None
    res = 0.0
    for icg in range(1, ncg + 2):
        res = rb / c1sq
        if rb < 0 or abs(E - E1) < 1e-15 or icg == ncg + 1:
            break
        pg = np_precond(prob, g, mloop)
        if len(others):
            xs = np.asarray(others)
            pg = pg - xs.T @ (xs.conj() @ pg * dV)
        rb = float(np.vdot(pg, g).real) * dV
        p = pg.copy() if icg == 1 else pg + (rb / gkgk) * p
        gkgk = rb
        hp = np_hpsi(prob, p, k)[0]
        B = np.array([[np.vdot(x, x), np.vdot(x, p)], [np.vdot(p, x), np.vdot(p, p)]]) * dV
        Am = np.array([[np.vdot(x, hx), np.vdot(x, hp)], [np.vdot(p, hx), np.vdot(p, hp)]]) * dV
        if not cpx:
            B, Am = B.real, Am.real
        w, z = sla.eigh(Am, B)
        u = z[:, 0]
        W = w[0]
        if abs(w[0] - E) > 0.1 and abs(w[1] - E) <= 0.1:
            u = z[:, 1]
            W = w[1]
        if cpx:
            u = u * (np.conj(u[0]) / abs(u[0]))
        elif u[0] < 0:
            u = -u
        E1, E = E, W
        hx = u[0] * hx + u[1] * hp
        g = gfac * (hx - W * (u[0] * x + u[1] * p))
        rb = float(np.vdot(g, g).real) * dV
        if rb / res > 1e8:
            E = E1
            continue
        x = u[0] * x + u[1] * p
    return x, E, res


def dispersion(prob, m1, m2, m3, k=0):
    """Eigenvalue of the FD kinetic operator for the plane wave exp(i theta.i), theta = 2 pi m / N."""
    md = prob.md
    kin = prob.kin
    th = [2 * np.pi * m1 / prob.n[0], 2 * np.pi * m2 / prob.n[1], 2 * np.pi * m3 / prob.n[2]]
    e = kin["coef_lap0"] + kin["const_k2"][k]
    for d in range(3):
        for m in range(1, md + 1):
            zc = kin["zcoef_kin"][k, d, md + m]
            e += 2.0 * (zc * np.exp(1j * m * th[d])).real
    return e


def principal_angles(A, B):
    """Largest principal angle (radians) between the row spaces of A and B."""
    qa, _ = np.linalg.qr(A.T)
    qb, _ = np.linalg.qr(B.T)
    s = np.linalg.svd(qa.conj().T @ qb, compute_uv=False)
    s = np.clip(s, -1.0, 1.0)
    return float(np.arccos(s.min()))


def np_cg_cggs(prob, psi, iswitch, k=0):
    """All bands of conjugate_gradient with MB_d = 1 and SWGS = iswitch, in band order: band n is
    orthogonalised against the (updated) bands m < n (1) or all other current bands (2)."""
    u = psi.copy()
    es, rs = [], []
    for n in range(u.shape[0]):
        idx = range(n) if iswitch == 1 else [m for m in range(u.shape[0]) if m != n]
        x, e, r = np_cg_band(prob, u[n], k, others=[u[m] for m in idx])
        u[n] = x
        es.append(e)
        rs.append(r)
    return u, np.array(es), np.array(rs)
