"""Norm-conserving pseudopotentials (PSV files) and the operator set-up built from them.

Host-side set-up that feeds the band update: it runs once per structure, as in the reference
(Fortran host code, called before the first sweep).  Restated from the reference:

  read_PSV                 src/ps_read_psv.f90:13-378 (PSV 2.x and xTAPP headers, local part,
                           KB projectors scaled by sqrt|D_ii|, Gaussian initial charge)
  Init_Ggrid               src/ggrid_module.f90:29-151 (cut-off sphere of the FFT box, shells)
  construct_strfac         src/strfac_module.f90:16-45
  init_ps_local            src/ps_local_module.f90:32-154 (short-range part by Simpson on the
                           log mesh, long-range erf part analytic), simp :156-194
  simc                     src/simc_module.f90:17-345 (fit of the erf parameters, MINPACK lmder1)
  construct_ps_local_fftw  src/ps_local_fftw_module.f90:12-84
  ps_nloc2_init            src/ps_nloc2_init_module.f90:72-225 (mask function, Fourier filtering
                           onto a 0.002 bohr linear mesh), opFiltering src/filtering.f90:12-180,
                           makemaskf src/maskf_module.f90:13-56, polint src/polint_module.f90:11-42
  prep_ps_nloc2            src/ps_nloc2_module.f90:42-1067 (spline interpolation, spline
                           src/spline_module.f90:11-74, Ylm src/ylm_module.f90:11-175) and the
                           folding of prep_uvk_ps_nloc2 :1070-1167
  construct_ps_initrho     src/ps_initrho_module.f90:58-134, 461-560 (analytic Gaussian charge)

Cells are given either by three orthorhombic edge lengths or by three lattice vectors (rows,
bohr; the reference's aa(:, i)), e.g. the FCC cell of its Si sample; positions are reduced
coordinates as in the reference's atom input.  Orthorhombic cells take the arithmetic of the
edge-length form unchanged.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


# ----------------------------------------------------------------------------
# PSV reader
# ----------------------------------------------------------------------------
@dataclasses.dataclass
class PseudoPotential:
    """One element's pseudopotential on its radial meshes (the reference's ps1d)."""
    zelement: float
    zps: float                # valence charge
    xc_pot: str
    nlf: int                  # angular momenta with projectors
    nrf: np.ndarray           # (nlf,) references per l
    lo: np.ndarray            # (norb,) l of each projector
    no: np.ndarray            # (norb,) reference index within its l
    anorm: np.ndarray         # (norb,) |D_ii|
    inorm: np.ndarray         # (norb,) sign(D_ii)
    dij: np.ndarray           # (norb, norb)
    nrps: np.ndarray          # (norb,) radial points of the projector (log mesh, 1-based count)
    rps: np.ndarray           # (norb,) cut-off radius
    rad: np.ndarray           # (Mr,) log mesh with r(1) = 0
    vql: np.ndarray           # (Mr,) local potential
    cdc: np.ndarray           # (Mr,) core charge (4 pi r^2 rho_c form as read)
    cdd: np.ndarray           # (Mr,) initial valence charge, 4 pi r^2 rho
    rab: np.ndarray           # (Mr,) dr/dx of the log mesh
    viod: np.ndarray          # (Mr, norb) projectors, sqrt(anorm) folded in
    parloc: np.ndarray        # (4,) erf fit of the long-range local part
    cdd_coef: np.ndarray      # (3, ngauss) a, b, c of (a + b r^2) exp(-c r^2)

    @property
    def mr(self) -> int:
        return self.rad.shape[0]

    @property
    def norb(self) -> int:
        return self.lo.shape[0]

    def printed(self) -> dict:
        """The values read_PSV prints (src/ps_read_psv.f90:341-361)."""
        return {
            "zatom": self.zelement, "mr": self.mr, "r_end": float(self.rad[-1]),
            "nrps": self.nrps.tolist(), "norb": self.norb, "lo": self.lo.tolist(),
            "rps": self.rps.tolist(), "zps": self.zps, "xc_pot": self.xc_pot,
            "parloc": self.parloc.tolist(), "nrf": self.nrf.tolist(),
            "anorm": self.anorm.tolist(), "inorm": self.inorm.tolist(),
            "sum_cdd": float(np.sum(self.cdd * self.rab)),
            "sum_cdc": float(np.sum(self.cdc * self.rab)) * 4.0 * math.pi,
        }


class _Records:
    """Fortran sequential reads over a text file: a list-directed read starts at the next
    record and takes tokens across records until it has what it asked for."""

    def __init__(self, lines):
        self.lines = lines
        self.pos = 0

    def line(self) -> str:
        s = self.lines[self.pos]
        self.pos += 1
        return s

    def values(self, n: int) -> list:
        out = []
        while len(out) < n:
            out.extend(self.line().replace(",", " ").split())
        return out[:n]

    def fixed(self, n: int, width: int, per_line: int) -> list:
        out = []
        while len(out) < n:
            s = self.line()
            for k in range(per_line):
                if len(out) == n:
                    break
                f = s[k * width:(k + 1) * width].strip()
                out.append(float(f.replace("D", "E").replace("d", "e")) if f else 0.0)
        return out


def _f(tok: str) -> float:
    return float(tok.replace("D", "E").replace("d", "e"))


def read_psv(path: str, uspp: bool = False) -> PseudoPotential:
    """read_PSV (src/ps_read_psv.f90:13-378): the local potential, the KB projectors beta
    scaled by sqrt|D_ii| (unscaled for multi-reference sets), the Gaussian initial charge.
    The ultrasoft extension (ippform > 100, readPSVG) is not read."""
    if uspp:
        raise NotImplementedError("ultrasoft PSV (readPSVG) is not supported")
    with open(path) as fh:
        rec = _Records(fh.read().splitlines())
    first = rec.line()
    if first.startswith("#PSV"):
        verpot = 2
        xc_pot, zatom, _ifchrg = rec.values(3)
        while rec.lines[rec.pos].startswith("#"):
            rec.pos += 1
        znuc = _f(rec.values(1)[0])
    elif first.startswith("#xPSV"):
        verpot = 3
        while rec.lines[rec.pos].startswith("#"):
            rec.pos += 1
        xc_pot = rec.values(1)[0]
        znuc, zatom = (_f(t) for t in rec.values(2))
    else:
        verpot = 1
        znuc, zatom = 0.0, 0.0
        xc_pot = "LDAPZ81"                     # the reader assumes LDA PZ81 for version 1
        rec.line()                             # one comment record follows the first
    xc_pot = str(xc_pot).strip("'\"")
    zatom = _f(str(zatom))
    nl = int(rec.values(1)[0])
    nr = [int(t) for t in rec.values(nl)]
    nsmpl, rc_in = rec.values(2)
    nsmpl, rc_in = int(nsmpl), _f(rc_in)
    a1, a2, a3, a4 = (_f(t) for t in rec.values(4))
    if abs(a1 + a3 - 1.0) > 1e-10:
        raise ValueError("PSV: local parameter fitting error (a1 + a3 != 1)")
    ndlc = int(rec.values(1)[0])
    # two columns (r, v) or three (r, v, core charge): the reference tells them apart by
    # reading three values from the first record
    ncol = len(rec.lines[rec.pos].split())
    rr = np.empty(ndlc)
    vl = np.empty(ndlc)
    cc = np.zeros(ndlc)
    for i in range(ndlc):
        t = rec.line().split()
        rr[i], vl[i] = _f(t[0]), _f(t[1])
        if ncol >= 3:
            cc[i] = _f(t[2])
    if rr[0] <= 0.0:
        raise ValueError("PSV: r(1) <= 0 in the local potential")
    h = math.exp(math.log(rr[-1] / rr[0]) / (ndlc - 1))
    if abs(h * rr[0] - rr[1]) > 1e-12:
        raise ValueError("PSV: local potential mesh is not logarithmic")
    rec.line()
    ndata, r1, rend, r2 = rec.values(4)
    ndata, r1, rend, r2 = int(ndata), _f(r1), _f(rend), _f(r2)
    if ndata != nsmpl:
        raise ValueError("PSV: NSMPL != NDATA")
    hn = math.exp(math.log(rend / r1) / (ndata - 1))
    rn = r1 * hn ** np.arange(ndata)
    if abs(rn[1] - r2) > 1e-6 or abs(rr[ndata - 1] - rend) > 1e-8:
        raise ValueError("PSV: nonlocal mesh differs from the local mesh")
    if math.sqrt(float(np.sum((rr[:ndata] - rn) ** 2)) / ndata) > 1e-7:
        raise ValueError("PSV: radial grid is inconsistent")
    mmax = max(nr) if nr else 0
    ddi = np.zeros((nl, mmax, mmax))
    bet = np.zeros((nl, mmax, nsmpl))
    for l in range(nl):
        rec.line()
        m = nr[l]
        v = rec.fixed(m * (m + 1) // 2, 20, 3)
        k = 0
        for j in range(m):
            for i in range(j + 1):
                ddi[l, i, j] = ddi[l, j, i] = v[k]
                k += 1
        rec.values(m * (m + 1) // 2)           # qqr (unused for norm-conserving sets)
        for j in range(m):
            rec.line()
            for i in range(nsmpl):
                t = rec.line().split()
                bet[l, j, i] = _f(t[2])
    coef = np.zeros((3, 0))
    if verpot != 3:
        while rec.pos < len(rec.lines):
            if rec.line()[:18] == "### initial charge":
                ng = int(rec.values(1)[0])
                coef = np.array([[_f(t) for t in rec.values(3)] for _ in range(ng)]).T.reshape(3, ng)
                break
        else:
            raise ValueError("PSV: no '### initial charge' section")
    else:
        raise NotImplementedError("xTAPP initial charge (.ichr file) is not read")
    mr = max(ndlc, nsmpl, ndata) + 1
    norb = sum(nr)
    lo = np.zeros(norb, np.int64)
    no = np.zeros(norb, np.int64)
    anorm = np.zeros(norb)
    inorm = np.zeros(norb)
    k = 0
    for l in range(nl):
        for j in range(nr[l]):
            lo[k], no[k] = l, j + 1
            anorm[k] = abs(ddi[l, j, j])
            inorm[k] = math.copysign(1.0, ddi[l, j, j])
            k += 1
    dij = np.zeros((norb, norb))
    for jo in range(norb):
        for io in range(norb):
            if lo[io] == lo[jo]:
                dij[io, jo] = ddi[lo[io], no[io] - 1, no[jo] - 1]
    multref = np.count_nonzero(anorm) < np.count_nonzero(dij)
    rad = np.zeros(mr)
    vql = np.zeros(mr)
    cdc = np.zeros(mr)
    rad[1:ndlc + 1] = rr
    vql[1:ndlc + 1] = vl
    cdc[1:ndlc + 1] = cc
    vql[0] = vql[1]
    viod = np.zeros((mr, norb))
    k = 0
    for l in range(nl):
        for j in range(nr[l]):
            s = 1.0 if multref else math.sqrt(anorm[k])
            viod[1:nsmpl + 1, k] = bet[l, j] * s
            k += 1
    rab, cdd = _radial_derived(rad, ndlc, coef)
    return PseudoPotential(
        zelement=zatom, zps=znuc, xc_pot=xc_pot, nlf=nl, nrf=np.array(nr, np.int64), lo=lo, no=no,
        anorm=anorm, inorm=inorm, dij=dij, nrps=np.full(norb, nsmpl + 1, np.int64),
        rps=np.full(norb, rc_in), rad=rad, vql=vql, cdc=cdc, cdd=cdd, rab=rab, viod=viod,
        parloc=np.array([a1, a2, a3, a4]), cdd_coef=coef)


def _radial_derived(rad: np.ndarray, ndlc: int, coef: np.ndarray):
    """rab = r h of the log mesh and the initial charge 4 pi r^2 sum_g (a + b r^2) exp(-c r^2)
    (terms with c r^2 > 700 skipped), both with the r = 0 point first (src/ps_read_psv.f90:293-325)."""
    mr = rad.size
    rr = rad[1:ndlc + 1]
    hl = math.log(rr[-1] / rr[0]) / (ndlc - 1)
    rab = np.zeros(mr)
    rab[1:ndlc + 1] = rr * hl
    cdd = np.zeros(mr)
    r2 = rr * rr
    for g in range(coef.shape[1]):
        a0, b0, c0 = coef[:, g]
        keep = c0 * r2 <= 700.0
        cdd[1:ndlc + 1] += np.where(keep, r2 * 4.0 * math.pi * (a0 + b0 * r2) * np.exp(-c0 * np.where(keep, r2, 0.0)), 0.0)
    return rab, cdd


_DERIVED = ("rab", "cdd")


def save_npz(pp: PseudoPotential, path: str) -> None:
    """The tables as read (the derived rab and cdd are rebuilt on load; viod is cut to its
    nonzero rows; the local mesh length is stored as ndlc)."""
    ndlc = int(np.count_nonzero(pp.rad))
    kw = {f.name: np.asarray(getattr(pp, f.name)) for f in dataclasses.fields(pp) if f.name not in _DERIVED}
    kw["viod"] = pp.viod[:int(pp.nrps.max())]
    kw["ndlc"] = np.array(ndlc)
    if not np.any(pp.cdc):
        kw["cdc"] = np.zeros(0)
    np.savez_compressed(path, **kw)


def load_npz(path: str) -> PseudoPotential:
    z = np.load(path)
    kw = {}
    mr = z["rad"].size
    for f in dataclasses.fields(PseudoPotential):
        if f.name in _DERIVED:
            continue
        v = z[f.name]
        if f.name in ("zelement", "zps"):
            v = float(v)
        elif f.name == "xc_pot":
            v = str(v)
        elif f.name == "nlf":
            v = int(v)
        elif f.name == "viod":
            full = np.zeros((mr, v.shape[1]))
            full[:v.shape[0]] = v
            v = full
        elif f.name == "cdc" and v.size == 0:
            v = np.zeros(mr)
        kw[f.name] = v
    kw["rab"], kw["cdd"] = _radial_derived(kw["rad"], int(z["ndlc"]), kw["cdd_coef"])
    return PseudoPotential(**kw)


# ----------------------------------------------------------------------------
# radial tools
# ----------------------------------------------------------------------------
def simp(f: np.ndarray, m: int = 2) -> float:
    """The reference's Simpson rule (src/ps_local_module.f90:156-194): the array is padded
    with zeros to the rule's length; for m = 2 and an even count the last point drops out."""
    f = np.asarray(f, dtype=np.float64)
    n = f.size
    nmax = (n // m) * m
    for i in range(m + 1):
        nmax += i
        if nmax >= n:
            break
    g = np.zeros(max(nmax, n))
    g[:n] = f
    if m == 2:
        k = np.arange(0, nmax - 2, 2)
        return float(np.sum(g[k] + 4.0 * g[k + 1] + g[k + 2]) / 3.0)
    if m == 4:
        k = np.arange(0, nmax - 4, 4)
        return float(np.sum(7 * g[k] + 32 * g[k + 1] + 12 * g[k + 2] + 32 * g[k + 3] + 7 * g[k + 4]) * 2.0 / 45.0)
    if m == 6:
        k = np.arange(0, nmax - 6, 6)
        return float(np.sum(41 * g[k] + 216 * g[k + 1] + 27 * g[k + 2] + 272 * g[k + 3] + 27 * g[k + 4]
                            + 216 * g[k + 5] + 41 * g[k + 6]) / 140.0)
    return float(0.5 * (f[0] + f[-1]) + np.sum(f[1:-1]))


def polint_batch(xa: np.ndarray, ya: np.ndarray, x: np.ndarray):
    """polint (src/polint_module.f90:11-42) for many points at once: Neville's tableau over
    the rows of xa/ya (one window per point); returns the value and the reference's error
    estimate (change of the mean of the last tableau column)."""
    xa = np.asarray(xa, np.float64)
    f0 = np.array(ya, dtype=np.float64, copy=True)
    n = xa.shape[1]
    f0nm = f0[:, 0].copy()
    f0nm_0 = f0nm.copy()
    for m in range(1, n):
        a = x[:, None] - xa[:, :n - m]
        b = x[:, None] - xa[:, m:]
        f0[:, :n - m] = (b * f0[:, :n - m] - a * f0[:, 1:n - m + 1]) / (b - a)
        f0nm_0 = f0nm
        f0nm = np.sum(f0[:, :n - m], axis=1) / (n - m)
    return f0[:, 0].copy(), f0nm - f0nm_0


def _polint_best(xs: np.ndarray, ys: np.ndarray, x: np.ndarray, centre: np.ndarray, lo: int, hi: int,
                 mmax: int = 20, stop: float | None = None):
    """The reference's window search around polint: windows [c - m, c + m] clipped to
    [lo, hi] for m = 1..mmax, keeping the value with the smallest error estimate (the
    first one on ties; with stop, the search ends once the error is below it)."""
    best = np.zeros(x.size)
    err0 = np.full(x.size, 1e10)
    done = np.zeros(x.size, bool)
    for m in range(1, mmax + 1):
        m1 = np.maximum(centre - m, lo)
        m2 = np.minimum(centre + m, hi)
        ln = m2 - m1 + 1
        for L in np.unique(ln):
            sel = np.nonzero((ln == L) & ~done)[0]
            if sel.size == 0:
                continue
            idx = m1[sel, None] + np.arange(L)[None, :]
            y, dy = polint_batch(xs[idx], ys[idx], x[sel])
            better = np.abs(dy) < err0[sel]
            best[sel[better]] = y[better]
            err0[sel[better]] = np.abs(dy[better])
            if stop is not None:
                done[sel[better & (np.abs(dy) < stop)]] = True
    return best, err0


def makemaskf(eta: float):
    """Mask function table (src/maskf_module.f90:13-56): the lowest eigenvector of the
    band-limited concentration matrix on 200 points of [0, 1], normalised to 1 at 0."""
    nmsk = 201
    mx = nmsk - 1
    dx = 1.0 / mx
    x = dx * np.arange(1, mx + 1)
    x1 = x[:, None]
    x2 = x[None, :]
    with np.errstate(divide="ignore", invalid="ignore"):
        X = np.sin((x1 + x2) * eta) / (x1 + x2) - np.sin((x1 - x2) * eta) / (x1 - x2)
    d = np.sin(2 * x * eta) / (2 * x) + mx * math.pi - eta
    X[np.arange(mx), np.arange(mx)] = d
    _, vec = np.linalg.eigh(X)
    v = vec[:, 0]
    c = v[0] / dx
    maskr = np.zeros(nmsk + 1)
    maskr[1:mx + 1] = v / x / c
    maskr[0] = 1.0
    maskr[nmsk] = 0.0
    xm = dx * np.arange(nmsk + 1)
    return xm, maskr, dx


def _mask_values(x: np.ndarray, xm, maskr, dxm) -> np.ndarray:
    """Mask at x = r / Rc by the polint window search of ps_nloc2_init (:106-127, :173-199)."""
    nmsk = xm.size - 1
    out = np.ones(x.size)
    sel = np.nonzero(x > dxm)[0]
    if sel.size:
        m0 = (x[sel] / dxm).astype(np.int64)
        y, _ = _polint_best(xm, maskr, x[sel], m0, 1, nmsk)
        out[sel] = y
    return out


def filter_projector(qc: float, l: int, rad: np.ndarray, rad1: np.ndarray, vrad: np.ndarray) -> np.ndarray:
    """opFiltering (src/filtering.f90:12-180) for l = 0, 1, 2: (2/pi) int_0^qc of
    j_l(q r) j_l(q r') q^2 dq against vrad on the log mesh, by the reference's Simpson rule."""
    ep = 1e-14
    const = 2.0 / math.pi
    out = np.zeros(rad1.size)
    r1 = np.asarray(rad, np.float64)
    for i, r in enumerate(rad1):
        if l == 0:
            if abs(r) <= ep:
                with np.errstate(divide="ignore", invalid="ignore"):
                    tmp = np.sin(qc * r1) / r1 ** 3 - qc * np.cos(qc * r1) / r1 ** 2
                if abs(r1[0]) <= ep:
                    tmp[0] = qc ** 3 / 3.0
            else:
                with np.errstate(divide="ignore", invalid="ignore"):
                    tmp = (np.sin(qc * (r - r1)) / (r - r1) - np.sin(qc * (r + r1)) / (r + r1)) / (2.0 * r * r1)
                tmp = np.where(np.abs(r1) <= ep, math.sin(qc * r) / r ** 3 - qc * math.cos(qc * r) / r ** 2, tmp)
                tmp = np.where(np.abs(r1 - r) <= ep, (2 * qc * r - math.sin(2 * qc * r)) / (4 * r ** 3), tmp)
        elif l == 1:
            if abs(r) <= ep:
                continue
            sb0x = math.sin(qc * r) / (qc * r)
            sb1x = sb0x / (qc * r) - math.cos(qc * r) / (qc * r)
            with np.errstate(divide="ignore", invalid="ignore"):
                sb0y = np.sin(qc * r1) / (qc * r1)
                sb1y = sb0y / (qc * r1) - np.cos(qc * r1) / (qc * r1)
                tmp = (r1 * sb0y * sb1x - r * sb0x * sb1y) * qc * qc / (r * r - r1 * r1)
            tmp = np.where(np.abs(r1 - r) <= ep,
                           (2 * qc * r - math.sin(2 * qc * r)) / (4 * r ** 3) - qc * qc * sb0x * sb1x / r, tmp)
            tmp = np.where(np.abs(r1) <= ep, 0.0, tmp)
        elif l == 2:
            if abs(r) <= ep:
                continue
            sb0x = math.sin(qc * r) / (qc * r)
            sb1x = sb0x / (qc * r) - math.cos(qc * r) / (qc * r)
            with np.errstate(divide="ignore", invalid="ignore"):
                sb0y = np.sin(qc * r1) / (qc * r1)
                sb1y = sb0y / (qc * r1) - np.cos(qc * r1) / (qc * r1)
                tmp = ((r * sb0y * sb1x - r1 * sb0x * sb1y) * qc * qc / (r * r - r1 * r1)
                       - 3.0 * qc / (r * r1) * sb1x * sb1y)
            sb1d = math.sin(qc * r) / (qc * qc * r * r) - math.cos(qc * r) / (qc * r)
            tmp = np.where(np.abs(r1 - r) <= ep,
                           (2 * qc * r - math.sin(2 * qc * r)) / (4 * r ** 3) - 3.0 * qc * sb1d * sb1d / (r * r), tmp)
            tmp = np.where(np.abs(r1) <= ep, 0.0, tmp)
        else:
            raise NotImplementedError("projector filtering for l > 2")
        out[i] = simp(tmp * vrad, 2) * const
    return out


def spline_natural(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Second derivatives of the natural cubic spline (src/spline_module.f90:11-44)."""
    n = x.size
    a = np.zeros(n)
    b = np.zeros(n)
    c = np.zeros(n)
    f = np.zeros(n)
    a[1:n - 1] = x[1:n - 1] - x[0:n - 2]
    b[1:n - 1] = (x[2:n] - x[0:n - 2]) * 2.0
    c[1:n - 2] = x[2:n - 1] - x[1:n - 2]
    f[1:n - 1] = 6.0 * ((y[2:n] - y[1:n - 1]) / (x[2:n] - x[1:n - 1]) - (y[1:n - 1] - y[0:n - 2]) / (x[1:n - 1] - x[0:n - 2]))
    for i in range(2, n - 1):
        b[i] = b[i] - a[i] * c[i - 1] / b[i - 1]
        f[i] = f[i] - a[i] * f[i - 1] / b[i - 1]
    y2 = np.zeros(n)
    y2[n - 2] = f[n - 2] / b[n - 2]
    for i in range(n - 3, 0, -1):
        y2[i] = (f[i] - c[i] * y2[i + 1]) / b[i]
    return y2


def splint(xa: np.ndarray, ya: np.ndarray, y2a: np.ndarray, x: np.ndarray) -> np.ndarray:
    """splint (src/spline_module.f90:46-74), vectorised; the bisection finds klo with
    xa[klo] <= x < xa[klo + 1] (klo = n - 2 at or past the last point)."""
    n = xa.size
    klo = np.searchsorted(xa, x, side="right") - 1
    klo = np.clip(klo, 0, n - 2)
    khi = klo + 1
    h = xa[khi] - xa[klo]
    a = ya[klo]
    b = (ya[khi] - ya[klo]) / h - (y2a[khi] + 2.0 * y2a[klo]) * h / 6.0
    c = y2a[klo] / 2.0
    d = (y2a[khi] - y2a[klo]) / (6.0 * h)
    t = x - xa[klo]
    return a + b * t + c * t ** 2 + d * t ** 3


def plm(l: int, m: int, x: np.ndarray) -> np.ndarray:
    """Associated Legendre function with the Condon-Shortley phase (src/ylm_module.f90:133-175)."""
    x = np.where(np.abs(np.abs(x) - 1.0) < 1e-13, np.sign(x), x)
    pmm = np.ones_like(x)
    if m > 0:
        somx2 = np.sqrt((1.0 - x) * (1.0 + x))
        fact = 1.0
        for _ in range(m):
            pmm = -pmm * fact * somx2
            fact += 2.0
    if l == m:
        return pmm
    pmmp1 = x * (2 * m + 1) * pmm
    if l == m + 1:
        return pmmp1
    pll = pmmp1
    for ll in range(m + 2, l + 1):
        pll = (x * (2 * ll - 1) * pmmp1 - (ll + m - 1) * pmm) / (ll - m)
        pmm, pmmp1 = pmmp1, pll
    return pll


def ylm(x: np.ndarray, y: np.ndarray, z: np.ndarray, l: int, m_in: int) -> np.ndarray:
    """Real spherical harmonics of the reference (src/ylm_module.f90:11-73); 0 at the origin for l > 0."""
    pi = 3.141592653589793238
    if l == 0:
        return np.full(np.shape(x), 1.0 / math.sqrt(4.0 * pi))
    m = abs(m_in)
    c = 1.0
    for k in range(l - m + 1, l + m + 1):
        c *= k
    clm = math.sqrt((2 * l + 1) / (c * 4.0 * pi))
    zero = (x == 0.0) & (y == 0.0) & (z == 0.0)
    r = np.sqrt(x * x + y * y + z * z)
    rs = np.where(zero, 1.0, r)
    ct = z / rs
    with np.errstate(divide="ignore", invalid="ignore"):
        phi = np.where(np.abs(x) < 1e-10, 0.5 * pi * np.where(y >= 0, 1.0, -1.0), np.arctan(y / np.where(x == 0, 1.0, x)))
    phi = np.where((np.abs(x) >= 1e-10) & (x < 0), phi + pi, phi)
    p = plm(l, m, ct)
    if m_in > 0:
        v = math.sqrt(2.0) * clm * p * np.cos(phi * m)
    elif m_in == 0:
        v = clm * p
    elif m % 2 == 0:
        v = -math.sqrt(2.0) * clm * p * np.sin(phi * m)
    else:
        v = math.sqrt(2.0) * clm * p * np.sin(phi * m)
    return np.where(zero, 0.0, v)


# ----------------------------------------------------------------------------
# local part
# ----------------------------------------------------------------------------
def fit_parloc(rad: np.ndarray, vin: np.ndarray, rc: float, zv: float) -> np.ndarray:
    """simc_0 (src/simc_module.f90:255-345): weighted least-squares fit of
    -zv/r (x1 erf(sqrt(x2) r) + (1 - x1) erf(sqrt(x3) r)) to the local potential on samples
    0.2 bohr apart, by MINPACK's lmder (tolerance 1e-5), with the reference's Jacobian."""
    from scipy.optimize import leastsq
    lam, vmax, rmax, vrzmin, smpstp, nummin = 3.5, 100.0, 10.0, 3.0e-6, 0.2, 6
    rads, vins, wgt = [], [], []
    nxt = 0.0
    for k in range(rad.size):
        if rad[k] > nxt:
            nxt += smpstp
            if abs(vin[k]) <= vmax:
                rads.append(rad[k])
                vins.append(vin[k])
                wgt.append(1.0 - math.exp(-(1.2 * rad[k] / rc) ** lam))
            if (abs(vin[k] * rad[k] + zv) < vrzmin or rad[k] > rmax) and len(rads) > nummin:
                break
    rads, vins, sw = np.array(rads), np.array(vins), np.sqrt(np.array(wgt))
    erf = np.vectorize(math.erf)

    def clamp(x):
        return np.array([x[0], max(x[1], 0.0), max(x[2], 0.0)])

    def fun(x):
        x = clamp(x)
        return (-zv / rads * (x[0] * erf(math.sqrt(x[1]) * rads) + (1.0 - x[0]) * erf(math.sqrt(x[2]) * rads)) - vins) * sw

    def jac(x):
        x = clamp(x)
        j = np.empty((rads.size, 3))
        j[:, 0] = -zv / rads * (erf(np.sqrt(x[1] * rads)) - erf(np.sqrt(x[2] * rads))) * sw
        j[:, 1] = -zv / math.sqrt(math.pi * x[1]) * x[0] * np.exp(-x[1] * rads ** 2) * sw
        j[:, 2] = -zv / math.sqrt(math.pi * x[2]) * (1.0 - x[0]) * np.exp(-x[2] * rads ** 2) * sw
        return j

    x, _, _, _, ier = leastsq(fun, np.array([1.0, 0.4, 0.6]), Dfun=jac, full_output=True, ftol=1e-5,
                              xtol=1e-5, gtol=0.0, maxfev=400, factor=100.0)
    if ier not in (1, 2, 3) or x[1] < 0 or x[2] < 0:
        raise RuntimeError(f"simc: the erf fit did not converge (info {ier})")
    return np.array([x[0], x[1], 1.0 - x[0], x[2]])


@dataclasses.dataclass
class GGrid:
    """The reference's G sphere (src/ggrid_module.f90:29-151): G = bb . (i1, i2, i3) with
    |i| <= (N - 1) / 2 and |G|^2 < Ecut, Ecut = Gcut^2 from the largest inscribed sphere."""
    n: tuple
    ecut: float
    gcut: float
    llg: np.ndarray           # (NG, 3) integer G, i1 fastest as the reference lists them
    g2: np.ndarray            # (NG,)
    mgl: np.ndarray           # (NG,) 0-based shell index
    gg: np.ndarray            # (NMGL,) shell |G|^2, ascending

    @property
    def ng(self) -> int:
        return self.llg.shape[0]

    @property
    def nmgl(self) -> int:
        return self.gg.size


def lattice(cell) -> tuple:
    """(A, orthogonal): the lattice vectors as rows of A (bohr) from three orthorhombic edge
    lengths or from a 3 x 3 array of vectors, and whether the cell is orthorhombic (the
    off-diagonal entries of A are exactly zero)."""
    c = np.asarray(cell, np.float64)
    if c.ndim == 1:
        return np.diag(c), True
    if c.shape != (3, 3):
        raise ValueError("cell: three edge lengths or three lattice vectors")
    return c.copy(), bool(np.all(c[~np.eye(3, dtype=bool)] == 0.0))


def reciprocal(A: np.ndarray) -> np.ndarray:
    """Reciprocal vectors b_i (rows) with a_i . b_j = 2 pi delta_ij (get_reciprocal_lattice)."""
    vol = float(np.dot(A[0], np.cross(A[1], A[2])))
    return 2.0 * math.pi / vol * np.array([np.cross(A[1], A[2]), np.cross(A[2], A[0]), np.cross(A[0], A[1])])


def make_ggrid(n: tuple, cell) -> GGrid:
    """Init_Ggrid for the FFT box n of the cell (edge lengths or lattice vectors): Gcut is half
    the smallest distance between opposite faces of the box's reciprocal parallelepiped
    (CalcCutoff_Ggrid, src/ggrid_module.f90:55-90), the sphere |G|^2 < Gcut^2 - 1e-14 and its
    shells (construct_NMGL_Ggrid :93-151)."""
    A, ortho = lattice(cell)
    ng = [(k - 1) // 2 for k in n]
    if ortho:
        b = [2.0 * math.pi / A[d, d] for d in range(3)]
        r = [b[d] * (2 * ng[d] + 1) for d in range(3)]
        gcut = min(r) * 0.5
    else:
        B = reciprocal(A)
        bl = [float(np.sqrt(np.sum(B[d] ** 2))) * (2 * ng[d] + 1) for d in range(3)]
        c = float(np.dot(B[0], B[1])) / (bl[0] * bl[1]) * (2 * ng[0] + 1) * (2 * ng[1] + 1)
        sn = math.sqrt(1.0 - c * c)
        b0 = np.cross(B[0], B[1])
        r3 = abs(float(np.dot(B[2], b0)) * (2 * ng[2] + 1) / math.sqrt(float(np.sum(b0 ** 2))))
        gcut = min(sn * bl[0], sn * bl[1], r3) * 0.5
    ecut = gcut * gcut
    i3, i2, i1 = np.meshgrid(np.arange(-ng[2], ng[2] + 1), np.arange(-ng[1], ng[1] + 1),
                             np.arange(-ng[0], ng[0] + 1), indexing="ij")
    i1, i2, i3 = i1.ravel(), i2.ravel(), i3.ravel()
    if ortho:
        s = (b[0] * i1) ** 2 + (b[1] * i2) ** 2 + (b[2] * i3) ** 2
    else:
        gx = [B[0, c] * i1 + B[1, c] * i2 + B[2, c] * i3 for c in range(3)]
        s = gx[0] ** 2 + gx[1] ** 2 + gx[2] ** 2
    keep = s < ecut - 1e-14
    llg = np.stack([i1[keep], i2[keep], i3[keep]], axis=1)
    g2 = s[keep]
    order = np.argsort(g2, kind="stable")
    mgl = np.zeros(g2.size, np.int64)
    shells = [0.0]
    s1 = 0.0
    k = 0
    for idx in order:
        if abs(g2[idx] - s1) > 1e-12:
            k += 1
            s1 = g2[idx]
            shells.append(s1)
        mgl[idx] = k
    return GGrid(n=tuple(n), ecut=ecut, gcut=gcut, llg=llg, g2=g2, mgl=mgl, gg=np.array(shells))


def local_form_factor(pp: PseudoPotential, gg: np.ndarray, vcell: float, parloc: np.ndarray | None = None) -> np.ndarray:
    """vqlg of init_ps_local (src/ps_local_module.f90:32-154) on the shells gg:
    (4 pi / Vcell) [int r^2 (v - v_long) j0(G r) dr + FT(v_long)]."""
    if parloc is None:
        rc = float(pp.rps.max()) if pp.norb else 0.0
        if rc < 1e-8:
            rc = 5.0
        parloc = fit_parloc(pp.rad, pp.vql, rc, pp.zps)
    const = 4.0 * math.pi / vcell
    p1, p2, p3, p4 = parloc[0], math.sqrt(parloc[1]), parloc[2], math.sqrt(parloc[3])
    r = pp.rad
    erf = np.vectorize(math.erf)
    with np.errstate(divide="ignore", invalid="ignore"):
        vlong = np.where(r < 1e-9, -2.0 * pp.zps / math.sqrt(math.pi) * (p1 * p2 + p3 * p4),
                         -pp.zps / np.where(r < 1e-9, 1.0, r) * (p1 * erf(p2 * r) + p3 * erf(p4 * r)))
    vshort = pp.vql - vlong
    base = r * r * vshort * pp.rab
    out = np.zeros(gg.size)
    for ig, g2 in enumerate(gg):
        G = math.sqrt(g2)
        if G == 0.0:
            out[ig] = simp(base, 2) * const
            continue
        x = G * r
        with np.errstate(divide="ignore", invalid="ignore"):
            sb = np.where(x < 0.1, -(x ** 10 / 39916800.0 - x ** 8 / 362880.0 + x ** 6 / 5040.0 - x ** 4 / 120.0
                                      + x ** 2 / 6.0 - 1.0), np.sin(x) / np.where(x == 0, 1.0, x))
        out[ig] = simp(base * sb, 2) * const
    q1, q2 = -pp.zps * parloc[0], 0.25 / parloc[1]
    q3, q4 = -pp.zps * parloc[2], 0.25 / parloc[3]
    with np.errstate(divide="ignore", invalid="ignore"):
        ana = np.where(gg == 0.0, -(q1 * q2 + q3 * q4) * const,
                       (q1 * np.exp(-gg * q2) + q3 * np.exp(-gg * q4)) / np.where(gg == 0.0, 1.0, gg) * const)
    return out + ana


def structure_factor(gr: GGrid, positions: np.ndarray) -> np.ndarray:
    """SGK = sum_a exp(-i 2 pi G . x_a) over the atoms of one element (src/strfac_module.f90:16-45)."""
    s = np.zeros(gr.ng, np.complex128)
    for a in positions:
        ph = 2.0 * math.pi * (gr.llg @ np.asarray(a, np.float64))
        s += np.cos(ph) - 1j * np.sin(ph)
    return s


def sphere_to_grid(gr: GGrid, vg: np.ndarray) -> np.ndarray:
    """sum_G vg(G) exp(+i G r) on the real-space grid (the backward FFT of
    construct_ps_local_fftw); returns the real part in the band update's layout (x fastest)."""
    n1, n2, n3 = gr.n
    z = np.zeros((n3, n2, n1), np.complex128)
    z[np.mod(gr.llg[:, 2], n3), np.mod(gr.llg[:, 1], n2), np.mod(gr.llg[:, 0], n1)] = vg
    return (np.fft.ifftn(z) * (n1 * n2 * n3)).real.reshape(-1)


def ionic_potential(species: list, gr: GGrid, vcell: float, parlocs: list | None = None) -> np.ndarray:
    """V_ion on the grid: sum over elements of vqlg(|G|) SGK(G), back to real space
    (construct_ps_local + construct_ps_local_fftw).  species: [(PseudoPotential, positions)]."""
    vg = np.zeros(gr.ng, np.complex128)
    for e, (pp, pos) in enumerate(species):
        vq = local_form_factor(pp, gr.gg, vcell, None if parlocs is None else parlocs[e])
        vg += vq[gr.mgl] * structure_factor(gr, pos)
    return sphere_to_grid(gr, vg)


# ----------------------------------------------------------------------------
# initial density
# ----------------------------------------------------------------------------
def initial_density(species: list, n: tuple, cell) -> np.ndarray:
    """construct_ps_initrho_r_spin (src/ps_initrho_module.f90:461-547), analytic form: the sum
    over atoms and the 27 nearest cell images of sum_g (a + b r^2) exp(-c r^2); the caller
    splits it over spins and normalises (normalize_initrho :550-560).  cell: edge lengths or
    lattice vectors."""
    A, ortho = lattice(cell)
    n1, n2, n3 = n
    i3, i2, i1 = np.meshgrid(np.arange(n3), np.arange(n2), np.arange(n1), indexing="ij")
    f1, f2, f3 = (i1 / n1).ravel(), (i2 / n2).ravel(), (i3 / n3).ravel()
    rho = np.zeros(n1 * n2 * n3)
    for pp, pos in species:
        for a in pos:
            for j3 in (-1, 0, 1):
                for j2 in (-1, 0, 1):
                    for j1 in (-1, 0, 1):
                        d1, d2, d3 = f1 - a[0] - j1, f2 - a[1] - j2, f3 - a[2] - j3
                        if ortho:
                            x, y, z = A[0, 0] * d1, A[1, 1] * d2, A[2, 2] * d3
                        else:
                            x, y, z = (A[0, c] * d1 + A[1, c] * d2 + A[2, c] * d3 for c in range(3))
                        rr = x * x + y * y + z * z
                        for g in range(pp.cdd_coef.shape[1]):
                            ca, cb, cc = pp.cdd_coef[:, g]
                            rho += (ca + cb * rr) * np.exp(-cc * rr)
    return rho


# ----------------------------------------------------------------------------
# nonlocal part
# ----------------------------------------------------------------------------
@dataclasses.dataclass
class FilteredProjectors:
    """Projectors after ps_nloc2_init: on the linear mesh rad1 = (i - 1) dr, masked."""
    rps: np.ndarray           # (norb,) new cut-off radius (a log-mesh point >= rcfac * Rc)
    nrps: np.ndarray          # (norb,) points of the linear mesh
    rad1: np.ndarray          # (max nrps,)
    viod: list                # per orbital (nrps,) values
    y2a: list                 # per orbital spline second derivatives


def filter_projectors(pp: PseudoPotential, qcut: float, rcfac: float = 1.5, qcfac: float = 1.0,
                      etafac: float = 8.0, dr: float = 2.0e-3) -> FilteredProjectors:
    """ps_nloc2_init (src/ps_nloc2_init_module.f90:72-225) with the reference's defaults
    rcfac 1.5, qcfac 1.0, etafac 8.0: widen the cut-off to rcfac Rc, divide by the mask,
    Fourier-filter at qc = qcfac Gcut onto a 0.002 bohr linear mesh, multiply by the mask."""
    qc = qcut * qcfac
    if qc <= 0.0:
        qc = qcut
    xm, maskr, dxm = makemaskf(etafac)
    rad = pp.rad
    nrps_new, rps_new = [], []
    for k in range(pp.norb):
        rc = pp.rps[k] * rcfac
        i0 = int(np.argmin(np.abs(rad - rc)))
        if rad[i0] < rc:
            i0 += 1
        if i0 >= rad.size:
            raise ValueError("rcfac is too large")
        nrps_new.append(i0 + 1)
        rps_new.append(rad[i0])
    nrps_lin = []
    for k in range(pp.norb):
        m = int(rps_new[k] / dr) + 1
        if (m - 1) * dr < rps_new[k]:
            m += 1
        nrps_lin.append(m)
    mlin = max(nrps_lin)
    rad1 = dr * np.arange(max(mlin, pp.mr))
    out_v, out_y2 = [], []
    for k in range(pp.norb):
        nrc_new = nrps_new[k]
        wm = _mask_values(rad[:nrc_new] / rps_new[k], xm, maskr, dxm)
        nrc0 = int(pp.nrps[k])
        vrad = rad[:nrc0] * pp.viod[:nrc0, k] * pp.rab[:nrc0] / wm[:nrc0]
        v = filter_projector(qc, int(pp.lo[k]), rad[:nrc0], rad1[:nrps_lin[k]], vrad)
        wl = _mask_values(rad1[:nrps_lin[k]] / rps_new[k], xm, maskr, dxm)
        v = v * wl
        out_v.append(v)
        out_y2.append(spline_natural(rad1[:nrps_lin[k]], v))
    return FilteredProjectors(rps=np.array(rps_new), nrps=np.array(nrps_lin, np.int64),
                              rad1=rad1[:mlin], viod=out_v, y2a=out_y2)


@dataclasses.dataclass
class ProjectorSet:
    """Grid projectors in the band update's layout (prep_ps_nloc2 + prep_uvk_ps_nloc2)."""
    nzlma: int
    mjj: np.ndarray           # (nzlma,)
    jjp: np.ndarray           # (nzlma, maxmjj) 1-based grid index
    uv: np.ndarray            # (nzlma, maxmjj)
    iuv: np.ndarray           # (nzlma,) sign of D_ii
    amap: np.ndarray
    lmap: np.ndarray
    mmap: np.ndarray
    uvk: np.ndarray | None = None   # (nk, nzlma, maxmjj) with the k phases, when k-points are given


def grid_projectors(species: list, filtered: list, n: tuple, cell, kbb: np.ndarray | None = None) -> ProjectorSet:
    """prep_ps_nloc2 (src/ps_nloc2_module.f90:42-1067): for each atom and projector, the grid
    points (periodic images included) within the filtered cut-off, the spline-interpolated
    radial value (0 at the atom itself for l > 0) times Ylm; then prep_uvk_ps_nloc2's folding
    (:1070-1167): repeated grid points summed, |u| <= 1e-14 dropped, in first-seen order.
    cell: edge lengths or lattice vectors.  kbb (nk, 3) reduced k: the folded values carry the
    phase exp(-i 2 pi k . (i / N + m)) of the unfolded point (in-cell index i, image m), as the
    complex16 build folds them; ProjectorSet.uvk then holds (nk, nzlma, maxmjj) complex values."""
    A, ortho = lattice(cell)
    B = reciprocal(A)
    n1, n2, n3 = n
    jj_all, uv_all, iuv, amap, lmap, mmap = [], [], [], [], [], []
    uvk_all = []
    atom_id = 0
    for (pp, pos), fp in zip(species, filtered):
        for a in pos:
            atom_id += 1
            if ortho:
                R = np.array([a[0] * A[0, 0], a[1] * A[1, 1], a[2] * A[2, 2]])
            else:
                R = np.array([a[0] * A[0, c] + a[1] * A[1, c] + a[2] * A[2, c] for c in range(3)])
            ic = [int(round(a[d] * n[d])) for d in range(3)]
            for k in range(pp.norb):
                l = int(pp.lo[k])
                rps2 = fp.rps[k] ** 2
                if ortho:
                    hw = [int(math.ceil(fp.rps[k] / (A[d, d] / n[d]))) + 2 for d in range(3)]
                else:
                    hw = [int(math.ceil(fp.rps[k] * float(np.linalg.norm(B[d])) * n[d] / (2.0 * math.pi))) + 2
                          for d in range(3)]
                o3, o2, o1 = np.meshgrid(np.arange(-hw[2], hw[2] + 1), np.arange(-hw[1], hw[1] + 1),
                                         np.arange(-hw[0], hw[0] + 1), indexing="ij")
                id1, id2, id3 = (ic[0] + o1).ravel(), (ic[1] + o2).ravel(), (ic[2] + o3).ravel()
                if ortho:
                    x = A[0, 0] * (id1 / n1) - R[0]
                    y = A[1, 1] * (id2 / n2) - R[1]
                    z = A[2, 2] * (id3 / n3) - R[2]
                else:
                    x, y, z = (A[0, c] * (id1 / n1) + A[1, c] * (id2 / n2) + A[2, c] * (id3 / n3) - R[c]
                               for c in range(3))
                r2 = x * x + y * y + z * z
                keep = r2 <= rps2 + 1e-10
                id1, id2, id3, x, y, z, r2 = (q[keep] for q in (id1, id2, id3, x, y, z, r2))
                r = np.sqrt(r2)
                nrc = int(fp.nrps[k])
                rad1 = fp.rad1[:nrc]
                v0 = splint(rad1, fp.viod[k], fp.y2a[k], r)
                at_atom = (np.abs(x) <= 1e-14) & (np.abs(y) <= 1e-14) & (np.abs(z) <= 1e-14)
                if l > 0:
                    v0 = np.where(at_atom, 0.0, v0)
                lin = np.mod(id1, n1) + n1 * np.mod(id2, n2) + n1 * n2 * np.mod(id3, n3)
                for m in range(-l, l + 1):
                    u = v0 * ylm(x, y, z, l, m)
                    big = np.abs(u) > 1e-14
                    uniq, first, inv = np.unique(lin[big], return_index=True, return_inverse=True)
                    rank = np.empty_like(first)
                    rank[np.argsort(first, kind="stable")] = np.arange(first.size)
                    slot = rank[inv]
                    jj_all.append(uniq[np.argsort(first, kind="stable")])
                    uv_all.append(np.bincount(slot, weights=u[big], minlength=first.size))
                    if kbb is not None:
                        ub = u[big]
                        t = np.stack([id1[big] / n1, id2[big] / n2, id3[big] / n3], axis=1)
                        ph = 2.0 * math.pi * (t @ np.asarray(kbb, np.float64).T)      # (npts, nk)
                        zk = (np.cos(ph) - 1j * np.sin(ph)) * ub[:, None]
                        uvk_all.append(np.stack([np.bincount(slot, weights=zk[:, q].real, minlength=first.size)
                                                 + 1j * np.bincount(slot, weights=zk[:, q].imag,
                                                                    minlength=first.size)
                                                 for q in range(zk.shape[1])]))
                    iuv.append(pp.inorm[k])
                    amap.append(atom_id)
                    lmap.append(l)
                    mmap.append(m)
    nzlma = len(jj_all)
    maxmjj = max(len(j) for j in jj_all)
    mjj = np.array([len(j) for j in jj_all], np.int32)
    jjp = np.zeros((nzlma, maxmjj), np.int32)
    uv = np.zeros((nzlma, maxmjj))
    uvk = None if kbb is None else np.zeros((len(kbb), nzlma, maxmjj), np.complex128)
    for p in range(nzlma):
        jjp[p, :mjj[p]] = jj_all[p] + 1
        uv[p, :mjj[p]] = uv_all[p]
        if uvk is not None:
            uvk[:, p, :mjj[p]] = uvk_all[p]
    return ProjectorSet(nzlma=nzlma, mjj=mjj, jjp=jjp, uv=uv, iuv=np.array(iuv), amap=np.array(amap, np.int32),
                        lmap=np.array(lmap, np.int32), mmap=np.array(mmap, np.int32), uvk=uvk)
