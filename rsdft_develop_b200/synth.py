"""Seeded synthetic RSDFT band-update problems.

The reference reads pseudopotential files and builds V_loc from an SCF density;
this module replaces both with seeded synthetic data of the same *form*, so the
GPU library and the CPU oracle receive bit-identical FP64 inputs:

* grid / cell: cubic cell, ``Hgrid = L/N`` and ``dV = L^3/N^3`` as in
  ``src/rgrid_sol_module.f90:25-38``;
* FD coefficients: ``src/fd_module.f90:18-78`` (``get_coef_lapla_fd`` and
  ``get_coef_nabla_fd``) restated exactly;
* kinetic coefficients ``coef_lap``, ``coef_lap0``, ``coef_nabk``,
  ``zcoef_kin`` and ``const_k2``: ``src/kinetic/kinetic_module.f90:59-162``
  for a cubic cell (``ggg(1:3)=1``, ``ggg(4:6)=0``);
* V_loc: a sum of Gaussians with seeded depth/width/centre;
* nonlocal projectors: Gaussian radial x real Y_lm on sphere footprints with
  periodic images, folded onto the grid exactly as ``prep_uvk_ps_nloc2``
  (``src/ps_nloc2_module.f90:1070-1167``): duplicate grid points from different
  images are summed, entries with ``|uV| <= 1e-14`` are dropped, and for k-points
  ``z_uVk = exp(-i 2 pi kbb.(i/N + m)) uV``;
* the per-atom coupling matrices are delivered in the reference's
  multi-reference pair form (``nzqr_pair``/``Dij00``,
  ``src/ps_nloc_mr_module.f90:852-897``), generalised to a dense symmetric
  block per atom (the reference's own form is the subset with different (l,m)
  entries zeroed, ``reference_form=True``);
* initial wavefunctions: a counter-based generator (splitmix64 + Irwin-Hall
  sum of 12 uniforms, mean 0 / variance 1) whose arithmetic is exact, so the
  CUDA library's device-side generator produces the same bits.
"""
from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass, field

import numpy as np

__all__ = [
    "Config", "Problem", "CONFIGS", "get_config", "fd_lap_coef", "fd_nab_coef",
    "kinetic_coefficients", "make_problem", "random_wavefunctions",
    "monkhorst_pack",
]


# ----------------------------------------------------------------------------
# finite-difference weights (src/fd_module.f90:18-78)
# ----------------------------------------------------------------------------
def fd_lap_coef(md: int) -> np.ndarray:
    """Central-difference weights of d^2/dx^2, ``lap(-Md:Md)`` with ``h=1``.

    Restates ``get_coef_lapla_fd`` (src/fd_module.f90:18-54) loop for loop.
    Returned array index ``m + md`` holds ``lap(m)``.
    """
    lap = np.zeros(2 * md + 1)
    s = 0.0
    for i in range(-md, md + 1):
        if i == 0:
            continue
        for j in range(-md, md + 1):
            if j == i or j == 0:
                continue
            s += 1.0 / float(i * j)
    lap[md] = s
    for j in range(1, md + 1):
        t = 1.0
        for i in range(-md, md + 1):
            if i == j:
                continue
            t *= (j - i)
        s = 0.0
        for k in range(-md, md + 1):
            if k == j or k == 0:
                continue
            s0 = 1.0
            for i in range(-md, md + 1):
                if i == k or i == j or i == 0:
                    continue
                s0 *= (-i)
            s += s0
        lap[md + j] = 2.0 * s / t
        lap[md - j] = lap[md + j]
    return lap


def fd_nab_coef(md: int) -> np.ndarray:
    """Central-difference weights of d/dx, ``nab(-Md:Md)`` (src/fd_module.f90:56-78).

    Note the reference stores ``nab(-j) = nab(j)`` (the sign is carried by the
    ``zcoef_kin`` construction), and so does this restatement.
    """
    nab = np.zeros(2 * md + 1)
    for j in range(1, md + 1):
        t = 1.0
        for i in range(-md, md + 1):
            if i == j:
                continue
            t *= (j - i)
        s = 1.0
        for i in range(-md, md + 1):
            if i == j or i == 0:
                continue
            s *= (-i)
        nab[md + j] = s / t
        nab[md - j] = nab[md + j]
    return nab


def kinetic_coefficients(h: float, md: int, kcart: np.ndarray) -> dict:
    """``init_kinetic`` for a cubic cell (src/kinetic/kinetic_module.f90:28-162).

    ``kcart`` is ``(nk, 3)`` Cartesian k (bohr^-1).  Returns ``coef_lap (3, md)``
    (index ``n-1`` holds ``coef_lap(:, n)``), ``coef_lap0``, ``coef_nabk
    (nk, 3, md)``, ``const_k2 (nk,)`` and ``zcoef_kin (nk, 3, 2md+1)`` with index
    ``m + md`` holding ``zcoef_kin(:, m, k)``.
    """
    lap = fd_lap_coef(md)
    nab = fd_nab_coef(md)
    ggg = np.ones(3)  # cubic cell: a_i^2 |b_i|^2 / (4 pi^2) = 1
    c = -0.5 * ggg / h**2
    coef_lap0 = lap[md] * c.sum()
    coef_lap = np.array([[lap[md + n] * c[d] for n in range(1, md + 1)] for d in range(3)])
    coef_nab = np.array([[nab[md + n] / h for n in range(1, md + 1)] for d in range(3)])
    kcart = np.atleast_2d(np.asarray(kcart, dtype=np.float64))
    nk = kcart.shape[0]
    coef_nabk = np.zeros((nk, 3, md))
    const_k2 = np.zeros(nk)
    zcoef = np.zeros((nk, 3, 2 * md + 1), dtype=np.complex128)
    for k in range(nk):
        for d in range(3):
            coef_nabk[k, d, :] = coef_nab[d, :] * kcart[k, d]
        const_k2[k] = 0.5 * float(np.dot(kcart[k], kcart[k]))
        for n in range(1, md + 1):
            zcoef[k, :, md - n] = coef_lap[:, n - 1] + 1j * coef_nabk[k, :, n - 1]
            zcoef[k, :, md + n] = coef_lap[:, n - 1] - 1j * coef_nabk[k, :, n - 1]
    return dict(coef_lap=coef_lap, coef_lap0=coef_lap0, coef_nab=coef_nab,
                coef_nabk=coef_nabk, const_k2=const_k2, zcoef_kin=zcoef, ggg=ggg)


def kinetic_coefficients_lattice(avec: np.ndarray, n: tuple, md: int, kbb: np.ndarray) -> dict:
    """``init_kinetic`` for any cell (src/kinetic/kinetic_module.f90:28-162, get_ggg_kinetic
    :196-211).  ``avec`` holds the lattice vectors a_i as rows (bohr), ``n`` the grid, ``kbb``
    ``(nk, 3)`` reduced k.  ggg(1:6) = |a_i||a_j| b_i . b_j / (4 pi^2) for the axis pairs
    (1,1), (2,2), (3,3), (1,2), (2,3), (3,1); coef_lap(d, m) = -ggg(d) lap(m) / (2 H_d^2),
    coef_nab(d, m) = nab(m) / H_d, and the k term c_d = |a_d| b_d . k / (2 pi) in coef_nabk.
    The off-diagonal ggg enter the stencil as -ggg(4) D_1 D_2 - ggg(5) D_2 D_3 - ggg(6) D_3 D_1.
    Same keys as :func:`kinetic_coefficients` plus ``hgrid``; ``ggg`` has six entries."""
    A = np.asarray(avec, dtype=np.float64)
    vol = float(np.dot(A[0], np.cross(A[1], A[2])))
    B = 2.0 * math.pi / vol * np.array([np.cross(A[1], A[2]), np.cross(A[2], A[0]), np.cross(A[0], A[1])])
    alen = np.sqrt(np.sum(A * A, axis=1))
    hgrid = alen / np.asarray(n, dtype=np.float64)
    const = 1.0 / (4.0 * math.pi ** 2)
    pair = ((0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (2, 0))
    ggg = np.array([alen[i] * alen[j] * float(np.dot(B[i], B[j])) * const for i, j in pair])
    lap = fd_lap_coef(md)
    nab = fd_nab_coef(md)
    c = -0.5 * ggg[:3] / hgrid ** 2
    coef_lap0 = lap[md] * (c[0] + c[1] + c[2])
    coef_lap = np.array([[lap[md + m] * c[d] for m in range(1, md + 1)] for d in range(3)])
    coef_nab = np.array([[nab[md + m] / hgrid[d] for m in range(1, md + 1)] for d in range(3)])
    kbb = np.atleast_2d(np.asarray(kbb, dtype=np.float64))
    nk = kbb.shape[0]
    kcart = kbb @ B
    coef_nabk = np.zeros((nk, 3, md))
    const_k2 = np.zeros(nk)
    zcoef = np.zeros((nk, 3, 2 * md + 1), dtype=np.complex128)
    for k in range(nk):
        ck = alen / (2.0 * math.pi) * (B @ kcart[k])
        for d in range(3):
            coef_nabk[k, d, :] = coef_nab[d, :] * ck[d]
        const_k2[k] = 0.5 * float(np.dot(kcart[k], kcart[k]))
        for m in range(1, md + 1):
            zcoef[k, :, md - m] = coef_lap[:, m - 1] + 1j * coef_nabk[k, :, m - 1]
            zcoef[k, :, md + m] = coef_lap[:, m - 1] - 1j * coef_nabk[k, :, m - 1]
    return dict(coef_lap=coef_lap, coef_lap0=coef_lap0, coef_nab=coef_nab, coef_nabk=coef_nabk,
                const_k2=const_k2, zcoef_kin=zcoef, ggg=ggg, hgrid=hgrid, kcart=kcart)


def generate_bz(mmm, use_inversion: int = 1):
    """k-points and weights of generate_bz without symmetry operations (src/bz_module.f90:65-189,
    Monkhorst_Pack :530-557): the MP mesh on the common integer grid of nk points per axis, k and
    -k merged (weight 2) unless use_inversion < 1, in the reference's loop order.  mmm = (0, 0, 0)
    is Gamma-point sampling.  Returns (kbb (N, 3) reduced, weights (N,))."""
    m1 = [int(x) for x in mmm]
    if all(x == 0 for x in m1):
        nk, mm1, mm2 = 2, [2, 2, 2], [2, 2, 2]
    else:
        lcm12 = m1[0] * m1[1] // math.gcd(m1[0], m1[1])
        nk = 2 * (lcm12 * m1[2] // math.gcd(lcm12, m1[2]))
        mm2 = [nk // x for x in m1]
        mm1 = [mm2[i] * m1[i] if m1[i] % 2 == 1 else (nk // 2) // m1[i] + mm2[i] * m1[i] for i in range(3)]
    iw0 = -1 if use_inversion >= 1 else 1
    seen = set()
    pts, wts = [], []
    for i1 in range(-mm1[0], mm1[0] + 1, mm2[0]):
        for i2 in range(-mm1[1], mm1[1] + 1, mm2[1]):
            for i3 in range(-mm1[2], mm1[2] + 1, mm2[2]):
                for iw in range(1, iw0 - 1, -2):
                    p = []
                    for v in (i1 * iw, i2 * iw, i3 * iw):
                        q = int(math.fmod(v, nk))
                        if q > nk // 2:
                            q -= nk
                        if q <= -nk // 2:
                            q += nk
                        p.append(q)
                    p = tuple(p)
                    if p in seen:
                        break
                    if iw == 1:
                        pts.append(p)
                        wts.append(1)
                    else:
                        wts[-1] = 2
                    seen.add(p)
    mmbz = len(seen)
    return np.array(pts, dtype=np.float64) / nk, np.array(wts, dtype=np.float64) / mmbz


def monkhorst_pack(n: int) -> np.ndarray:
    """Reduced Monkhorst-Pack points ``(2r - n - 1)/(2n)`` per axis (src/bz_module.f90:530-557)."""
    r = np.arange(1, n + 1)
    g = (2 * r - n - 1) / (2.0 * n)
    pts = np.array([[a, b, c] for a in g for b in g for c in g])
    return pts


# ----------------------------------------------------------------------------
# configurations
# ----------------------------------------------------------------------------
@dataclass
class Config:
    name: str
    n: int                 # grid points per axis (cubic)
    h: float               # grid spacing (bohr)
    nband: int             # bands (per k-point, unless nband_k is given)
    n_gauss: int           # Gaussians in V_loc
    natom: int             # atoms carrying projectors
    lmax: int              # 0: s, 1: s+p, 2: s+p+d
    rc: float              # projector cutoff radius (bohr)
    md: int = 6
    seed: int = 0
    mp: int = 0            # Monkhorst-Pack divisions (0: Gamma only, real8 build)
    nband_range: tuple | None = None  # uneven active band counts per k (seeded)
    reference_form: bool = False       # Dij restricted to equal (l,m) pairs
    dij_sigma: float = 0.5
    kpoints: tuple | None = None       # explicit reduced k-points (complex16), e.g. a band trajectory

    @property
    def L(self) -> float:
        return self.n * self.h

    @property
    def is_complex(self) -> bool:
        return self.mp > 0 or self.kpoints is not None


CONFIGS = {
    # plain method, real8 Gamma, 24^3 (h=0.35), 32 bands, 8 Gaussians, 8 s+p atoms rc 2.0
    "c0": Config("c0", n=24, h=0.35, nband=32, n_gauss=8, natom=8, lmax=1, rc=2.0),
    # plain FP64 GPU drop-in, 64^3 (h=0.3), 256 bands, 64 Gaussians, 64 s+p atoms rc 2.2
    "c1": Config("c1", n=64, h=0.3, nband=256, n_gauss=64, natom=64, lmax=1, rc=2.2),
    # mixed precision, 96^3, 1024 bands, 216 s+p+d atoms
    "c2": Config("c2", n=96, h=0.3, nband=1024, n_gauss=216, natom=216, lmax=2, rc=2.2),
    # learned preconditioner, 128^3, 2048 bands, 512 s+p atoms
    "c3": Config("c3", n=128, h=0.3, nband=2048, n_gauss=512, natom=512, lmax=1, rc=2.2),
    # complex16 k-points: 64^3, 8 MP k-points, 256-512 active bands, 128 s+p atoms
    "c4": Config("c4", n=64, h=0.3, nband=512, n_gauss=128, natom=128, lmax=1, rc=2.2,
                 mp=2, nband_range=(256, 512)),
    # small cases for tests
    "t0": Config("t0", n=16, h=0.4, nband=8, n_gauss=4, natom=2, lmax=1, rc=1.6),
    "t1": Config("t1", n=20, h=0.4, nband=16, n_gauss=6, natom=4, lmax=2, rc=1.8),
    "tk": Config("tk", n=16, h=0.4, nband=8, n_gauss=4, natom=2, lmax=1, rc=1.6, mp=2,
                 nband_range=(6, 8)),
}


def get_config(name: str, **over) -> Config:
    cfg = CONFIGS[name]
    return dataclasses.replace(cfg, **over) if over else cfg


# ----------------------------------------------------------------------------
# problem
# ----------------------------------------------------------------------------
@dataclass
class Problem:
    cfg: Config
    n: tuple            # (N1, N2, N3)
    h: float
    dV: float
    md: int
    kin: dict
    vloc: np.ndarray    # (Ng,) float64
    # projectors in the reference layout (C order == Fortran JJP(MAXMJJ,nzlma))
    nzlma: int
    mjj: np.ndarray     # (nzlma,) int32
    jjp: np.ndarray     # (nzlma, maxmjj) int32, 1-based grid index
    uvk: np.ndarray     # (nk, nzlma, maxmjj) float64 or complex128
    amap: np.ndarray    # (nzlma,) int32 atom (1-based)
    lmap: np.ndarray    # (nzlma,) int32
    mmap: np.ndarray    # (nzlma,) int32
    pairs: np.ndarray   # (npair, 2) int32 (lma1, lma2), 1-based
    dij: np.ndarray     # (npair,) float64
    kbb: np.ndarray     # (nk, 3) reduced k
    kcart: np.ndarray   # (nk, 3)
    nband_k: np.ndarray  # (nk,) active bands per k

    @property
    def ng(self) -> int:
        return self.n[0] * self.n[1] * self.n[2]

    @property
    def nk(self) -> int:
        return self.kbb.shape[0]

    @property
    def is_complex(self) -> bool:
        return self.cfg.is_complex

    @property
    def maxmjj(self) -> int:
        return self.jjp.shape[1]

    @property
    def nband(self) -> int:
        return int(self.nband_k.max())


def _ylm_real(l: int, m: int, x, y, z, r):
    """Real spherical harmonics (Cartesian form); zero at the origin for l>0."""
    pi = math.pi
    with np.errstate(invalid="ignore", divide="ignore"):
        if l == 0:
            return np.full_like(r, 1.0 / math.sqrt(4 * pi))
        rr = np.where(r > 0, r, 1.0)
        if l == 1:
            c = math.sqrt(3.0 / (4 * pi))
            v = {-1: y, 0: z, 1: x}[m] / rr
        elif l == 2:
            r2 = rr * rr
            if m == -2:
                v = math.sqrt(15.0 / (4 * pi)) * x * y / r2
            elif m == -1:
                v = math.sqrt(15.0 / (4 * pi)) * y * z / r2
            elif m == 0:
                v = math.sqrt(5.0 / (16 * pi)) * (3 * z * z - r * r) / r2
            elif m == 1:
                v = math.sqrt(15.0 / (4 * pi)) * x * z / r2
            else:
                v = math.sqrt(15.0 / (16 * pi)) * (x * x - y * y) / r2
            c = 1.0
        else:
            raise ValueError("lmax <= 2 supported")
        out = c * v
    return np.where(r > 0, out, 0.0)


def _gaussian_vloc(cfg: Config, rng: np.random.Generator) -> np.ndarray:
    n, h, L = cfg.n, cfg.h, cfg.L
    ng = n ** 3
    centres = rng.uniform(0.0, L, size=(cfg.n_gauss, 3))
    depth = rng.uniform(-2.0, -0.5, size=cfg.n_gauss)
    width = rng.uniform(0.8, 1.5, size=cfg.n_gauss)
    v = np.zeros(ng)
    for g in range(cfg.n_gauss):
        hw = int(math.ceil(5.0 * width[g] / h))
        c = centres[g] / h
        base = np.floor(c).astype(np.int64)
        off = np.arange(-hw, hw + 2)
        i1 = base[0] + off
        i2 = base[1] + off
        i3 = base[2] + off
        d1 = (i1 * h - centres[g][0]) ** 2
        d2 = (i2 * h - centres[g][1]) ** 2
        d3 = (i3 * h - centres[g][2]) ** 2
        r2 = d3[:, None, None] + d2[None, :, None] + d1[None, None, :]
        val = depth[g] * np.exp(-r2 / width[g] ** 2)
        idx = (np.mod(i3, n)[:, None, None] * n * n + np.mod(i2, n)[None, :, None] * n
               + np.mod(i1, n)[None, None, :])
        v += np.bincount(idx.ravel(), weights=val.ravel(), minlength=ng)
    return v


def _projectors(cfg: Config, rng: np.random.Generator, kbb: np.ndarray):
    """Sphere footprints + folding, following prep_uvk_ps_nloc2 (src/ps_nloc2_module.f90:1070-1167)."""
    n, h, L = cfg.n, cfg.h, cfg.L
    atoms = rng.uniform(0.0, L, size=(cfg.natom, 3))
    sigma = cfg.rc / 2.5
    lm = [(l, m) for l in range(cfg.lmax + 1) for m in range(-l, l + 1)]
    hw = int(math.ceil(cfg.rc / h)) + 1
    jj_all, uv_all, amap, lmap, mmap = [], [], [], [], []
    dV = h ** 3
    nk = kbb.shape[0]
    for a in range(cfg.natom):
        c = atoms[a] / h
        base = np.floor(c).astype(np.int64)
        off = np.arange(-hw, hw + 2)
        g3, g2, g1 = np.meshgrid(base[2] + off, base[1] + off, base[0] + off, indexing="ij")
        g1 = g1.ravel(); g2 = g2.ravel(); g3 = g3.ravel()
        x = g1 * h - atoms[a][0]
        y = g2 * h - atoms[a][1]
        z = g3 * h - atoms[a][2]
        r = np.sqrt(x * x + y * y + z * z)
        inside = r <= cfg.rc
        g1, g2, g3, x, y, z, r = (q[inside] for q in (g1, g2, g3, x, y, z, r))
        w1, w2, w3 = np.mod(g1, n), np.mod(g2, n), np.mod(g3, n)
        m1, m2, m3 = (g1 - w1) // n, (g2 - w2) // n, (g3 - w3) // n
        lin = w1 + w2 * n + w3 * n * n            # 0-based
        radial = np.exp(-(r / sigma) ** 2)
        for (l, m) in lm:
            u = (r ** l) * radial * _ylm_real(l, m, x, y, z, r)
            u = u / math.sqrt(float(np.sum(u * u)) * dV)
            # fold duplicates / drop tiny values (prep_uvk_ps_nloc2, :1114-1127 and :1145-1158)
            kidx = np.nonzero(np.abs(u) > 1.0e-14)[0]
            uniq, first, inv = np.unique(lin[kidx], return_index=True, return_inverse=True)
            # slot order = order of first occurrence, as the reference's running counter j
            rank = np.empty_like(first)
            rank[np.argsort(first, kind="stable")] = np.arange(first.size)
            slot = rank[inv]
            jj = uniq[np.argsort(first, kind="stable")]
            uvk = np.zeros((nk, jj.size), dtype=np.complex128)
            for kk in range(nk):
                d = 2.0 * math.pi * kbb[kk]
                kr = (d[0] * (w1[kidx] / n + m1[kidx]) + d[1] * (w2[kidx] / n + m2[kidx])
                      + d[2] * (w3[kidx] / n + m3[kidx]))
                val = (np.cos(kr) - 1j * np.sin(kr)) * u[kidx]
                uvk[kk] = (np.bincount(slot, weights=val.real, minlength=jj.size)
                           + 1j * np.bincount(slot, weights=val.imag, minlength=jj.size))
            jj_all.append(np.asarray(jj, dtype=np.int64))
            uv_all.append(uvk)
            amap.append(a + 1)
            lmap.append(l)
            mmap.append(m)
    nzlma = len(jj_all)
    maxmjj = max(len(j) for j in jj_all)
    mjj = np.array([len(j) for j in jj_all], dtype=np.int32)
    jjp = np.zeros((nzlma, maxmjj), dtype=np.int32)
    uvk = np.zeros((nk, nzlma, maxmjj), dtype=np.complex128)
    for p in range(nzlma):
        jjp[p, :mjj[p]] = jj_all[p] + 1          # 1-based like the reference
        uvk[:, p, :mjj[p]] = uv_all[p]
    return atoms, nzlma, mjj, jjp, uvk, np.array(amap, np.int32), np.array(lmap, np.int32), \
        np.array(mmap, np.int32)


def _dij_pairs(cfg: Config, rng, amap, lmap, mmap):
    """Per-atom symmetric coupling blocks in nzqr_pair/Dij00 form (src/ps_nloc_mr_module.f90:852-897)."""
    pairs, vals = [], []
    nz = amap.shape[0]
    for a in np.unique(amap):
        idx = np.nonzero(amap == a)[0]
        pa = idx.size
        blk = rng.normal(0.0, cfg.dij_sigma, size=(pa, pa))
        blk = np.triu(blk) + np.triu(blk, 1).T
        for i1, p1 in enumerate(idx):
            for i2, p2 in enumerate(idx):
                if cfg.reference_form and not (lmap[p1] == lmap[p2] and mmap[p1] == mmap[p2]):
                    continue
                pairs.append((p1 + 1, p2 + 1))
                vals.append(blk[i1, i2])
    return np.array(pairs, dtype=np.int32).reshape(-1, 2), np.array(vals, dtype=np.float64)


_PROBLEM_CACHE: dict = {}


def make_problem(cfg: Config | str, cache: bool = True) -> Problem:
    """Build the seeded synthetic operator for ``cfg`` (V_loc, projectors, Dij, k-points)."""
    if isinstance(cfg, str):
        cfg = get_config(cfg)
    key = dataclasses.astuple(cfg)
    if cache and key in _PROBLEM_CACHE:
        return _PROBLEM_CACHE[key]
    rng = np.random.default_rng(cfg.seed + 1000003 * cfg.n)
    vloc = _gaussian_vloc(cfg, rng)
    if cfg.kpoints is not None:
        kbb = np.array(cfg.kpoints, dtype=np.float64).reshape(-1, 3)
    elif cfg.mp > 0:
        kbb = monkhorst_pack(cfg.mp)
    else:
        kbb = np.zeros((1, 3))
    kcart = kbb * (2.0 * math.pi / cfg.L)
    _, nzlma, mjj, jjp, uvk, amap, lmap, mmap = _projectors(cfg, rng, kbb)
    pairs, dij = _dij_pairs(cfg, rng, amap, lmap, mmap)
    if cfg.is_complex:
        uv = uvk
        if cfg.nband_range is not None:
            lo, hi = cfg.nband_range
            nband_k = rng.integers(lo, hi + 1, size=kbb.shape[0]).astype(np.int32)
            nband_k[int(np.argmax(nband_k))] = hi
        else:
            nband_k = np.full(kbb.shape[0], cfg.nband, np.int32)
    else:
        uv = np.ascontiguousarray(uvk.real)
        nband_k = np.array([cfg.nband], np.int32)
    kin = kinetic_coefficients(cfg.h, cfg.md, kcart)
    prob = Problem(cfg=cfg, n=(cfg.n, cfg.n, cfg.n), h=cfg.h, dV=cfg.h ** 3, md=cfg.md,
                   kin=kin, vloc=vloc, nzlma=nzlma, mjj=mjj, jjp=jjp, uvk=uv, amap=amap,
                   lmap=lmap, mmap=mmap, pairs=pairs, dij=dij, kbb=kbb, kcart=kcart,
                   nband_k=nband_k)
    if cache:
        _PROBLEM_CACHE[key] = prob
    return prob


# ----------------------------------------------------------------------------
# initial wavefunctions (counter-based, bit-reproducible on CPU and GPU)
# ----------------------------------------------------------------------------
_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def random_wavefunctions(seed: int, nband: int, ng: int, is_complex: bool = False,
                         kindex: int = 0, band0: int = 0) -> np.ndarray:
    """Seeded N(0,1)-like wavefunctions in [band][grid] layout.

    Element ``e`` (``e = ((kindex*2^20 + band)*ng + grid)*2 + reim``) is
    ``sum_{t<12} u(e,t) - 6`` with ``u = (splitmix64(seed*2^40 + 12e + t) >> 11) * 2^-53``
    summed in order ``t = 0..11`` -- exact double arithmetic, so the library's
    device generator (``rsdft_gpu_random_wf``) reproduces the same bits.
    """
    ncomp = 2 if is_complex else 1
    bands = np.arange(band0, band0 + nband, dtype=np.uint64)
    grid = np.arange(ng, dtype=np.uint64)
    comp = np.arange(ncomp, dtype=np.uint64)
    with np.errstate(over="ignore"):
        e = (((np.uint64(kindex) * np.uint64(1 << 20) + bands[:, None, None]) * np.uint64(ng)
              + grid[None, :, None]) * np.uint64(2) + comp[None, None, :])
        base = np.uint64(seed) * np.uint64(1 << 40) + e * np.uint64(12)
        acc = np.zeros(e.shape, dtype=np.float64)
        for t in range(12):
            u = (_splitmix64(base + np.uint64(t)) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)
            acc = acc + u
    acc = acc - 6.0
    if is_complex:
        return (acc[..., 0] + 1j * acc[..., 1]).astype(np.complex128)
    return acc[..., 0].copy()
