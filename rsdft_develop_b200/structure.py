"""Operators of real structures: atoms + PSV pseudopotentials -> the band update's inputs.

The set-up the reference runs before its first sweep (src/rsdft.f90 initialisation order:
read_pseudopot, Init_Ggrid, init_ps_local + construct_ps_local, construct_ps_initrho,
ps_nloc_initiate -> prep_ps_nloc2, init_hartree + calc_hartree, calc_xc, init_localpot),
for orthorhombic or general (e.g. FCC) cells, at the Gamma point (real8, or complex16) or on a
set of k-points (complex16, projectors with the k phases of prep_uvk_ps_nloc2):

  V_loc(s) = V_ion + V_H[rho] + V_xc[rho_up, rho_down](s)     (src/localpot_module.f90:209-215)

with rho the analytic Gaussian initial density split over spins (Nelectron_spin =
(Nelectron +- Ndspin) / 2), V_H by the cut-off-sphere FFT solve and V_xc by PBE;
the nonlocal part is the filtered KB projector set with D = sign(D_ii) on the diagonal.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import gga, pseudo, synth


@dataclasses.dataclass
class Structure:
    ax: float                          # lattice constant (bohr)
    cell: tuple                        # (A1, A2, A3) diagonal factors of an orthorhombic cell, or
                                       # three lattice vectors (rows) in units of ax
    n: tuple                           # grid points per axis
    species: list                      # [(PseudoPotential, (natom, 3) reduced positions)]
    nband: int
    nspin: int = 1
    ndspin: float = 0.0                # initial N_up - N_down
    md: int = 6
    xc: str = "GGAPBE96"
    kbb: np.ndarray | None = None      # (nk, 3) reduced k-points (complex16 band update); None: Gamma
    wbz: np.ndarray | None = None      # (nk,) k weights summing to 1

    @property
    def orthorhombic(self) -> bool:
        return np.asarray(self.cell).ndim == 1

    @property
    def avec(self) -> np.ndarray:
        """Lattice vectors a_i as rows (bohr), the reference's aa(:, i)."""
        c = np.asarray(self.cell, np.float64)
        return self.ax * (np.diag(c) if c.ndim == 1 else c)

    @property
    def lengths(self) -> tuple:
        if self.orthorhombic:
            return tuple(self.ax * c for c in self.cell)
        return tuple(float(x) for x in np.sqrt(np.sum(self.avec ** 2, axis=1)))

    @property
    def volume(self) -> float:
        if self.orthorhombic:
            L = self.lengths
            return L[0] * L[1] * L[2]
        A = self.avec
        return abs(float(np.dot(A[0], np.cross(A[1], A[2]))))

    @property
    def nelectron(self) -> float:
        return float(sum(pp.zps * len(pos) for pp, pos in self.species))


@dataclasses.dataclass
class Setup:
    structure: Structure
    ggrid: pseudo.GGrid
    vion: np.ndarray                   # (ng,)
    rho: np.ndarray                    # (nspin, ng)
    vh: np.ndarray
    vxc: np.ndarray                    # (nspin, ng)
    vloc: np.ndarray                   # (nspin, ng)
    e_hartree: float
    e_xc: float
    nelectron_spin: np.ndarray
    projectors: pseudo.ProjectorSet
    problem: synth.Problem             # operator of spin 1 (see problem_for_spin)
    bmat: np.ndarray | None = None     # gga.grid_metric of a non-orthogonal cell (PBE gradient)

    def problem_for_spin(self, s: int) -> synth.Problem:
        """The band update's operator for spin s (1-based)."""
        return dataclasses.replace(self.problem, vloc=np.ascontiguousarray(self.vloc[s - 1]))


def is_pbe(xc: str) -> bool:
    return xc.upper() in ("GGAPBE96", "PBE", "PBE96")


def host_xc(xc: str, rho: np.ndarray, n: tuple, h: tuple, dV: float, md: int, bmat=None):
    """V_xc and (E_x, E_c) of rho for the structure's XCtype: GGAPBE96 (calc_GGAPBE96_2) or
    LDAPZ81 (calc_LDAPZ81, the reference's default)."""
    if is_pbe(xc):
        return gga.pbe(rho, n, h, dV, md, bmat=bmat)
    if xc.upper() in ("LDAPZ81", "LDA", "PZ81"):
        return gga.lda_pz81(rho, dV)
    raise NotImplementedError(f"xc {xc}: GGAPBE96 or LDAPZ81")


def setup(st: Structure, rcfac: float = 1.5, qcfac: float = 1.0, etafac: float = 8.0,
          complex16: bool = False) -> Setup:
    """The band update's inputs for st.  complex16: the operator for the complex16 build at the
    Gamma point (complex wavefunctions, projectors with unit phases), as the reference's
    complex16 sample runs use it."""
    n = tuple(st.n)
    L = st.lengths
    h = tuple(L[d] / n[d] for d in range(3))
    if not (abs(h[0] - h[1]) < 1e-12 * h[0] and abs(h[0] - h[2]) < 1e-12 * h[0]):
        raise NotImplementedError("the band update's stencil takes one grid spacing (equal H on the three axes)")
    ortho = st.orthorhombic
    cell = L if ortho else st.avec
    ng = n[0] * n[1] * n[2]
    vcell = st.volume
    dV = h[0] * h[1] * h[2] if ortho else vcell / ng
    gr = pseudo.make_ggrid(n, cell)
    species = [(pp, np.asarray(pos, np.float64).reshape(-1, 3)) for pp, pos in st.species]
    vion = pseudo.ionic_potential(species, gr, vcell)
    rho0 = pseudo.initial_density(species, n, cell)
    bmat = None if ortho else gga.grid_metric(st.avec, n)
    kpts = st.kbb is not None
    if kpts and not complex16:
        complex16 = True                      # k-points need complex bands
    ns = st.nspin
    nel = st.nelectron
    if ns == 1:
        nes = np.array([nel])
    else:
        nes = np.array([0.5 * (nel + st.ndspin), 0.5 * (nel - st.ndspin)])
    rho = np.zeros((ns, ng))
    for s in range(ns):
        r = rho0 / ns
        rho[s] = r * (nes[s] / (float(r.sum()) * dV))
    vh, eh = gga.hartree_sphere(rho.sum(axis=0), gr, dV)
    vxc, ex, ec = host_xc(st.xc, rho, n, h, dV, st.md, bmat)
    exc = ex + ec
    vloc = vion[None, :] + vh[None, :] + vxc
    filtered = [pseudo.filter_projectors(pp, gr.gcut, rcfac, qcfac, etafac) for pp, _ in species]
    kbb = np.asarray(st.kbb, np.float64).reshape(-1, 3) if kpts else np.zeros((1, 3))
    ps = pseudo.grid_projectors(species, filtered, n, cell, kbb if kpts else None)
    natom = sum(len(pos) for _, pos in species)
    lmax = max(int(pp.lo.max()) for pp, _ in species)
    cfg = synth.Config(name="structure", n=n[0], h=h[0], nband=st.nband, n_gauss=0, natom=natom,
                       lmax=lmax, rc=float(max(f.rps.max() for f in filtered)), md=st.md,
                       kpoints=tuple(tuple(k) for k in kbb) if complex16 else None)
    if ortho and not kpts:
        kin = synth.kinetic_coefficients(h[0], st.md, kbb * 0.0)
        kcart = kbb.copy()
    else:
        kin = synth.kinetic_coefficients_lattice(st.avec, n, st.md, kbb)
        kcart = kin["kcart"]
    if kpts:
        uvk = ps.uvk
    else:
        uvk = ps.uv[None, :, :].astype(np.complex128 if complex16 else np.float64)
    pairs = np.stack([np.arange(1, ps.nzlma + 1), np.arange(1, ps.nzlma + 1)], axis=1).astype(np.int32)
    prob = synth.Problem(cfg=cfg, n=n, h=h[0], dV=dV, md=st.md, kin=kin,
                         vloc=np.ascontiguousarray(vloc[0]), nzlma=ps.nzlma, mjj=ps.mjj, jjp=ps.jjp,
                         uvk=uvk, amap=ps.amap, lmap=ps.lmap, mmap=ps.mmap,
                         pairs=pairs, dij=ps.iuv.astype(np.float64), kbb=kbb, kcart=kcart,
                         nband_k=np.full(kbb.shape[0], st.nband, np.int32))
    return Setup(structure=st, ggrid=gr, vion=vion, rho=rho, vh=vh, vxc=vxc, vloc=vloc, e_hartree=eh,
                 e_xc=exc, nelectron_spin=nes, projectors=ps, problem=prob, bmat=bmat)


def o2_molecule(pp: pseudo.PseudoPotential, nband: int = 18) -> Structure:
    """The reference's O2 sample (samples_for_supercomputers/*/02_O2-molecule_optimize): cubic
    cell AX = 18.89726878 bohr, 48^3 grid, two O atoms at reduced z = -/+0.06, PBE, two spins
    with N_up - N_down = 2, Md = 6; Nband 16 is raised to 18 by the reference's ScaLAPACK
    block rule on its 36-process layout."""
    pos = np.array([[0.0, 0.0, -0.06], [0.0, 0.0, 0.06]])
    return Structure(ax=18.89726878, cell=(1.0, 1.0, 1.0), n=(48, 48, 48), species=[(pp, pos)],
                     nband=nband, nspin=2, ndspin=2.0, md=6, xc="GGAPBE96")


def si_crystal(pp: pseudo.PseudoPotential, kbb: np.ndarray | None = None, wbz: np.ndarray | None = None,
               nband: int = 16) -> Structure:
    """The reference's Si sample (samples_for_supercomputers/*/01_Si_band): FCC cell, AX = 10.261
    bohr, lattice vectors (0, 1/2, 1/2), (1/2, 0, 1/2), (1/2, 1/2, 0), 12^3 grid, two Si atoms at
    reduced (0, 0, 0) and (1/4, 1/4, 1/4), PBE, one spin, 16 bands, Md = 6; kbb/wbz the k-point
    set (the 5 x 5 x 5 Monkhorst-Pack mesh of generate_bz: 63 points)."""
    cell = ((0.0, 0.5, 0.5), (0.5, 0.0, 0.5), (0.5, 0.5, 0.0))
    pos = np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.25]])
    return Structure(ax=10.261, cell=cell, n=(12, 12, 12), species=[(pp, pos)], nband=nband, nspin=1,
                     ndspin=0.0, md=6, xc="GGAPBE96", kbb=kbb, wbz=wbz)
