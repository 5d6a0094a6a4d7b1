"""Operators of real structures: atoms + PSV pseudopotentials -> the band update's inputs.

The set-up the reference runs before its first sweep (src/rsdft.f90 initialisation order:
read_pseudopot, Init_Ggrid, init_ps_local + construct_ps_local, construct_ps_initrho,
ps_nloc_initiate -> prep_ps_nloc2, init_hartree + calc_hartree, calc_xc, init_localpot),
for orthorhombic cells and a Gamma-point band update (real8, or complex16 at Gamma):

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
    cell: tuple                        # (A1, A2, A3) diagonal factors of the orthorhombic cell
    n: tuple                           # grid points per axis
    species: list                      # [(PseudoPotential, (natom, 3) reduced positions)]
    nband: int
    nspin: int = 1
    ndspin: float = 0.0                # initial N_up - N_down
    md: int = 6
    xc: str = "GGAPBE96"

    @property
    def lengths(self) -> tuple:
        return tuple(self.ax * c for c in self.cell)

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

    def problem_for_spin(self, s: int) -> synth.Problem:
        """The band update's operator for spin s (1-based)."""
        return dataclasses.replace(self.problem, vloc=np.ascontiguousarray(self.vloc[s - 1]))


def setup(st: Structure, rcfac: float = 1.5, qcfac: float = 1.0, etafac: float = 8.0,
          complex16: bool = False) -> Setup:
    """The band update's inputs for st.  complex16: the operator for the complex16 build at the
    Gamma point (complex wavefunctions, projectors with unit phases), as the reference's
    complex16 sample runs use it."""
    n = tuple(st.n)
    L = st.lengths
    h = tuple(L[d] / n[d] for d in range(3))
    if not (abs(h[0] - h[1]) < 1e-12 * h[0] and abs(h[0] - h[2]) < 1e-12 * h[0]):
        raise NotImplementedError("the band update's stencil takes one grid spacing (cubic grid cells)")
    dV = h[0] * h[1] * h[2]
    vcell = L[0] * L[1] * L[2]
    ng = n[0] * n[1] * n[2]
    gr = pseudo.make_ggrid(n, L)
    species = [(pp, np.asarray(pos, np.float64).reshape(-1, 3)) for pp, pos in st.species]
    vion = pseudo.ionic_potential(species, gr, vcell)
    rho0 = pseudo.initial_density(species, n, L)
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
    if st.xc.upper() not in ("GGAPBE96", "PBE", "PBE96"):
        raise NotImplementedError(f"xc {st.xc}: structures from PSV files take PBE here")
    vxc, ex, ec = gga.pbe(rho, n, h, dV, st.md)
    exc = ex + ec
    vloc = vion[None, :] + vh[None, :] + vxc
    filtered = [pseudo.filter_projectors(pp, gr.gcut, rcfac, qcfac, etafac) for pp, _ in species]
    ps = pseudo.grid_projectors(species, filtered, n, L)
    natom = sum(len(pos) for _, pos in species)
    lmax = max(int(pp.lo.max()) for pp, _ in species)
    cfg = synth.Config(name="structure", n=n[0], h=h[0], nband=st.nband, n_gauss=0, natom=natom,
                       lmax=lmax, rc=float(max(f.rps.max() for f in filtered)), md=st.md,
                       kpoints=((0.0, 0.0, 0.0),) if complex16 else None)
    kbb = np.zeros((1, 3))
    kin = synth.kinetic_coefficients(h[0], st.md, kbb * 0.0)
    pairs = np.stack([np.arange(1, ps.nzlma + 1), np.arange(1, ps.nzlma + 1)], axis=1).astype(np.int32)
    prob = synth.Problem(cfg=cfg, n=n, h=h[0], dV=dV, md=st.md, kin=kin,
                         vloc=np.ascontiguousarray(vloc[0]), nzlma=ps.nzlma, mjj=ps.mjj, jjp=ps.jjp,
                         uvk=ps.uv[None, :, :].astype(np.complex128 if complex16 else np.float64),
                         amap=ps.amap, lmap=ps.lmap, mmap=ps.mmap,
                         pairs=pairs, dij=ps.iuv.astype(np.float64), kbb=kbb, kcart=kbb.copy(),
                         nband_k=np.array([st.nband], np.int32))
    return Setup(structure=st, ggrid=gr, vion=vion, rho=rho, vh=vh, vxc=vxc, vloc=vloc, e_hartree=eh,
                 e_xc=exc, nelectron_spin=nes, projectors=ps, problem=prob)


def o2_molecule(pp: pseudo.PseudoPotential, nband: int = 18) -> Structure:
    """The reference's O2 sample (samples_for_supercomputers/*/02_O2-molecule_optimize): cubic
    cell AX = 18.89726878 bohr, 48^3 grid, two O atoms at reduced z = -/+0.06, PBE, two spins
    with N_up - N_down = 2, Md = 6; Nband 16 is raised to 18 by the reference's ScaLAPACK
    block rule on its 36-process layout."""
    pos = np.array([[0.0, 0.0, -0.06], [0.0, 0.0, 0.06]])
    return Structure(ax=18.89726878, cell=(1.0, 1.0, 1.0), n=(48, 48, 48), species=[(pp, pos)],
                     nband=nband, nspin=2, ndspin=2.0, md=6, xc="GGAPBE96")
