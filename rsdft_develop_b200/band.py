"""Band-structure driver: eigenvalues along a k trajectory at a fixed potential.

Reference: band_module (src/band_module.f90:47-361).  The trajectory runs through the vertices
ak(1:3, 1..nbk+1) (reduced, in units of the reciprocal lattice vectors) with nfki(i) points on
segment i, ak(:, i) + (j - 1) (ak(:, i+1) - ak(:, i)) / nfki(i) for j = 1..nfki(i), followed by
the last vertex (:125-141).  At every trajectory point the kinetic coefficients (init_kinetic,
src/kinetic/kinetic_module.f90:141-162) and the projector phases (prep_uvk_ps_nloc2,
src/ps_nloc2_module.f90:1145-1158) are set for that k and calc_sweep runs with
init_sweep(2, mb2_band, esp_conv_tol) (:207, :241-265): sweeps until no eigenvalue of bands
1..mb2_band moves by esp_conv_tol, at most maxiter_band sweeps, starting from the wavefunctions
of the previous point.  The eigenvalues esp(1:mb2_band) of every point are collected and, on
request, written in the layout of the reference's band_eigv file (:201-206, :316-337).

The device side is the library's complex16 context holding one k-point whose operator is reset
through the C ABI (rsdft_gpu_set_kpoint, rsdft_gpu_set_uvk_z) at every trajectory point.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import api, synth


def k_trajectory(ak: np.ndarray, nfki, bb: np.ndarray | None = None) -> np.ndarray:
    """(nktrj, 6): reduced k of every trajectory point and, in columns 3:6, the Cartesian step
    bb @ dak of its segment (zero for the closing vertex), as band_module builds ktrj
    (src/band_module.f90:124-139).  bb: reciprocal vectors as columns (the identity when None,
    which leaves the reduced step dak)."""
    ak = np.asarray(ak, dtype=np.float64).reshape(-1, 3)
    bmat = np.eye(3) if bb is None else np.asarray(bb, dtype=np.float64)
    nbk = ak.shape[0] - 1
    nfki = [int(x) for x in nfki]
    assert len(nfki) == nbk and all(x >= 1 for x in nfki)
    rows = []
    for i in range(nbk):
        dak = (ak[i + 1] - ak[i]) / nfki[i]
        for j in range(nfki[i]):
            rows.append(np.concatenate([ak[i] + j * dak, bmat @ dak]))
    nk = len(rows)
    if nk > 0:  # nktrj > 1 in the reference always holds for a trajectory of one or more segments
        rows.append(np.concatenate([ak[nbk], np.zeros(3)]))
    return np.array(rows)


@dataclasses.dataclass
class BandResult:
    ktrj: np.ndarray      # (nktrj, 6) as k_trajectory
    esp: np.ndarray       # (nktrj, mb2) eigenvalues (Ha)
    desp: np.ndarray      # (nktrj, mb2) |esp - esp of the previous sweep| at exit
    sweeps: np.ndarray    # (nktrj,) sweeps taken per point
    res: np.ndarray       # (nktrj, mb2) FP64 residuals at exit


def trajectory_problem(cfg: synth.Config, ak, nfki) -> synth.Problem:
    """The synthetic operator of cfg (its V_loc, atoms and Dij) with one k-point per trajectory
    point of (ak, nfki)."""
    ktrj = k_trajectory(ak, nfki)
    pcfg = dataclasses.replace(cfg, mp=0, nband_range=None, kpoints=tuple(tuple(float(x) for x in k[:3]) for k in ktrj))
    return synth.make_problem(pcfg)


def band_structure(cfg: synth.Config, ak, nfki, mb2: int, esp_conv_tol: float = 1e-7, maxiter: int = 100,
                   precision: int = api.PREC_FP64, seed: int = 1, eigv_path: str | None = None,
                   vloc: np.ndarray | None = None, nonlocal_on: bool = True) -> BandResult:
    """Run the band driver for the synthetic operator of cfg (its V_loc, atoms and Dij; vloc
    replaces V_loc when given) along the trajectory (ak, nfki); cfg.nband bands are carried,
    bands 1..mb2 are converged."""
    ktrj = k_trajectory(ak, nfki, np.eye(3) * (2.0 * np.pi / cfg.L))
    nkt = ktrj.shape[0]
    prob = trajectory_problem(cfg, ak, nfki)
    if vloc is not None:
        prob = dataclasses.replace(prob, vloc=np.asarray(vloc, dtype=np.float64))
    first = dataclasses.replace(prob, kbb=prob.kbb[:1], kcart=prob.kcart[:1], uvk=prob.uvk[:1],
                                nband_k=prob.nband_k[:1],
                                kin=dict(prob.kin, coef_nabk=prob.kin["coef_nabk"][:1],
                                         const_k2=prob.kin["const_k2"][:1], zcoef_kin=prob.kin["zcoef_kin"][:1]))
    nb = int(prob.nband_k[0])
    assert 1 <= mb2 <= nb
    esp = np.zeros((nkt, mb2))
    desp = np.zeros((nkt, mb2))
    res = np.zeros((nkt, mb2))
    sweeps = np.zeros(nkt, dtype=np.int64)
    with api.BandUpdate(first, precision=precision, nonlocal_on=nonlocal_on) as g:
        g.init_sweep(mb2)
        g.sweep_check(2)
        g.random_wf(seed)
        g.gram_schmidt()
        prev = None
        for ik in range(nkt):
            g.set_kpoint_operator(prob, ik, nonlocal_on=nonlocal_on)
            it, e, r = g.calc_sweep(maxiter, tol=esp_conv_tol)
            esp[ik] = e[0, 0, :mb2]
            res[ik] = r[0, 0, :mb2]
            sweeps[ik] = it
            desp[ik] = np.abs(esp[ik] - prev) if prev is not None else np.nan
            prev = esp[ik].copy()
    out = BandResult(ktrj=ktrj, esp=esp, desp=desp, sweeps=sweeps, res=res)
    if eigv_path:
        write_band_eigv(eigv_path, out, prob)
    return out


def write_band_eigv(path: str, r: BandResult, prob: synth.Problem | None = None, efermi: float = 0.0,
                    mbv: int = 1, bb: np.ndarray | None = None):
    """The reference's band_eigv file (src/band_module.f90:191-198, :316-337), as its plotting
    tool utility/band2gp.f90 reads it: the format tag "version2.1" and the noncollinear flag, the
    Fermi energy, the reciprocal vectors (bb, columns; 2 pi / L of prob's cubic cell when None),
    then per trajectory point a line (index, mb2, reduced k, MBV) and one line per band (index,
    energy, and a second column the reference fills with |esp - esp0| of two copies of the same
    gathered eigenvalues, i.e. 0).  MBV, the number of valence bands, falls back to 1 outside
    1..mb2 as the reference's band() does."""
    if bb is None:
        bb = np.eye(3) * (2.0 * np.pi / prob.cfg.L)
    mb2 = r.esp.shape[1]
    if mbv < 1 or mbv > mb2:
        mbv = 1
    with open(path, "w") as f:
        f.write(" version2.1 F\n")
        f.write(f" Fermi_energy(hartree):{efermi:20.15f}\n")
        f.write(" Reciprocal_Lattice_Vectors:\n")
        for d in range(3):
            f.write(" " + "".join(f"{x:20.15f}" for x in bb[:, d]) + "\n")
        for ik in range(r.esp.shape[0]):
            f.write(f" {ik + 1:6d}{mb2:6d}" + "".join(f"{x:20.12f}" for x in r.ktrj[ik, :3]) + f"{mbv:8d}\n")
            for n in range(mb2):
                f.write(f" {n + 1:5d}  {r.esp[ik, n]:22.12G} {0.0:15.5G}\n")
