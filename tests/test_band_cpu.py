"""Host side of the band-structure driver against the reference's Si band run.

* k_trajectory on the sample's BAND input (vertices Gamma, X = (0, 1/2, 1/2), L = (1/2, 1/2, 1/2),
  Gamma with 20, 5 and 20 steps) reproduces the 46-point trajectory the reference printed:
  reduced k and the Cartesian step bb dak of every point (src/band_module.f90:124-146).
* write_band_eigv writes a file that the reference's plotting tool reads as its own: the steps
  of utility/band2gp.f90:17-100 (format tag, Fermi energy, reciprocal vectors, per-point blocks)
  applied to the written text recover the trajectory, MBV and the band energies of the
  reference's band_eigv.
"""
import json
import os

import numpy as np

from rsdft_develop_b200 import band, pseudo, structure

HERE = os.path.dirname(__file__)
AK = [[0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.5, 0.5], [0.0, 0.0, 0.0]]
NFKI = [20, 5, 20]


def _si_bb():
    pp = pseudo.load_npz(os.path.join(HERE, "golden", "si_pbe_tm_psv.npz"))
    st = structure.si_crystal(pp)
    return pseudo.reciprocal(st.avec).T          # columns b_i, the reference's bb(:, i)


def _golden(key):
    return json.load(open(os.path.join(HERE, "golden", "reference_logs.json")))[key]


def test_trajectory_matches_the_printed_si_trajectory():
    t = band.k_trajectory(AK, NFKI, _si_bb())
    for log in _golden("si"):
        ref = np.array(log["ktrj"])
        assert t.shape == ref.shape == (46, 6)
        assert np.max(np.abs(t - ref)) < 6e-11, np.max(np.abs(t - ref))


def _read_like_band2gp(path):
    """utility/band2gp.f90:17-100 with Fortran list-directed reads: returns (versioned,
    noncollinear, efermi, bb (columns), [(k index, mb2, kbb, mbv)], eval (nbk, mb))."""
    lines = [ln.split() for ln in open(path).read().splitlines()]
    i = 0
    versioned = lines[0][0].startswith("version")
    noncol = False
    efermi = None
    if versioned:
        if lines[0][0] == "version2.1":
            noncol = lines[0][1] in ("T", ".TRUE.")
        efermi = float(lines[1][1]) if len(lines[1]) > 1 else float(lines[1][0].split(":")[1])
        i = 3
    bb = np.array([[float(x) for x in lines[i + j]] for j in range(3)]).T
    i += 3
    heads, evals = [], []
    while i < len(lines) and lines[i]:
        k, mb, kx, ky, kz, mbv = lines[i]
        heads.append((int(k), int(mb), [float(kx), float(ky), float(kz)], int(mbv)))
        evals.append([float(lines[i + 1 + n][1]) for n in range(int(mb))])
        i += 1 + int(mb)
    return versioned, noncol, efermi, bb, heads, np.array(evals)


def test_band_eigv_reads_back_like_the_reference_file(tmp_path):
    bb = _si_bb()
    t = band.k_trajectory(AK, NFKI, bb)
    for ref in _golden("si_band"):
        esp = np.array(ref["esp"])
        r = band.BandResult(ktrj=t, esp=esp, desp=np.zeros_like(esp), sweeps=np.ones(46, np.int64),
                            res=np.zeros_like(esp))
        path = str(tmp_path / "band_eigv")
        band.write_band_eigv(path, r, efermi=0.234669645097743, mbv=4, bb=bb)
        versioned, noncol, ef, bb2, heads, ev = _read_like_band2gp(path)
        assert versioned and not noncol and abs(ef - 0.234669645097743) < 1e-15
        assert np.allclose(bb2, bb, atol=1e-15)
        assert [h[0] for h in heads] == list(range(1, 47)) and all(h[1] == 12 and h[3] == 4 for h in heads)
        assert np.allclose([h[2] for h in heads], ref["kpoints"], atol=1e-12)
        assert np.max(np.abs(ev - esp)) < 1e-12
    # the written header lines carry the reference's labels
    text = open(path).read().splitlines()
    assert text[0].split() == ["version2.1", "F"]
    assert text[1].startswith(" Fermi_energy(hartree):") and text[2] == " Reciprocal_Lattice_Vectors:"
