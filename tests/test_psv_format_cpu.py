"""read_PSV's record layout on small synthetic files (src/ps_read_psv.f90:13-378).

The three header versions (#PSV 2.x, #xPSV, and the old unmarked one that assumes LDA PZ81 and
skips one comment record), local-potential tables with two columns (no core charge) and three,
the fixed-width (3e20.12) D_ij records, the multi-reference case (projectors not scaled by
sqrt|D_ii|) and the consistency checks the reference stops on (a1 + a3 != 1, a non-logarithmic
mesh).  The tables are made up; only the layout is the reference's.
"""
import math

import numpy as np
import pytest

from rsdft_develop_b200 import pseudo

NDLC = 21
NSMPL = 15


def _mesh():
    r1, rend = 1.0e-4, 20.0
    h = math.exp(math.log(rend / r1) / (NDLC - 1))
    return r1 * h ** np.arange(NDLC)


def _write(path, header, nr=(1, 1), three_col=False, a=(1.2, 2.0, -0.2, 1.1), ddi=None, charge=True,
           bad_mesh=False):
    rr = _mesh()
    if bad_mesh:
        rr = rr.copy()
        rr[1] *= 1.01
    lines = list(header)
    lines.append(f"    {len(nr)}")
    lines.append("    " + "    ".join(str(n) for n in nr))
    lines.append(f"      {NSMPL}    {rr[NSMPL - 1]:.15e}")
    lines.append("    ".join(f"{x:.8f}" for x in a))
    lines.append(f"{NDLC}")
    for i in range(NDLC):
        v = -6.0 / max(rr[i], 0.5)
        lines.append(f"  {rr[i]:.15e}  {v:.15e}" + (f"  {0.1 * math.exp(-rr[i]):.15e}" if three_col else ""))
    lines.append("### NON-LOCAL POTENTIAL PARAMETERS ###")
    lines.append(f"    {NSMPL}    {rr[0]:.10e}    {rr[NSMPL - 1]:.10e}    {rr[1]:.10e}")
    k = 0
    for l, m in enumerate(nr):
        lines.append(f"### L= {l} :")
        vals = []
        for j in range(m):
            for i in range(j + 1):
                vals.append(ddi[l][i][j] if ddi else (0.5 + 0.1 * l if i == j else 0.0))
        for c in range(0, len(vals), 3):
            lines.append("".join(f"{v:20.12e}" for v in vals[c:c + 3]))
        lines.append("  ".join("0.0" for _ in vals))
        for j in range(m):
            lines.append(f"** PSI, PHI, BETA, R FOR {j + 1}-TH REF.")
            for i in range(NSMPL):
                b = (k + 1) * rr[i] * math.exp(-rr[i])
                lines.append(f"  {0.1:.12e}  {0.1:.12e}  {b:.12e}  {rr[i]:.4e}")
            k += 1
    if charge:
        lines.append("#### DATA OF PSEUDO CORE ###")
        lines.append("### initial charge and spin ###")
        lines.append("    2")
        lines.append("   0.5   0.1   1.5")
        lines.append("   0.2   0.0   0.7")
    path.write_text("\n".join(lines) + "\n")


def test_psv2_header_two_column_local_table(tmp_path):
    f = tmp_path / "a.psv"
    _write(f, ["#PSV-2.3  test", "'GGAPBE96'   8.00000000 1", "# comment", "# another", "     6.0"])
    pp = pseudo.read_psv(str(f))
    assert pp.xc_pot == "GGAPBE96" and pp.zelement == 8.0 and pp.zps == 6.0
    assert pp.mr == NDLC + 1 and pp.rad[0] == 0.0 and np.allclose(pp.rad[1:], _mesh(), rtol=1e-14)
    assert pp.norb == 2 and list(pp.lo) == [0, 1] and list(pp.nrps) == [NSMPL + 1] * 2
    assert np.all(pp.cdc == 0.0) and pp.vql[0] == pp.vql[1]
    rr = _mesh()[:NSMPL]
    assert np.allclose(pp.viod[1:NSMPL + 1, 0], rr * np.exp(-rr) * math.sqrt(0.5), rtol=1e-11)
    assert np.allclose(pp.viod[1:NSMPL + 1, 1], 2 * rr * np.exp(-rr) * math.sqrt(0.6), rtol=1e-11)
    assert list(pp.inorm) == [1.0, 1.0] and np.allclose(pp.anorm, [0.5, 0.6])
    assert pp.cdd_coef.shape == (3, 2) and np.allclose(pp.cdd_coef[:, 1], [0.2, 0.0, 0.7])
    # cdd = 4 pi r^2 sum_g (a + b r^2) exp(-c r^2) on the mesh; rab = r h
    r = pp.rad[1:]
    ref = 4 * math.pi * r ** 2 * ((0.5 + 0.1 * r ** 2) * np.exp(-1.5 * r ** 2) + 0.2 * np.exp(-0.7 * r ** 2))
    assert np.allclose(pp.cdd[1:], ref, rtol=1e-12, atol=1e-300)
    assert np.allclose(pp.rab[1:], r * math.log(r[-1] / r[0]) / (NDLC - 1), rtol=1e-13)


def test_three_column_local_table_reads_the_core_charge(tmp_path):
    f = tmp_path / "b.psv"
    _write(f, ["#PSV-2.3", "'LDAPZ81'  14.0 1", "    4.0"], three_col=True)
    pp = pseudo.read_psv(str(f))
    assert pp.xc_pot == "LDAPZ81" and pp.zps == 4.0
    assert np.allclose(pp.cdc[1:], 0.1 * np.exp(-_mesh()), rtol=1e-13)


def test_old_header_assumes_lda_and_skips_one_comment(tmp_path):
    f = tmp_path / "c.psv"
    _write(f, ["an old potential", "comment record"])
    pp = pseudo.read_psv(str(f))
    assert pp.xc_pot == "LDAPZ81" and pp.zps == 0.0 and pp.zelement == 0.0 and pp.norb == 2


def test_multi_reference_set_keeps_unscaled_projectors(tmp_path):
    """Two references for l = 0 with an off-diagonal D_12: more nonzero D_ij than diagonal
    anorm, so the projectors are not scaled by sqrt|D_ii| (multref in read_PSV)."""
    f = tmp_path / "d.psv"
    ddi = [[[0.5, 0.2], [0.2, -0.3]]]
    _write(f, ["#PSV-2.3", "'GGAPBE96'  8.0 1", "    6.0"], nr=(2,), ddi=ddi)
    pp = pseudo.read_psv(str(f))
    assert pp.norb == 2 and list(pp.lo) == [0, 0] and list(pp.no) == [1, 2]
    assert np.allclose(pp.dij, [[0.5, 0.2], [0.2, -0.3]]) and list(pp.inorm) == [1.0, -1.0]
    rr = _mesh()[:NSMPL]
    assert np.allclose(pp.viod[1:NSMPL + 1, 1], 2 * rr * np.exp(-rr), rtol=1e-11)


def test_xtapp_header_needs_its_charge_file(tmp_path):
    f = tmp_path / "e.psv"
    _write(f, ["#xPSV test", "# comment", "'GGAPBE96'", "   6.0   8.0"], charge=False)
    with pytest.raises(NotImplementedError):
        pseudo.read_psv(str(f))


def test_inconsistent_files_are_refused(tmp_path):
    f = tmp_path / "f.psv"
    _write(f, ["#PSV-2.3", "'GGAPBE96'  8.0 1", "    6.0"], a=(1.2, 2.0, -0.1, 1.1))
    with pytest.raises(ValueError, match="a1 \\+ a3"):
        pseudo.read_psv(str(f))
    g = tmp_path / "g.psv"
    _write(g, ["#PSV-2.3", "'GGAPBE96'  8.0 1", "    6.0"], bad_mesh=True)
    with pytest.raises(ValueError, match="logarithmic"):
        pseudo.read_psv(str(g))
