"""Kinetic set-up pinned by numbers the reference printed itself.

The reference's O2 sample runs (cubic cell AX = 18.89726878 bohr, 48^3 grid, Md = 6) log the
init_kinetic table (src/kinetic/kinetic_module.f90:28-162): the FD weights lap(m), nab(m) and the
coefficients coef_lap(1:3, m) = lap(m) (-1/2 ggg/H^2), coef_lap0 = lap(0) sum_d (-1/2 ggg/H^2)
and coef_nab(1:3, m) = nab(m)/H.  tests/golden/reference_logs.json holds them, extracted from the
logs by tests/golden/extract_reference_logs.py; this library's set-up (synth.fd_lap_coef,
fd_nab_coef, kinetic_coefficients, which feed rsdft_gpu_init / rsdft_gpu_set_kpoint) must
reproduce every printed digit.
"""
import json
import os

import numpy as np

from rsdft_develop_b200 import synth

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_logs.json")


def test_kinetic_coefficients_match_reference_logs():
    data = json.load(open(GOLDEN))["kinetic"]
    assert len(data) >= 1
    md = 6
    lap = synth.fd_lap_coef(md)
    nab = synth.fd_nab_coef(md)
    for d in data:
        n = d["ngrid"][0]
        assert d["ngrid"] == [n, n, n] and np.allclose(d["ggg"][:3], 1.0) and np.allclose(d["ggg"][3:], 0.0)
        h = d["ax"] / n
        kin = synth.kinetic_coefficients(h, md, np.zeros((1, 3)))
        for row in d["lap_table"]:
            m = row[0]
            assert abs(lap[md + m] - row[1]) <= 5e-16 * max(1.0, abs(row[1])), (m, lap[md + m], row[1])
            if m == 0:
                assert abs(kin["coef_lap0"] - row[2]) <= 1e-14 * abs(row[2])
            else:
                for dd in range(3):
                    assert abs(kin["coef_lap"][dd, m - 1] - row[2 + dd]) <= 2e-15 * max(1.0, abs(row[2 + dd])), (m, dd)
        for row in d["nab_table"]:
            m = row[0]
            assert abs(nab[md + m] - row[1]) <= 5e-16, (m, nab[md + m], row[1])
            for dd in range(3):
                assert abs(kin["coef_nab"][dd, m - 1] - row[2 + dd]) <= 2e-15 * max(1.0, abs(row[2 + dd])), (m, dd)


def test_monkhorst_pack_points_match_reference_logs():
    """generate_bz (src/bz_module.f90:65-189, Monkhorst_Pack :530-557) without symmetry, k and -k
    merged: the Si sample's 5 x 5 x 5 mesh gives the printed 63 points, order and weights."""
    bz = json.load(open(GOLDEN))["bz"]
    assert len(bz) >= 1
    for b in bz:
        kbb, w = synth.generate_bz(b["mmm"])
        ref = np.array(b["kpoints"])
        assert kbb.shape == (ref.shape[0], 3), (kbb.shape, ref.shape)
        assert np.allclose(kbb, ref[:, :3], atol=5e-6)  # printed with 5 decimals
        assert np.allclose(w, ref[:, 3], atol=5e-6)
    kbb, w = synth.generate_bz([0, 0, 0])  # "gamma point sampling is assumed"
    assert kbb.shape == (1, 3) and np.allclose(kbb, 0.0) and np.allclose(w, 1.0)
