"""Regenerates tests/golden/oracle_golden.npz (run from the repository root).

The reference has no golden vectors for the band-update path, so these fixtures pin the
oracle's own FP64 outputs on seeded inputs (plus the exact t0 eigenvalues from a dense
diagonalisation) and guard against regressions of the oracle and the generator.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402
from rsdft_develop_b200 import synth  # noqa: E402
from tests import npref  # noqa: E402


def main():
    seed = 20240611
    prob = synth.make_problem("c0")
    o = orc.Oracle(prob)
    psi = synth.random_wavefunctions(seed, 4, prob.ng)
    h = o.hpsi(psi)
    pt = synth.make_problem("t0")
    H = npref.np_hpsi(pt, np.eye(pt.ng))
    eigs = np.linalg.eigvalsh(0.5 * (H + H.T))[:pt.nband]
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_golden.npz"),
                        seed=seed, psi_sample=psi[:, ::997].ravel(), hpsi_sample=h[:, ::997].ravel(),
                        hpsi_norm2=np.sum(h * h, axis=1), t0_eigs=eigs)


if __name__ == "__main__":
    main()
