"""Save the pseudopotentials of the reference's O2 and Si samples as compact fixtures.

Run here (where the reference tree exists): ``python tests/golden/extract_psv.py``.  It reads
samples_for_supercomputers/FLOW-FX_NAGOYA-U/02_O2-molecule_optimize/real8/O_PBE_RC1.5.psv and
samples_for_supercomputers/pseudopotential/Si-PBE-TM.psv with this library's PSV reader
(rsdft_develop_b200.pseudo.read_psv) and writes the parsed tables (radial mesh, local potential,
projectors, initial-charge Gaussians) to o_pbe_rc15_psv.npz and si_pbe_tm_psv.npz beside this
script, so that the tests that build the O2 and Si operators run where the reference tree is
absent.  test_pseudo_cpu.py checks the fixtures against a fresh read when the files are present.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from rsdft_develop_b200 import pseudo  # noqa: E402

PSV = ("/root/reference/samples_for_supercomputers/FLOW-FX_NAGOYA-U/02_O2-molecule_optimize/real8/"
       "O_PBE_RC1.5.psv")
PSV_SI = "/root/reference/samples_for_supercomputers/pseudopotential/Si-PBE-TM.psv"


def main():
    for src, name in ((PSV, "o_pbe_rc15_psv.npz"), (PSV_SI, "si_pbe_tm_psv.npz")):
        pp = pseudo.read_psv(src)
        out = os.path.join(HERE, name)
        pseudo.save_npz(pp, out)
        print(f"{out}: {os.path.getsize(out)} bytes")


if __name__ == "__main__":
    main()
