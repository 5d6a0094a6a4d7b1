"""k-points split over ranks in the crystal SCF (gloo, world size 2, CPU): the reference's
comm_bzsm layout (contiguous blocks, the first nk mod np ranks one larger), the eigenvalues
gathered for the occupations, the density and band-energy sums added over the ranks.  Both ranks
must return the single-process result (the Si sample's operator on the 2 x 2 x 2 mesh, oracle
band update, stop at 1e-14): the same iteration count, the total energy to 1e-11 Ha, the
eigenvalues to 1e-10 Ha and the last output density to 1e-8 (the two runs differ only in the
order of the density's sum over k, ~1e-16 per iteration, which the SCF's last steps, moving the
density by ~1e-7 rms, carry to the 1e-10 level)."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from rsdft_develop_b200 import kparallel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_k_blocks_follow_the_reference_layout():
    # the Si sample's 63 k-points over 8 k groups: 8 x 7 + 7 (its log prints id_bzsm 0, 8, ..., 56)
    assert kparallel.k_blocks(63, 8) == [(0, 8), (8, 8), (16, 8), (24, 8), (32, 8), (40, 8), (48, 8), (56, 7)]
    assert kparallel.k_blocks(5, 2) == [(0, 3), (3, 2)]
    assert sum(c for _, c in kparallel.k_blocks(10, 3)) == 10


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(kgroup_ws, rank, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from rsdft_develop_b200 import kparallel, pseudo, scf_structure, structure, synth
    from tests.test_si_cpu import OracleBandsK
    from oracle import oracle as orc
    orc.set_threads(2)
    if kgroup_ws > 1:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        dist.init_process_group("gloo", rank=rank, world_size=kgroup_ws)
    pp = pseudo.load_npz(os.path.join(ROOT, "tests", "golden", "si_pbe_tm_psv.npz"))
    kbb, w = synth.generate_bz((2, 2, 2))
    su = structure.setup(structure.si_crystal(pp, kbb, w, nband=8))
    kg = kparallel.KpointGroup(su.problem.nk) if kgroup_ws > 1 else None
    bands = OracleBandsK(su, orc, klist=None if kg is None else kg.klist)
    res = scf_structure.run_scf_kpoints(su, bands, nsweep=8, diter=30, scf_conv=1e-14, kgroup=kg)
    if kgroup_ws > 1:
        dist.destroy_process_group()
    out.put((rank, res.iterations, res.energies["total"], res.esp, res.rho))


def test_two_ranks_reproduce_one():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p1 = ctx.Process(target=_run, args=(1, 0, 0, q))
    p1.start()
    one = q.get(timeout=600)
    p1.join(timeout=60)
    assert p1.exitcode == 0
    port = _free_port()
    procs = [ctx.Process(target=_run, args=(2, r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    two = sorted((q.get(timeout=600) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, it, total, esp, rho in two:
        assert it == one[1]
        assert abs(total - one[2]) < 1e-11, (rank, total - one[2])
        assert np.max(np.abs(esp - one[3])) < 1e-10, np.max(np.abs(esp - one[3]))
        assert np.max(np.abs(rho - one[4])) < 1e-8, np.max(np.abs(rho - one[4]))
