"""Time the many-band hamiltonian (hpsi) on one configuration, FP64 and FP32.

    python -m rsdft_develop_b200.profile_hpsi c1 [reps] [max_bands] [--no-nonlocal] [--fused]

Wavefunctions are generated on the device (uniform(-1, 1), larger than L2 for the named
configurations); each precision runs one untimed call (module load, stencil autotuning),
then `reps` timed calls whose per-launch CUDA-event times and algorithmic bytes (read psi +
write H psi per band, V_loc and projector records once) come from the library's own
profiling.  The nonlocal term is added by the scatter kernel after the stencil, or inside the
stencil with --fused.  This is the driver the ncu captures under profiles/ run.
"""
from __future__ import annotations

import sys

import torch

from . import api, synth


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    nl_on = "--no-nonlocal" not in argv
    fused = "--fused" in argv
    argv = [a for a in argv if a not in ("--no-nonlocal", "--fused")]
    cfg = argv[0] if argv else "c1"
    reps = int(argv[1]) if len(argv) > 1 else 3
    nbmax = int(argv[2]) if len(argv) > 2 else 0
    prob = synth.make_problem(cfg)
    nb = prob.nband if nbmax == 0 else min(nbmax, prob.nband)
    with api.BandUpdate(prob, nonlocal_on=nl_on) as g:
        g.nl_form(fused)
        x = torch.empty((nb, prob.ng), dtype=torch.float64, device="cuda")
        x.uniform_(-1.0, 1.0)
        for name, f32 in (("fp64", False), ("fp32", True)):
            a = x.float() if f32 else x
            b = torch.empty_like(a)
            g.hamiltonian_device(a.data_ptr(), b.data_ptr(), nb, fp32=f32)
            g.synchronize()
            pre = "stencil" if f32 else "stencil64"
            tune = "  (autotune: rows/thread 1 %.3f ms, 2 %.3f ms" % (
                g.profile_get(pre + "_tune_r1")[0], g.profile_get(pre + "_tune_r2")[0])
            for r in ("r1", "r2"):
                tune += "; %s stages %d record slots %d smem %.0f KB" % (
                    r, g.profile_get(f"{pre}_{r}_stages")[0], g.profile_get(f"{pre}_{r}_rec_slots")[0],
                    g.profile_get(f"{pre}_{r}_smem_kb")[0])
            tune += ")"
            g.profile(True)
            for _ in range(reps):
                g.hamiltonian_device(a.data_ptr(), b.data_ptr(), nb, fp32=f32)
            g.synchronize()
            ms, n, by, _ = g.profile_get("hpsi_stencil")
            gms, gn, gby, _ = g.profile_get("nl_gather")
            sms, sn, sby, _ = g.profile_get("nl_scatter")
            print(f"{cfg} {name} nonlocal={int(nl_on)} bands={nb}: stencil {n} launches avg {ms / max(n, 1):.3f} ms "
                  f"{by / max(ms, 1e-9) / 1e6:.1f} GB/s algorithmic; gather avg {gms / max(gn, 1):.3f} ms; "
                  f"scatter avg {sms / max(sn, 1):.3f} ms{tune}", flush=True)
            g.profile(False)
            del a, b


if __name__ == "__main__":
    main()
