"""Benchmark: seconds to band residual 1e-8 on one B200 (plus hpsi HBM GB/s).

A step is one complete band-update solve of the seeded synthetic problem: device-side
seeded wavefunctions -> Gram-Schmidt -> calc_sweep (CG -> GS -> SD per sweep, FP64
residual check after each sweep) until max_n res(n) <= 1e-8, res = dV |H psi - e psi|^2
(the reference's definition, src/conjugate_gradient/cg_module.f90:231).

JSON line keys beyond the driver contract: ``roofline`` (hpsi stencil kernel, CUDA events
inside the library on its own stream over the timed region), ``cpu_baseline`` (the CPU
oracle that restates the reference's CPU path, timed on a bounded sample), ``e2e`` (same
solve through the C ABI from pinned host buffers, host<->device copies inside the timed
region), ``clocks`` (nvidia-smi samples during the timed region).

--impl reference runs the CPU restatement of the reference path (oracle/) on the host
cores for the same config and metric.  Multi-GPU runs are independent replicas (the path
is one GPU per problem): every rank solves its own copy, the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s to band residual 1e-8: mixed+learned vs plain FP64 on 1 GPU; hpsi HBM GB/s"
TOL = 1e-8
MAX_SWEEPS = 600

# DRAM traffic per stencil launch from ncu (dram__bytes_read.sum + dram__bytes_write.sum over
# the algorithmic bytes), by (config, precision); source: profiles/hpsi_stencil_c1.md
# (316.3 + 226.2 MB against 537.9 MB for all 256 bands).
NCU_TRAFFIC_RATIO: dict = {("c1", "mixed"): 1.009}

# Sweeps the plain FP64 method needs to reach max res <= 1e-8 from the seeded start
# (same algorithm on CPU and GPU; measured by the FP64 GPU path).
SWEEPS_TO_TOL = {"c0": 75, "c1": None}


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        pw = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        loaded = [s for s, p in zip(sm, pw) if p > 200.0] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows), "power_w_max": max(pw) if pw else None}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return None, 0, 1
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    import datetime
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return dist, dist.get_rank(), ws


def _max_over_ranks(dist, x: float) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(dist):
    if dist is not None:
        dist.barrier()


def cpu_sweep_time(cfg_name: str, nthreads: int, nsweep: int = 1):
    """Seconds per oracle sweep (CG+GS+SD) on the host cores, after an untimed GS."""
    from oracle import oracle as orc
    from rsdft_develop_b200 import synth
    orc.build()
    orc.set_threads(nthreads)
    prob = synth.make_problem(cfg_name)
    o = orc.Oracle(prob)
    psi = o.gram_schmidt(synth.random_wavefunctions(1, prob.nband, prob.ng))
    t0 = time.perf_counter()
    o.sweep(psi, nsweep)
    return (time.perf_counter() - t0) / nsweep


def run_reference(args, dist, rank, ws):
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    n_conv = SWEEPS_TO_TOL.get(args.config) or args.sweeps_to_tol
    samples = []
    for i in range(args.warmup + args.steps):
        t = cpu_sweep_time(args.config, nthreads)
        if i >= args.warmup:
            samples.append(t)
    per = statistics.median(samples)
    val = per * n_conv
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1000.0,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": args.config, "precision": "fp64", "sweeps_to_tol": n_conv},
        "cpu_baseline": {"value": val, "unit": "s", "cores": nthreads, "kind": "port",
                         "sample": f"1 CG+GS+SD sweep of {args.config} per step on {nthreads} host threads "
                                   f"(oracle/ restatement of the reference CPU path), x {n_conv} sweeps"},
        "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def mb_ref_of(nband: int) -> int:
    """Convergence band set: bands 1..mb_ref, mb_ref = (nband + nocc)/2 with nocc = 3/4 nband
    (the reference's DOS driver rule max_ref_band = (nb + nocc)/2, src/dos_module.f90:64-65)."""
    return nband - nband // 8


def solve(g, seed: int, tol: float):
    """One complete solve on the resident (device-generated) wavefunctions; returns sweeps."""
    g.random_wf(seed)
    g.gram_schmidt()
    it, esp, res = g.calc_sweep(MAX_SWEEPS, tol=tol)
    return it, esp, res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c1")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--pc", default="hprsdft", choices=["auto", "learned", "hprsdft", "none"],
                    help="CG preconditioner; auto = learned when trained weights for the grid spacing exist")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the comparison solves (plain FP64, and mixed with precond_hprsdft)")
    ap.add_argument("--sweeps-to-tol", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer (C ABI) solves (large configs)")
    ap.add_argument("--gemm-terms", default="3,3",
                    help="BF16 terms of the mixed overlap/Hsub and rotation contractions (2 or 3 each)")
    args = ap.parse_args()
    dist, rank, ws = _dist()
    if args.impl == "reference":
        run_reference(args, dist, rank, ws)
        if dist is not None:
            dist.destroy_process_group()
        return

    import torch
    from rsdft_develop_b200 import api, synth
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    from rsdft_develop_b200 import lpc_train
    prob = synth.make_problem(args.config)
    prec = api.PREC_MIXED if args.precision == "mixed" else api.PREC_FP64
    wpath = lpc_train.default_weights_path(prob.h)
    pc = args.pc
    if pc == "auto":
        pc = "learned" if (prec == api.PREC_MIXED and os.path.exists(wpath)) else "hprsdft"
    pc_mode = {"learned": api.PC_LEARNED, "hprsdft": api.PC_HPRSDFT, "none": api.PC_NONE}[pc]
    g = api.BandUpdate(prob, precision=prec, pc_mode=pc_mode)
    terms = tuple(int(t) for t in args.gemm_terms.split(","))
    g.gemm_terms(*terms)
    if pc == "learned":
        g.lpc_set_weights(np.load(wpath))
    mb_ref = mb_ref_of(prob.nband)
    g.init_sweep(mb_ref)
    stream = torch.cuda.ExternalStream(g.stream())

    for _ in range(args.warmup):
        solve(g, 1, TOL)
    g.synchronize()
    _barrier(dist)
    torch.cuda.synchronize()
    launches0 = g.kernel_launches()
    g.profile(True)
    iters = []
    with ClockSampler(local) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            it, esp, res = solve(g, 1, TOL)
            iters.append(it)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    dt_ms = ev0.elapsed_time(ev1)
    launches = g.kernel_launches() - launches0
    st_ms, st_n, st_bytes, _ = g.profile_get("hpsi_stencil")
    names = ["hpsi_stencil", "nl_gather", "nl_scatter", "cg", "pc", "lpc", "gs", "gemm", "sd_gemm", "sd_eig",
             "sd_rot", "residual"]
    shares = {n: g.profile_get(n)[0] for n in names}
    g.profile(False)
    lpc_state = g.lpc_status()
    clocks = clk.summary()
    res_max = float(np.max(res[..., :mb_ref]))
    per_step = dt_ms / args.steps
    t_solve = _max_over_ranks(dist, per_step / 1000.0)

    e2e_t, h2d, d2h = [], 0, 0
    if not args.no_e2e:
        # e2e: the same solve through the C ABI from pinned host buffers
        psi0 = synth.random_wavefunctions(1, prob.nband, prob.ng)
        pin = torch.from_numpy(psi0).pin_memory()
        pin_np = pin.numpy()
        out = torch.empty_like(pin).pin_memory().numpy()
        e2e_t = []
        for i in range(1 + args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            g.set_wf(pin_np)
            g.gram_schmidt()
            it, esp, res = g.calc_sweep(MAX_SWEEPS, tol=TOL)
            g.lib.rsdft_gpu_get_wf_d(1, 1, out.ctypes.data, prob.ng, prob.nband)
            torch.cuda.synchronize()
            if i > 0:
                e2e_t.append(time.perf_counter() - t0)
        h2d = int(psi0.nbytes)
        d2h = int(out.nbytes + esp.nbytes + res.nbytes)
    e2e_val = _max_over_ranks(dist, statistics.median(e2e_t)) if e2e_t else None

    g.close()
    # comparison solves on the same GPU: the plain FP64 method (the drop-in's FP64 path with
    # precond_hprsdft) and, when the main arm is learned, mixed precision with precond_hprsdft
    compare = {}
    if not args.no_compare:
        arms = [("fp64_hprsdft", api.PREC_FP64, api.PC_HPRSDFT)]
        if pc != "hprsdft" and prec == api.PREC_MIXED:
            arms.append(("mixed_hprsdft", api.PREC_MIXED, api.PC_HPRSDFT))
        if pc != "learned" and os.path.exists(wpath):
            arms.append(("mixed_learned", api.PREC_MIXED, api.PC_LEARNED))
        for name, pr, pm in arms:
            if pr == prec and pm == pc_mode:
                continue
            with api.BandUpdate(prob, precision=pr, pc_mode=pm) as h:
                if pm == api.PC_LEARNED:
                    h.lpc_set_weights(np.load(wpath))
                h.init_sweep(mb_ref)
                hs = torch.cuda.ExternalStream(h.stream())
                solve(h, 1, TOL)
                h.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(hs)
                itc, _, _ = solve(h, 1, TOL)
                e1.record(hs)
                e1.synchronize()
                tc = _max_over_ranks(dist, e0.elapsed_time(e1) / 1000.0)
            compare[name] = {"s": round(tc, 4), "sweeps": itc}
        if "fp64_hprsdft" in compare:
            compare["speedup_vs_fp64_hprsdft"] = round(compare["fp64_hprsdft"]["s"] / t_solve, 3)

    hbm, bf16, peak_kind = _peaks()
    achieved = (st_bytes / st_n) / ((st_ms / st_n) * 1e-3) / 1e9 if st_n else 0.0
    ratio = NCU_TRAFFIC_RATIO.get((args.config, args.precision))
    kname = "k_stencil_stream<float>" if prec == api.PREC_MIXED else "k_stencil_stream<double>"
    roof = {"bound": "hbm", "kernel": f"{kname} (hpsi: 37-point stencil + V_loc; the nonlocal scatter is a separate kernel)",
            "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
            "frac": round(achieved / hbm, 4), "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
            "traffic": (ratio * st_bytes / st_n) if ratio else None,
            "launches": st_n, "avg_launch_ms": (st_ms / st_n) if st_n else None,
            "algorithmic_bytes_per_launch": (st_bytes / st_n) if st_n else None}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        nthreads = os.cpu_count() or 1
        per = cpu_sweep_time(args.config, nthreads)
        n_conv = int(statistics.median(iters))
        cpu = {"value": per * n_conv, "unit": "s", "cores": nthreads, "kind": "port",
               "sample": f"1 oracle CG+GS+SD sweep of {args.config} on {nthreads} host threads "
                         f"({per:.2f} s), x {n_conv} sweeps the plain method needs to reach 1e-8"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": t_solve, "unit": "s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per_step, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32+bf16x%d/x%d+f64" % terms,
            "data": "synthetic (seeded Gaussian V_loc, Gaussian s/p projectors, seeded psi0)",
            "config": {"workload": args.config, "grid": list(prob.n), "bands": prob.nband,
                       "atoms": prob.cfg.natom, "projectors": prob.nzlma, "precision": args.precision,
                       "pc": pc, "lpc_fallbacks": lpc_state[2] if pc == "learned" else None,
                       "lpc_weights": os.path.relpath(wpath, ROOT) if pc == "learned" else None,
                       "gemm_terms": list(terms) if prec == api.PREC_MIXED else None,
                       "mb_ref": mb_ref, "sweeps_to_tol": iters, "final_res_max": res_max,
                       "l2": "inputs larger than L2 (psi >= 0.5 GB)", "parallelism": f"replicas x{ws}"},
            "gpu_launches": int(launches),
            "roofline": roof,
            "time_shares_ms": {k: round(v, 3) for k, v in shares.items()},
            "compare": compare,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
