#!/usr/bin/env python
"""Benchmark of md_run's per-step force/integrate path on the B200 engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the solvated-polymer system (159-residue chain + 7,000 waters + ions, 22,860
atoms, 62 A cubic PBC cell, zero-dipole cut-off 12 A, SHAKE on X-H and rigid waters,
METHOD= CANO at 300 K, 2 fs), synthetic and seeded.  One step = one md_run MD step
(forces, Hoover-Evans thermostat with the SHAKE<->thermostat loop, SHAKE) with the pair
list rebuilt every UPDATE=10 steps, exactly as runmd does.

Reported (one JSON line on rank 0):
  value      aggregate ns/day of the mixed-precision path (FP32 pair arithmetic, 64-bit
             fixed-point forces, FP64 integration), device-timed with CUDA events, state
             resident in HBM, L2 flushed between timed steps
  e2e        the same metric through the C ABI with host buffers: per step copy x, v in
             from pinned host memory, one jp_step, copy x, v and the energies out
  fp64       the plain FP64 GPU path on the same workload, and the speed-up over it
  rms_force_err  RMS relative force error of the mixed path against the FP64 path
  roofline   the pair kernel (dominant) against the measured FP32 FMA peak
  cpu_baseline  the CPU oracle (OpenMP FP64 restatement of md_run) on the host cores
With N > 1 (torchrun) every rank runs its own replica of the workload (replicas only, no
data-path collective); value = all ranks' simulated time / max-over-ranks device time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "aggregate ns/day & pairs/s: mixed vs FP64 GPU path at ≤1e-5 RMS force err"
DT_FS = 2.0
FLOPS_PER_PAIR = 52          # FP32 flops per pair interaction within rc (FMA = 2)
L2_FLUSH_BYTES = 256 << 20   # > 126 MB L2
PAIR_PROFILE = os.path.join(ROOT, "profiles", "k_pair_mixed_c2.md")


def workload_name(natom):
    return (f"solvated polymer: 159-residue chain + 7,000 waters + Na+/Cl-, {natom:,} atoms, "
            "62 A cubic PBC, ZD cut-off 12 A (list 13.5 A, UPDATE 10), SHAKE X-H + rigid "
            "water, METHOD= CANO 300 K, dt 2 fs")


def ns_per_day(nsteps, seconds):
    return nsteps * DT_FS * 1e-6 * 86400.0 / seconds


def dist_setup(n):
    rank, world, local = 0, 1, 0
    if n > 1 or "RANK" in os.environ:
        import torch
        import torch.distributed as dist
        import datetime
        rank = int(os.environ.get("RANK", 0))
        world = int(os.environ.get("WORLD_SIZE", 1))
        local = int(os.environ.get("LOCAL_RANK", 0))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def allmax(x):
    """Max over ranks (NCCL on the GPU; a CPU tensor under gloo)."""
    import torch
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor([float(x)], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return float(x)


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None
        # raw samples go to JP_CLOCKS_DIR (default: the system temporary directory); the
        # JSON line carries their summary
        import tempfile
        out = os.environ.get("JP_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out, f"clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.5)          # nvidia-smi start-up, so that sampling covers the region
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def ncu_traffic():
    """Per-launch DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the pair
    kernel, from the committed ncu summary's `dram_bytes_per_launch:` line."""
    if os.path.exists(PAIR_PROFILE):
        for line in open(PAIR_PROFILE):
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":", 1)[1].split()[0]), os.path.relpath(PAIR_PROFILE, ROOT)
    return None, None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    return json.load(open(p)) if os.path.exists(p) else {}


def cpu_baseline(top, budget_s=15.0):
    """The CPU oracle (FP64 OpenMP restatement of md_run) on a bounded sample of the same
    workload, all host threads."""
    import oracle
    from j_presto_b200 import abi
    nth = os.cpu_count() or 1
    o = oracle.Oracle(top, method=abi.JP_METHOD_CANO, nthreads=nth)
    t0 = time.perf_counter()
    o.run(1)
    t1 = time.perf_counter() - t0
    n = int(max(2, min(200, budget_s / max(t1, 1e-3))))
    t0 = time.perf_counter()
    ier, _, _ = o.run(n)
    el = time.perf_counter() - t0
    return {"value": ns_per_day(n, el), "unit": "ns/day", "cores": nth, "kind": "port",
            "sample": f"{n} CANO steps of the same {top['natom']}-atom workload "
                      f"(oracle/oracle.cpp, OpenMP FP64), {el:.1f} s", "ier": ier}


def run_reference(args, rank):
    """--impl reference: the reference path's CPU implementation (md_run cannot be built
    here: no Fortran compiler), i.e. the oracle port, on the host cores."""
    if rank != 0:
        return
    from j_presto_b200 import systems
    top = systems.config_c2()
    import oracle
    from j_presto_b200 import abi
    nth = os.cpu_count() or 1
    o = oracle.Oracle(top, method=abi.JP_METHOD_CANO, nthreads=nth)
    w = max(1, min(args.warmup, 3))
    o.run(w)
    t0 = time.perf_counter()
    done, budget = 0, 150.0
    while done < args.steps:
        o.run(1)
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    v = ns_per_day(done, el)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "ns/day", "n_gpus": args.gpus,
            "steps": done, "warmup": w, "ms_per_step": 1e3 * el / done, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(int(top["natom"])), "atoms": int(top["natom"])},
            "cpu_baseline": {"value": v, "unit": "ns/day", "cores": nth, "kind": "port",
                             "sample": f"{done} CANO steps, oracle/oracle.cpp OpenMP FP64 "
                                       "(md_run itself needs a Fortran compiler, absent)"},
            "e2e": {"value": v, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def c4_measure(dev, steps=20, warmup=3):
    """C4: 64 uneven McMD replicas (8-30-residue chains in 600-9,000 waters), batched in one
    mixed-precision context (one CUDA graph per step) against the same 64 run one after the
    other on the FP64 path.  Both device-timed over `steps` steps after `warmup`."""
    from j_presto_b200 import abi, engine, systems
    reps = systems.config_c4(workers=os.cpu_count())
    natoms = [int(t["natom"]) for t in reps]
    for t in reps:                       # a placeholder to create the McMD contexts
        t["ge"] = systems.mcmd_weight(-1.0e7, 1.0e7)
    kw = dict(method=abi.JP_METHOD_GE, device=dev)
    eng = engine.Engine(reps, precision=abi.JP_PREC_MIXED, **kw)
    weights = []
    for r, t in enumerate(reps):         # 280-700 K over a range around each start energy
        e0 = eng.energy_grad(r)[0][0]
        w = systems.mcmd_weight(e0 - 0.1 * natoms[r], e0 + 0.3 * natoms[r])
        weights.append(w)
        eng.ge_set(w, r)
    eng.step(warmup, energies=False, temps=False)
    eng.step(steps, energies=False, temps=False)
    t_mix = eng.last_timing()[0] / 1e3
    per_step, _ = eng.launch_counts()
    eng.close()
    t64 = 0.0
    for r, t in enumerate(reps):
        t["ge"] = weights[r]
        e = engine.Engine(t, precision=abi.JP_PREC_FP64, **kw)
        e.step(warmup, energies=False, temps=False)
        e.step(steps, energies=False, temps=False)
        t64 += e.last_timing()[0] / 1e3
        e.close()
    n = len(reps)
    mix = ns_per_day(steps * n, t_mix)
    fp64 = ns_per_day(steps * n, t64)
    return {"workload": f"{n} McMD replicas (METHOD= GE, degree-8 weights 280-700 K): 8-30-residue "
                        f"chains in 600-9,000 waters, {min(natoms):,}-{max(natoms):,} atoms, "
                        f"{sum(natoms):,} in total, 2 fs, SHAKE X-H + rigid water",
            "atoms": sum(natoms), "replicas": n, "steps": steps,
            "mixed_batched": {"value": mix, "unit": "ns/day (aggregate)",
                              "ms_per_step": 1e3 * t_mix / steps, "launches_per_step": per_step},
            "fp64_back_to_back": {"value": fp64, "unit": "ns/day (aggregate)",
                                  "ms_per_step": 1e3 * t64 / steps},
            "speedup": mix / fp64}


def timed_loop(eng, steps, flush_buf):
    """K device-timed steps, L2 flushed between steps; returns per-step ms."""
    import torch
    per = []
    for _ in range(steps):
        eng.step(1, energies=False, temps=False)
        per.append(eng.last_timing()[0])
        flush_buf.zero_()
        torch.cuda.synchronize()
    return per


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle baseline")
    ap.add_argument("--no-c4", action="store_true", help="skip the 64-replica batched McMD line")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank, world, local = dist_setup(args.gpus)
    if args.impl == "reference":
        run_reference(args, rank)
        barrier()
        return
    import torch
    from j_presto_b200 import abi, build, engine, systems
    if rank == 0:
        build.build()
    barrier()
    dev = local
    torch.cuda.set_device(dev)
    top = systems.config_c2()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{dev}")
    kw = dict(method=abi.JP_METHOD_CANO, device=dev)
    eng = engine.Engine(top, precision=abi.JP_PREC_MIXED, **kw)
    e_mix, g_mix = eng.energy_grad()
    pairs0 = eng.pair_count()
    ntiles, nlisted, nslots = eng.list_stats()
    per_step, per_rebuild = eng.launch_counts()
    # warm-up + timed (mixed, resident state, per-step L2 flush)
    eng.step(args.warmup, energies=False, temps=False)
    barrier()
    torch.cuda.synchronize()
    with Clocks(dev) as clk:
        per = timed_loop(eng, args.steps, flush)
    torch.cuda.synchronize()
    t_mix = sum(per) / 1e3
    t_max = allmax(t_mix)
    value = ns_per_day(args.steps * world, t_max)
    # steady-state without flushes (informational)
    eng.step(args.steps, energies=False, temps=False)
    t_resident = eng.last_timing()[0] / 1e3
    # pair-kernel duration from CUDA events around each launch (timing mode, same stream)
    eng.set_timing(True)
    eng.step(args.steps, energies=False, temps=False)
    _, ph, ln = eng.last_timing()
    eng.set_timing(False)
    pair_ms = ph[0] / max(1, ln[0])
    _, _ = eng.energy_grad()
    pairs1 = eng.pair_count()
    pairs = 0.5 * (pairs0 + pairs1)
    # e2e through the C ABI with host buffers (pinned)
    n = top["natom"]
    hx = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    hv = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    eng.get_state(0, hx, hv)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.set_state(0, hx, hv)
        eng.step(1, energies=True, temps=False)
        eng.get_state(0, hx, hv)
    t_e2e = allmax(time.perf_counter() - t0)
    e2e = ns_per_day(args.steps * world, t_e2e)
    eng.close()
    # FP64 path on the same workload
    eng64 = engine.Engine(top, precision=abi.JP_PREC_FP64, **kw)
    e64, g64 = eng64.energy_grad()
    eng64.step(args.warmup, energies=False, temps=False)
    per64 = timed_loop(eng64, args.steps, flush)
    t64 = allmax(sum(per64) / 1e3)
    v64 = ns_per_day(args.steps * world, t64)
    eng64.close()
    rms = float(np.sqrt(((g_mix - g64) ** 2).sum() / (g64 ** 2).sum()))
    if rank != 0:
        barrier()
        return
    peak = engine.calibrate_fp32(dev)
    achieved = FLOPS_PER_PAIR * pairs / (pair_ms * 1e-3) / 1e12
    traffic, tsrc = ncu_traffic()
    hbm_peak = measured_peaks().get("hbm_gbs")
    hbm_src = "of measured"
    if not hbm_peak:   # the pool's earlier copy-bandwidth measurement
        hbm_peak, hbm_src = 6650.0, "of fallback (MEASURED_PEAKS.json absent)"
    cpu = None if args.no_cpu else cpu_baseline(top)
    c4 = None if (args.no_c4 or world > 1) else c4_measure(dev)
    clocks = clk.summary()
    nreb = args.steps // 10
    line = {
        "metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(int(n)), "atoms": int(n), "precision": "FP32 pair arithmetic, "
                   "64-bit fixed-point force/energy accumulation, FP64 integrate+SHAKE",
                   "l2": "flushed (256 MB write) between timed steps", "replicas_per_gpu": 1,
                   "parallelism": f"replicas x{world}"},
        "pairs_per_s": pairs * world * args.steps / t_max,
        "pairs_in_cutoff": pairs, "tiles": ntiles, "pairs_listed": nlisted,
        "tile_efficiency": pairs / (ntiles * 1024.0) if ntiles else None,
        "ms_per_step_resident": 1e3 * t_resident / args.steps,
        "fp64": {"value": v64, "unit": "ns/day", "ms_per_step": 1e3 * t64 / args.steps},
        "speedup_vs_fp64": value / v64,
        "rms_force_err": rms,
        "phase_ms_per_step": {"pair": ph[0] / max(1, ln[0]), "bonded": ph[1] / max(1, ln[1]),
                              "integrate": ph[2] / max(1, ln[2]),
                              "rebuild_per_call": ph[3] / max(1, ln[3])},
        "clocks": clocks,
        "e2e": {"value": e2e, "unit": "ns/day", "h2d_bytes_per_step": 2 * 3 * 8 * int(n),
                "d2h_bytes_per_step": 2 * 3 * 8 * int(n) + 8 * abi.JP_MAXENE,
                "timing": "host wall clock around set_state + jp_step(1) + get_state"},
        "gpu_launches": args.steps * per_step + nreb * per_rebuild,
        "roofline": {"bound": "fp32", "kernel": "k_pair_mixed", "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_source": tsrc,
                     "hbm": None if traffic is None or not hbm_peak else
                     {"achieved_gbs": traffic / (pair_ms * 1e-3) / 1e9, "peak_gbs": hbm_peak,
                      "frac": traffic / (pair_ms * 1e-3) / 1e9 / hbm_peak,
                      "note": "ncu DRAM bytes per launch / CUDA-event launch time, " + hbm_src},
                     "note": f"{FLOPS_PER_PAIR} FP32 flops per pair within rc x pairs per launch / "
                             "CUDA-event launch time; peak = FP32 FMA loop measured in this run "
                             "(MEASURED_PEAKS.json lists HBM and bf16 tensor peaks only)"},
        "cpu_baseline": cpu,
        "c4_batched_mcmd": c4,
    }
    print(json.dumps(line), flush=True)
    barrier()


if __name__ == "__main__":
    main()
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()
    except Exception:
        pass
