#!/usr/bin/env python
"""Benchmark of md_run's per-step force/integrate path on the B200 engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload (the metric's target configuration): 64 independent McMD replicas of
uneven size -- 8-30-residue chains in 600-9,000 waters, 2,000-30,000 atoms each, about
1.06 M atoms in all -- METHOD= GE with degree-8 weights spanning 280-700 K, zero-dipole
cut-off 12 A, SHAKE on X-H and rigid waters, 2 fs, the pair list rebuilt every UPDATE=10
steps as runmd does.  All 64 run in one mixed-precision context: one CUDA graph per step.
Synthetic and seeded.

Reported (one JSON line on rank 0):
  value      aggregate ns/day of the batched mixed path (FP32 pair arithmetic, 64-bit
             fixed-point forces, FP64 integration), device-timed with CUDA events, state
             resident in HBM, L2 flushed between timed steps
  e2e        the same metric through the C ABI with host buffers: every step copies all
             replicas' coordinates and velocities in from pinned host memory, runs one step
             and copies coordinates, velocities and energies out (jp_step_io, one
             synchronisation), timed by the host clock
  fp64       the 64 replicas one after another on the plain FP64 GPU path; speedup_vs_fp64
  roofline   the pair kernel (dominant) against the measured FP32 FMA peak
  accuracy   per configuration the mixed path against the FP64 path (RMS relative force
             error, potential-energy error) and the NVE drift of both paths
  c2, c3     the single-system configurations (solvated polymer, 99,200-atom water box)
  cpu_baseline  the CPU oracle (OpenMP FP64 restatement of md_run) on a bounded sample
With N > 1 (torchrun) every rank runs its own copy of the workload (replicas only, no
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
PAIR_PROFILE = os.path.join(ROOT, "profiles", "k_pair_mixed_c4.md")


def c4_name(natoms):
    return (f"{len(natoms)} McMD replicas batched (METHOD= GE, degree-8 weights 280-700 K): "
            f"8-30-residue chains in 600-9,000 waters, {min(natoms):,}-{max(natoms):,} atoms, "
            f"{sum(natoms):,} in total; ZD cut-off 12 A (list 13.5 A, UPDATE 10), SHAKE X-H + rigid "
            "water, dt 2 fs")


def c2_name(natom):
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


def c4_system(dev):
    """The 64 replicas and their McMD weights: 280-700 K over a range around each replica's
    starting potential energy (evaluated once on the FP64 path)."""
    from j_presto_b200 import abi, engine, systems
    reps = systems.config_c4(workers=os.cpu_count())
    natoms = [int(t["natom"]) for t in reps]
    for t in reps:                       # a placeholder to create the McMD context
        t["ge"] = systems.mcmd_weight(-1.0e7, 1.0e7)
    with engine.Engine(reps, precision=abi.JP_PREC_FP64, method=abi.JP_METHOD_GE, device=dev) as e:
        for r, t in enumerate(reps):
            e0 = e.energy_grad(r)[0][0]
            t["ge"] = systems.mcmd_weight(e0 - 0.1 * natoms[r], e0 + 0.3 * natoms[r])
    return reps, natoms


def cpu_baseline(reps, budget_s=15.0):
    """The CPU oracle (FP64 OpenMP restatement of md_run) on a bounded sample of the same
    workload, all host threads: every replica advanced by the same number of steps."""
    import oracle
    from j_presto_b200 import abi
    nth = os.cpu_count() or 1
    ors = [oracle.Oracle(t, method=abi.JP_METHOD_GE, nthreads=nth) for t in reps]
    t0 = time.perf_counter()
    for o in ors:
        o.run(1)
    t1 = time.perf_counter() - t0
    n = int(max(1, min(20, budget_s / max(t1, 1e-3))))
    t0 = time.perf_counter()
    ier = 0
    for o in ors:
        ier = ier or o.run(n)[0]
    el = time.perf_counter() - t0
    return {"value": ns_per_day(n * len(ors), el), "unit": "ns/day (aggregate)", "cores": nth,
            "kind": "port",
            "sample": f"{n} McMD steps of each of the {len(ors)} replicas (oracle/oracle.cpp, OpenMP "
                      f"FP64, one replica after another), {el:.1f} s", "ier": int(ier)}


def run_reference(args, rank):
    """--impl reference: the reference path's CPU implementation (md_run cannot be built
    here or on the GPU box: no Fortran compiler), i.e. the oracle port, on the host cores,
    on the same 64-replica workload: a step advances every replica by one MD step."""
    if rank != 0:
        return
    import oracle
    from j_presto_b200 import abi, systems
    reps = systems.config_c4(workers=os.cpu_count())
    natoms = [int(t["natom"]) for t in reps]
    nth = os.cpu_count() or 1
    ors = []
    for t in reps:
        o0 = oracle.Oracle(t, method=abi.JP_METHOD_MICR, nthreads=nth)
        e0 = o0.energy_grad()[0][0]
        t["ge"] = systems.mcmd_weight(e0 - 0.1 * t["natom"], e0 + 0.3 * t["natom"])
        ors.append(oracle.Oracle(t, method=abi.JP_METHOD_GE, nthreads=nth))
    w = max(1, min(args.warmup, 3))
    for o in ors:
        o.run(w)
    t0 = time.perf_counter()
    done, budget = 0, 150.0
    while done < args.steps:
        for o in ors:
            o.run(1)
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    v = ns_per_day(done * len(ors), el)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "ns/day", "n_gpus": args.gpus,
            "steps": done, "warmup": w, "ms_per_step": 1e3 * el / done, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": c4_name(natoms), "atoms": sum(natoms), "replicas": len(natoms)},
            "cpu_baseline": {"value": v, "unit": "ns/day", "cores": nth, "kind": "port",
                             "sample": f"{done} steps of each of the {len(ors)} McMD replicas, "
                                       "oracle/oracle.cpp OpenMP FP64, one replica after another "
                                       "(md_run itself needs a Fortran compiler, absent)"},
            "e2e": {"value": v, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


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


def phase_times(eng, steps):
    """Per-launch device times of the step's phases (timing mode: direct launches with CUDA
    events on the context's stream around each phase)."""
    eng.set_timing(True)
    eng.step(steps, energies=False, temps=False)
    _, ph, ln = eng.last_timing()
    eng.set_timing(False)
    return {"pair": ph[0] / max(1, ln[0]), "bonded": ph[1] / max(1, ln[1]),
            "integrate": ph[2] / max(1, ln[2]), "rebuild_per_call": ph[3] / max(1, ln[3])}


def e2e_loop(eng, natom_total, nrep, steps):
    """jp_step_io per step with pinned host buffers; host wall clock."""
    import torch
    hx = torch.empty((natom_total, 3), dtype=torch.float64, pin_memory=True).numpy()
    hv = torch.empty((natom_total, 3), dtype=torch.float64, pin_memory=True).numpy()
    he = torch.empty((1, nrep, 15), dtype=torch.float64, pin_memory=True).numpy()
    eng.step_io(None, None, hx, hv, nsteps=0)
    t0 = time.perf_counter()
    for _ in range(steps):
        eng.step_io(hx, hv, hx, hv, he, nsteps=1)
    return time.perf_counter() - t0, 2 * hx.nbytes, 2 * hx.nbytes + he.nbytes


def single_config(top, dev, steps, warmup, flush, with_e2e=False):
    """A single-system configuration (CANO): mixed and FP64 ns/day, phase times, errors."""
    from j_presto_b200 import abi, engine
    kw = dict(method=abi.JP_METHOD_CANO, device=dev)
    out = {"atoms": int(top["natom"])}
    grads = {}
    for name, prec in (("mixed", abi.JP_PREC_MIXED), ("fp64", abi.JP_PREC_FP64)):
        with engine.Engine(top, precision=prec, **kw) as e:
            ene, g = e.energy_grad()
            grads[name] = (ene, g)
            pairs = e.pair_count()
            ntiles, nlisted, _ = e.list_stats()
            e.step(warmup, energies=False, temps=False)
            per = timed_loop(e, steps, flush)
            t = sum(per) / 1e3
            out[name] = {"value": ns_per_day(steps, t), "unit": "ns/day", "ms_per_step": 1e3 * t / steps,
                         "phase_ms": phase_times(e, max(10, steps))}
            if name == "mixed":
                out.update(pairs_in_cutoff=pairs, tiles=ntiles, pairs_listed=nlisted,
                           tile_efficiency=pairs / (ntiles * 512.0) if ntiles else None)
                if with_e2e:
                    te, bi, bo = e2e_loop(e, int(top["natom"]), 1, steps)
                    out["e2e"] = {"value": ns_per_day(steps, te), "unit": "ns/day",
                                  "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo}
    out["speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    (em, gm), (e64, g64) = grads["mixed"], grads["fp64"]
    out["rms_force_err"] = float(np.sqrt(((gm - g64) ** 2).sum() / (g64 ** 2).sum()))
    out["energy_err"] = float(abs(em[0] - e64[0]) / abs(e64[0]))
    return out


def c5_measure(dev, steps, warmup, flush):
    """C5: 32 ALSD replicas (12-residue chain in 3,000 waters, a 4-residue lambda cluster,
    CLSTMETHOD= LMD with the McMD weight in lambda, torsions scaled) batched in one mixed
    context against the same replicas one after another on the FP64 path."""
    from j_presto_b200 import abi, engine, systems
    reps = systems.config_c5(workers=os.cpu_count())
    natoms = [int(t["natom"]) for t in reps]
    kw = dict(method=abi.JP_METHOD_GE, alsd=abi.JP_ALSD_LMD, lambda0=0.8,
              scale_terms=abi.JP_SCALE_TORS, device=dev)
    with engine.Engine(reps, precision=abi.JP_PREC_MIXED, **kw) as e:
        e.step(warmup, energies=False, temps=False)
        t_mix = sum(timed_loop(e, steps, flush)) / 1e3
    t64 = 0.0
    for t in reps:
        with engine.Engine(t, precision=abi.JP_PREC_FP64, **kw) as e:
            e.step(warmup, energies=False, temps=False)
            e.step(steps, energies=False, temps=False)
            t64 += e.last_timing()[0] / 1e3
    n = len(reps)
    mix, v64 = ns_per_day(steps * n, t_mix), ns_per_day(steps * n, t64)
    return {"workload": f"{n} ALSD replicas (CLSTMETHOD= LMD, METHOD= GE, weight in lambda on "
                        f"[0.6, 1.0]): 12-residue chain in 3,000 waters, {min(natoms):,}-"
                        f"{max(natoms):,} atoms, {sum(natoms):,} in total, 2 fs",
            "atoms": sum(natoms), "replicas": n, "steps": steps,
            "mixed_batched": {"value": mix, "unit": "ns/day (aggregate)", "ms_per_step": 1e3 * t_mix / steps},
            "fp64_back_to_back": {"value": v64, "unit": "ns/day (aggregate)", "ms_per_step": 1e3 * t64 / steps},
            "speedup_vs_fp64": mix / v64}


def accuracy(dev, c2_acc, c3_acc):
    """Mixed against FP64 on every single-system configuration, and NVE drift (C1': 1,000
    waters at liquid density, METHOD= MICR, SHAKE, 2 fs, 1 ns) of both paths in kT per ns
    per degree of freedom, the total energy kept as md_run keeps it (potential energy at t
    plus the kinetic energy of (v(t-dt/2) + v(t+dt/2)) / 2)."""
    import oracle
    from j_presto_b200 import abi, engine, systems
    kb = 8.31451 / 4184.0
    acc = {"c2": c2_acc, "c3": c3_acc}
    c1 = systems.config_c1()
    g = {}
    for name, prec in (("mixed", abi.JP_PREC_MIXED), ("fp64", abi.JP_PREC_FP64)):
        with engine.Engine(c1, precision=prec, method=abi.JP_METHOD_MICR, device=dev) as e:
            g[name] = e.energy_grad()
    (em, gm), (e64, g64) = g["mixed"], g["fp64"]
    acc["c1"] = {"rms_force_err": float(np.sqrt(((gm - g64) ** 2).sum() / (g64 ** 2).sum())),
                 "energy_err": float(abs(em[0] - e64[0]) / abs(e64[0]))}
    top = systems.config_c1_prime()
    dof = oracle.Oracle(top, method=abi.JP_METHOD_MICR).dof
    with engine.Engine(top, precision=abi.JP_PREC_FP64, method=abi.JP_METHOD_CANO, tempco=1,
                       device=dev) as e:     # 10 ps at 300 K from the lattice start
        e.step(5000, energies=False, temps=False)
        x0, v0 = e.get_state()
    nsteps = 500000
    drift = {}
    # md_run's SHAKE tolerance (COVSHK 1e-6), and 1e-10 to show how much of the drift it makes
    runs = (("mixed", abi.JP_PREC_MIXED, 1e-6), ("fp64", abi.JP_PREC_FP64, 1e-6),
            ("mixed_covshk1e-10", abi.JP_PREC_MIXED, 1e-10), ("fp64_covshk1e-10", abi.JP_PREC_FP64, 1e-10))
    for name, prec, tol in runs:
        with engine.Engine(top, precision=prec, method=abi.JP_METHOD_MICR, shake_tol=tol, device=dev) as e:
            e.set_state(cord=x0, vel=v0)
            e.rebuild()
            E, T = e.step(nsteps)
        tot = E[:, 0, 0] + 0.5 * dof * kb * T[:, 0]
        skip = nsteps // 10
        t_ns = np.arange(nsteps) * DT_FS * 1e-6
        unit = kb * T[skip:, 0].mean() * dof
        # the total energy wanders slowly (about 0.1 kcal/mol between 1 ps means), so the
        # scatter of points about one fitted line understates the slope's error: the slope is
        # that of the whole run and its error the scatter of the slopes of 10 independent
        # segments divided by sqrt(10)
        slope = np.polyfit(t_ns[skip:], tot[skip:], 1)[0]
        seg = np.array_split(np.arange(skip, nsteps), 10)
        ss = np.array([np.polyfit(t_ns[q], tot[q], 1)[0] for q in seg])
        drift[name] = float(slope / unit)
        drift[name + "_stderr"] = float(ss.std(ddof=1) / np.sqrt(len(ss)) / unit)
        drift[name + "_wander_kcal"] = float(tot[skip:].std())
    acc["nve_drift_kT_per_ns_per_dof"] = {
        "workload": f"C1': 1,000 waters (3,000 atoms) in a 31 A box, 10 ps METHOD= CANO at 300 K, "
                    f"then METHOD= MICR, SHAKE (COVSHK 1e-6, md_run's default, and 1e-10), 2 fs, "
                    f"{nsteps} steps ({nsteps * DT_FS / 1000:.0f} ps), {dof} degrees of freedom",
        **drift}
    return acc


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle baseline")
    ap.add_argument("--no-extra", action="store_true", help="only the headline (no C2/C3/accuracy)")
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
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{dev}")
    reps, natoms = c4_system(dev)
    nrep, ntot = len(reps), sum(natoms)
    kw = dict(method=abi.JP_METHOD_GE, device=dev)
    eng = engine.Engine(reps, precision=abi.JP_PREC_MIXED, **kw)
    for r in range(nrep):
        eng.energy_grad(r)
    pairs = float(sum(eng.pair_count(r) for r in range(nrep)))
    ntiles, nlisted, _ = eng.list_stats()
    per_step, per_rebuild = eng.launch_counts()
    shapes = [eng.tile_shape(r) for r in range(nrep)]
    tshape = {"note": "block-shape tuner: per replica the column-edge factor with the fewest pair "
                      "records of five (jp_tile_shape); counts of the 64 replicas summed per factor",
              "chosen_factor_counts": {str(f): sum(1 for g, _ in shapes if g == f)
                                       for f in sorted({g for g, _ in shapes})},
              "tiles_per_factor": [int(sum(t[q] for _, t in shapes)) for q in range(5)],
              "tiles_chosen": int(sum(min(t) for _, t in shapes))}
    # warm-up + timed (resident state, L2 flushed between steps)
    eng.step(args.warmup, energies=False, temps=False)
    barrier()
    torch.cuda.synchronize()
    with Clocks(dev) as clk:
        per = timed_loop(eng, args.steps, flush)
    torch.cuda.synchronize()
    t_max = allmax(sum(per) / 1e3)
    value = ns_per_day(args.steps * nrep * world, t_max)
    phases = phase_times(eng, max(10, args.steps))
    pair_ms = phases["pair"]
    barrier()
    te, h2d, d2h = e2e_loop(eng, ntot, nrep, args.steps)
    t_e2e = allmax(te)
    e2e = ns_per_day(args.steps * nrep * world, t_e2e)
    eng.close()
    # the same replicas one after another on the FP64 path
    t64 = 0.0
    for t in reps:
        with engine.Engine(t, precision=abi.JP_PREC_FP64, **kw) as e:
            e.step(args.warmup, energies=False, temps=False)
            e.step(args.steps, energies=False, temps=False)
            t64 += e.last_timing()[0] / 1e3
    t64 = allmax(t64)
    v64 = ns_per_day(args.steps * nrep * world, t64)
    if rank != 0:
        barrier()
        return
    clocks = clk.summary()
    c2 = c3 = c5 = acc = None
    if not args.no_extra and world == 1:
        c2 = single_config(systems.config_c2(), dev, args.steps, args.warmup, flush, with_e2e=True)
        c3 = single_config(systems.config_c3(), dev, args.steps, args.warmup, flush)
        c5 = c5_measure(dev, args.steps, args.warmup, flush)
        acc = accuracy(dev, {k: c2[k] for k in ("rms_force_err", "energy_err")},
                       {k: c3[k] for k in ("rms_force_err", "energy_err")})
    peak = engine.calibrate_fp32(dev)
    achieved = FLOPS_PER_PAIR * pairs / (pair_ms * 1e-3) / 1e12
    traffic, tsrc = ncu_traffic()
    hbm_peak = measured_peaks().get("hbm_gbs")
    hbm_src = "of measured"
    if not hbm_peak:   # the pool's earlier copy-bandwidth measurement
        hbm_peak, hbm_src = 6650.0, "of fallback (MEASURED_PEAKS.json absent)"
    cpu = None if args.no_cpu else cpu_baseline(reps)
    nreb = args.steps // 10
    line = {
        "metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": c4_name(natoms), "atoms": ntot, "replicas": nrep,
                   "precision": "FP32 pair arithmetic, 64-bit fixed-point force/energy accumulation, "
                                "FP64 integrate+SHAKE",
                   "l2": "flushed (256 MB write) between timed steps",
                   "parallelism": f"replicas x{world}"},
        "pairs_per_s": pairs * world * args.steps / t_max,
        "pairs_in_cutoff": pairs, "tiles": ntiles, "pairs_listed": nlisted,
        "tile_efficiency": pairs / (ntiles * 512.0) if ntiles else None,   # 16 x 32 slots per record
        "fp64": {"value": v64, "unit": "ns/day", "ms_per_step": 1e3 * t64 / args.steps,
                 "note": "the same replicas one after another, each in its own FP64 context"},
        "speedup_vs_fp64": value / v64,
        "phase_ms": phases,
        "clocks": clocks,
        "e2e": {"value": e2e, "unit": "ns/day", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "timing": "host wall clock around jp_step_io(1): all replicas' x, v in from pinned "
                          "memory, one step, x, v and energies out, one synchronisation"},
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
        "accuracy": acc,
        "c2": c2,
        "c3": c3,
        "c5": c5,
        "tile_shape": tshape,
        "cpu_baseline": cpu,
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
