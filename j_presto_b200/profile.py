"""Profiling driver: a fixed number of MD steps of one workload, for ncu.

    python -m j_presto_b200.profile --workload c2 --precision mixed --steps 20 [--direct]

--direct launches every kernel individually (timing mode) instead of replaying CUDA graphs.
Workloads: c1 (3,000 waters, 31 A), c1p (1,000 waters), c2 (solvated polymer, 22,860
atoms), c3 (33,000 waters + 200 ions), c4 (64 McMD replicas, 1.06 M atoms), c4q (the first 16
of those replicas, 266 k atoms: a pair-tile list of several times L2 in a few hundred MB of
device memory), small (6-residue chain in 700 waters), w7000 (7,000 waters, 62 A), and tour
(every kernel of the library at least once on small systems: mixed and FP64 pair tiles,
MICR, CANO in both integrator forms, McMD with the network weight, ALSD, CMM, H-bond pairs,
restraints with the CAP, steepest descent, network training).
"""
import argparse
import time

import numpy as np

from . import abi, build, engine, systems


def _c4(nrep=64):
    import os
    top = systems.config_c4(nrep=nrep, workers=os.cpu_count())   # the first nrep of the 64
    for t in top:
        t["ge"] = systems.mcmd_weight(-1.0e7, 1.0e7)
    return top


def tour(steps):
    """Each feature's kernels on a small system, `steps` MD steps (timing mode: one launch per
    kernel); prints one line per run."""
    MIXED, FP64 = abi.JP_PREC_MIXED, abi.JP_PREC_FP64
    CANO, GE, MICR = abi.JP_METHOD_CANO, abi.JP_METHOD_GE, abi.JP_METHOD_MICR
    poly = systems.solvated_polymer(20, 1500, seed=7)
    drop = dict(systems.droplet(12, 1200, seed=9), box=np.full(3, 28.0))
    ge_poly = dict(poly, ge=systems.mcmd_weight(-1.0e7, 1.0e7))
    hb_pairs = systems.HBOND_PAIRS + ((systems.T_HW, systems.T_OW),)
    runs = [
        ("mixed CANO", poly, dict(precision=MIXED, method=CANO), 0),
        ("FP64 CANO", poly, dict(precision=FP64, method=CANO), 0),
        ("mixed MICR", poly, dict(precision=MIXED, method=MICR), 0),
        ("mixed CANO per-phase", poly, dict(precision=MIXED, method=CANO), 2),
        ("CMM", drop, dict(precision=MIXED, method=CANO, cal15m=abi.JP_CAL15M_CMM,
                           bounda=abi.JP_BOUND_NONE), 0),
        ("H-bond", systems.with_hbond(dict(poly), pairs=hb_pairs), dict(precision=MIXED, method=CANO), 0),
        ("restraints + CAP", systems.with_restraints(dict(drop), cap=True),
         dict(precision=MIXED, method=CANO, bounda=abi.JP_BOUND_NONE), 0),
        ("ALSD", systems.alsd_replica(systems.solvated_polymer(4, 500, seed=31), walls=20000.0),
         dict(precision=MIXED, method=GE, alsd=abi.JP_ALSD_LMD, lambda0=0.81,
              scale_terms=abi.JP_SCALE_TORS), 0),
    ]
    for name, top, kw, grid in runs:
        with engine.Engine(top, **kw) as e:
            if grid:
                e.set_grid_limit(grid)
            e.set_timing(True)
            e.step(steps, energies=False, temps=False)
            tot, _, ln = e.last_timing()
        print(f"tour {name}: natom={top['natom']} ms/step={tot / steps:.4f} launches={ln}", flush=True)
    # McMD with the network weight (k_ge_scale, the network forward pass)
    rng = np.random.default_rng(1)
    x = np.sort(rng.uniform(0.0, 1.0, 64))
    data = (x, 1.0 / (0.0019872 * (280.0 + 420.0 * x)), np.ones_like(x))
    params, _, _ = engine.mlp_train([data], epochs=20)
    with engine.Engine(ge_poly, precision=MIXED, method=GE) as e:
        e.ge_set_mlp(params[0])
        e.set_timing(True)
        e.step(steps, energies=False, temps=False)
    print("tour McMD network weight: done", flush=True)
    with engine.Engine(poly, precision=FP64, method=CANO) as e:
        its, _, _, _ = e.minimize(warn_ok=True, max_loop=6, update=5)
    print(f"tour steepest descent: iterations={int(its[0])}", flush=True)

WORKLOADS = {
    "c1": systems.config_c1,
    "c1p": systems.config_c1_prime,
    "c2": systems.config_c2,
    "c3": systems.config_c3,
    "small": lambda: systems.solvated_polymer(6, 700, seed=11),
    "w7000": lambda: systems.water_box(7000, 62.0, seed=9),
    "c4": None,   # 64 McMD replicas, built below
    "c4q": None,  # the first 16 of them
    "tour": None,
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--method", default="cano", choices=["micr", "cano"])
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--direct", action="store_true")
    ap.add_argument("--rebuilds", type=int, default=0,
                    help="then time this many list builds (host clock around each synchronous call)")
    ap.add_argument("--tempco", type=int, default=2, choices=[1, 2])
    a = ap.parse_args()
    build.build()
    prec = abi.JP_PREC_MIXED if a.precision == "mixed" else abi.JP_PREC_FP64
    meth = abi.JP_METHOD_CANO if a.method == "cano" else abi.JP_METHOD_MICR
    if a.workload == "tour":
        tour(a.steps)
        return
    if a.workload in ("c4", "c4q"):
        top = _c4(64 if a.workload == "c4" else 16)
        meth = abi.JP_METHOD_GE
    else:
        top = WORKLOADS[a.workload]()
    with engine.Engine(top, precision=prec, method=meth, tempco=a.tempco) as e:
        e.step(2, energies=False, temps=False)   # every kernel launched once before timing
        e.set_timing(a.direct)
        e.step(a.steps, energies=False, temps=False)
        tot, ph, ln = e.last_timing()
        nt, nl, ns = e.list_stats()
        reb = []
        for _ in range(a.rebuilds):
            t0 = time.perf_counter()
            e.rebuild()
            reb.append(1e3 * (time.perf_counter() - t0))
    natom = sum(t["natom"] for t in top) if isinstance(top, list) else top["natom"]
    print(f"{a.workload} natom={natom} steps={a.steps} ms/step={tot / a.steps:.4f} "
          f"tiles={nt} listed={nl} phases_ms={[round(p, 4) for p in ph]} launches={ln}"
          + (f" rebuild_ms_median={sorted(reb)[len(reb) // 2]:.4f}" if reb else ""))


if __name__ == "__main__":
    main()
