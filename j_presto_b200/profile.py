"""Profiling driver: a fixed number of MD steps of one workload, for ncu.

    python -m j_presto_b200.profile --workload c2 --precision mixed --steps 20 [--direct]

--direct launches every kernel individually (timing mode) instead of replaying CUDA graphs.
Workloads: c1 (3,000 waters, 31 A), c1p (1,000 waters), c2 (solvated polymer, 22,860
atoms), c3 (33,000 waters + 200 ions), c4 (64 McMD replicas, 1.06 M atoms), small
(6-residue chain in 700 waters), w7000 (7,000 waters, 62 A).
"""
import argparse

from . import abi, build, engine, systems

WORKLOADS = {
    "c1": systems.config_c1,
    "c1p": systems.config_c1_prime,
    "c2": systems.config_c2,
    "c3": systems.config_c3,
    "small": lambda: systems.solvated_polymer(6, 700, seed=11),
    "w7000": lambda: systems.water_box(7000, 62.0, seed=9),
    "c4": None,   # 64 McMD replicas, built below
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--method", default="cano", choices=["micr", "cano"])
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--direct", action="store_true")
    ap.add_argument("--tempco", type=int, default=2, choices=[1, 2])
    a = ap.parse_args()
    build.build()
    prec = abi.JP_PREC_MIXED if a.precision == "mixed" else abi.JP_PREC_FP64
    meth = abi.JP_METHOD_CANO if a.method == "cano" else abi.JP_METHOD_MICR
    if a.workload == "c4":
        import os
        top = systems.config_c4(workers=os.cpu_count())
        for t in top:
            t["ge"] = systems.mcmd_weight(-1.0e7, 1.0e7)
        meth = abi.JP_METHOD_GE
    else:
        top = WORKLOADS[a.workload]()
    with engine.Engine(top, precision=prec, method=meth, tempco=a.tempco) as e:
        e.set_timing(a.direct)
        e.step(a.steps, energies=False, temps=False)
        tot, ph, ln = e.last_timing()
        nt, nl, ns = e.list_stats()
    natom = sum(t["natom"] for t in top) if isinstance(top, list) else top["natom"]
    print(f"{a.workload} natom={natom} steps={a.steps} ms/step={tot / a.steps:.4f} "
          f"tiles={nt} listed={nl} phases_ms={[round(p, 4) for p in ph]} launches={ln}")


if __name__ == "__main__":
    main()
