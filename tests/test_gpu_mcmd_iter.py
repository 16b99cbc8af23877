"""One McMD weight iteration measured, not predicted: four small McMD replicas run with a
starting weight and record their energy histograms on the device; GEprep's fit (the
polynomial, fallback and yardstick) and the surrogate network are made from those histograms;
each then drives the next run of all four replicas from the same state, and the flatness
of the energy histograms those runs actually record (distrib_MULT's percentage and the
max/min visit ratio) decides: the network is kept only if it is no worse.
"""
import numpy as np
import pytest

from j_presto_b200 import abi, engine as _eng, ge, geprep, systems

pytestmark = pytest.mark.gpu

NBIN, NBOR = 60, 4


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    return _eng


def _flat(counts, emin, emax):
    d = geprep.distribution(counts, emin, emax, NBIN, NBOR)
    inner = np.sum(counts, 0)[NBOR:NBOR + NBIN]
    return d["flat"], (inner.max() / inner.min() if inner.min() > 0 else float("inf"))


def test_measured_flatness_decides(eng_mod):
    tops = [systems.solvated_polymer(4, 500, seed=41 + r) for r in range(4)]
    for t in tops:   # a flat 300 K weight: canonical dynamics while the start relaxes
        t["ge"] = systems.mcmd_weight(-1.0e7, 1.0e7, t_lo=300.0, t_hi=300.0)
    kw = dict(method=abi.JP_METHOD_GE)
    nsteps = 2000
    with eng_mod.Engine(tops, precision=abi.JP_PREC_MIXED, **kw) as e:
        # the lattice start releases some 5000 kcal/mol over its first thousand steps:
        # minimise (200 iterations: with SHAKE the step length of a longer descent vanishes,
        # JP_E_MIN_STEP) and run 800 steps at 300 K first; the weight's range starts 300
        # kcal/mol below the energy reached, where its temperature ramp (280 K at the bottom,
        # 700 K at the top) is near the system's 300 K, so the McMD walk starts inside the
        # range and explores upwards (on the oracle: up 1,400 kcal/mol in 2,000 steps, and the
        # polynomial's run then records a flatness of 11 % on the sampled range)
        e.minimize(warn_ok=True, max_loop=200)
        e.step(800, energies=False, temps=False)
        e1 = [e.energy_grad(r)[0][0] for r in range(4)]
        w0 = [systems.mcmd_weight(x - 300.0, x + 1500.0) for x in e1]
        for r in range(4):
            e.ge_set(w0[r], r)
            e.ge_hist_setup(w0[r]["celw"], w0[r]["ceup"], NBIN, NBOR, rep=r)
        e.step(nsteps, energies=False, temps=False)
        hist = [e.ge_hist_get(r) for r in range(4)]
        state = [e.get_state(r) for r in range(4)]
    assert all(h.sum() > 0 for h in hist)
    # the next weight spans the energies the runs sampled (GEprep's next range: a polynomial
    # is not extrapolated over a range without data), and its flatness is measured there
    nxt = []
    for r in range(4):
        de = (w0[r]["ceup"] - w0[r]["celw"]) / NBIN
        centres = w0[r]["celw"] + (np.arange(NBIN + 2 * NBOR) - NBOR + 0.5) * de
        seen = centres[hist[r] > 0]
        nxt.append((float(seen.min()), float(seen.max()) + de))
    its = [ge.iterate(hist[r], w0[r], w0[r]["celw"], w0[r]["ceup"], NBIN, NBOR, nxt[r][0], nxt[r][1],
                      300.0, epochs=1500, seed=r) for r in range(4)]

    def run(use_net):
        with eng_mod.Engine(tops, precision=abi.JP_PREC_MIXED, **kw) as e:
            for r in range(4):
                e.set_state(r, *state[r])
                e.ge_set(its[r]["poly"], r)
                if use_net:
                    e.ge_set_mlp(its[r]["mlp"], r)
                e.ge_hist_setup(nxt[r][0], nxt[r][1], NBIN, NBOR, rep=r)
            e.rebuild()
            e.step(nsteps, energies=False, temps=False)
            out = [_flat([e.ge_hist_get(r)], nxt[r][0], nxt[r][1]) for r in range(4)]
        return out

    poly, net = run(False), run(True)
    fp = float(np.mean([f for f, _ in poly]))
    fn = float(np.mean([f for f, _ in net]))
    assert 0.0 < fp <= 100.0 and 0.0 < fn <= 100.0
    keep = fn >= fp
    print(f"measured flatness: polynomial {fp:.1f} %, network {fn:.1f} % -> "
          f"{'network kept' if keep else 'polynomial kept'}")
