"""ALSD weight iteration on the GPU: the engine's lambda histograms (jp_alsd_hist_*), the
GEprep distrib_ALSD fit of the weight in lambda, and the (E, lambda) network weight.

* after one step the lambda histogram holds one visit at lambda(t) with the step's
  dE/dlambda of the cluster energy, 2 lambda E_AA + E_AB (LMD), E_AA and E_AB the class
  energies of that force evaluation (to 1e-10 relative), and the (E, lambda) histogram one
  visit at the step's total potential energy;
* one iteration on four small replicas: the polynomial weight from distrib_ALSD and the
  network trained on the (E, lambda) histograms each drive a run from the same state; both
  runs count every step, and the network is kept only if the flatness measured on its run
  (GEprep's percentage) is no worse than the polynomial's, the polynomial being the yardstick.
"""
import numpy as np
import pytest

from j_presto_b200 import abi, engine as _eng, geprep, systems

pytestmark = pytest.mark.gpu

KW = dict(method=abi.JP_METHOD_GE, alsd=abi.JP_ALSD_LMD, lambda0=0.81, scale_terms=abi.JP_SCALE_TORS)
LMIN, LMAX, NBIN, NBOR = 0.6, 1.0, 20, 2
WALL = 20000.0


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    return _eng


def _reps(n):
    # walls that hold lambda near [0.6, 1.0]: the cluster's solvation force
    # (-2 lambda E_AA - E_AB, some 300 kcal/mol) drives lambda past a weak wall until the
    # trajectory fails (the oracle shows the same); with slope 20000 the oracle keeps lambda
    # in [0.90, 1.09] over 1500 steps for these four seeds
    return [systems.alsd_replica(systems.solvated_polymer(4, 500, seed=31 + r), seed=r, walls=WALL)
            for r in range(n)]


def test_histogram_records_the_step(eng_mod):
    top = _reps(1)[0]
    with eng_mod.Engine(top, precision=abi.JP_PREC_FP64, **KW) as e:
        e0 = e.energy_grad()[0][0]
        e.alsd_hist_setup(LMIN, LMAX, NBIN, NBOR, e0 - 400.0, e0 + 400.0, 40)
        E, _ = e.step(1)
        (lam, _), ec = e.get_lambda()
        c, f, c2, f2 = e.alsd_hist_get()
    assert lam != 0.81                       # lambda moved, the record is of lambda(t)
    k = int((0.81 - (LMIN - 0.02 * NBOR)) / 0.02)
    assert c.sum() == 1 and c[k] == 1
    assert f[k] == pytest.approx(2.0 * 0.81 * ec[0] + ec[1], rel=1e-10)
    a = int((E[0, 0, 0] - (e0 - 400.0)) / 20.0)
    assert c2.sum() == 1 and c2[a, k] == 1 and f2[a, k] == pytest.approx(f[k], rel=1e-12)


def _run(reps, setup, nsteps, x0v0):
    flats = []
    with _eng.Engine(reps, precision=abi.JP_PREC_MIXED, **KW) as e:
        for r, (x, v) in enumerate(x0v0):
            e.set_state(r, x, v)
            e.set_lambda(0.81, 0.0, rep=r)
        e.rebuild()
        setup(e)
        for r in range(len(reps)):
            e.alsd_hist_setup(LMIN, LMAX, NBIN, NBOR, rep=r)
        e.step(nsteps, energies=False, temps=False)
        for r in range(len(reps)):
            c, _, _, _ = e.alsd_hist_get(r)
            assert c.sum() <= nsteps
            flats.append(c)
    d = geprep.alsd_distribution(flats, [np.zeros_like(c) for c in flats], LMIN, LMAX, NBIN, NBOR, 300.0)
    return d["flat"], d["maxmin"], int(sum(c.sum() for c in flats))


def test_one_iteration_polynomial_and_network(eng_mod):
    reps = _reps(4)
    nsteps = 1500
    with eng_mod.Engine(reps, precision=abi.JP_PREC_MIXED, **KW) as e:
        e0 = [e.energy_grad(r)[0][0] for r in range(len(reps))]
        lo, hi = min(e0) - 600.0, max(e0) + 600.0
        for r in range(len(reps)):
            e.alsd_hist_setup(LMIN, LMAX, NBIN, NBOR, lo, hi, 60, rep=r)
        e.step(nsteps, energies=False, temps=False)
        hist = [e.alsd_hist_get(r) for r in range(len(reps))]
        x0v0 = [e.get_state(r) for r in range(len(reps))]
    counts = [h[0] for h in hist]
    assert all(c.sum() > 0 for c in counts)
    d = geprep.alsd_distribution(counts, [h[1] for h in hist], LMIN, LMAX, NBIN, NBOR, 300.0)
    # the next weight spans the lambda range the runs sampled (a polynomial is not
    # extrapolated), with steep walls outside it
    seen = d["EE"][d["P"] > 0]
    nf, _, _ = geprep.alsd_fit(d, float(seen.min()), float(seen.max()), 300.0, 1, 2, WALL, WALL)
    X = np.concatenate([geprep.alsd_net_data(h[2], h[3], lo, hi, LMIN, LMAX, NBIN, NBOR, 300.0)[0]
                        for h in hist])
    Y = np.concatenate([geprep.alsd_net_data(h[2], h[3], lo, hi, LMIN, LMAX, NBIN, NBOR, 300.0)[1]
                        for h in hist])
    W = np.concatenate([geprep.alsd_net_data(h[2], h[3], lo, hi, LMIN, LMAX, NBIN, NBOR, 300.0)[2]
                        for h in hist])
    params, loss, _ = _eng.mlp_train([(X, Y, W)], nin=2, nout=2, epochs=1500, lr=1e-3, seed=3)
    assert np.isfinite(loss).all() and np.isfinite(params).all()

    def poly(e):
        for r in range(len(reps)):
            e.ge_set(nf, r)

    def net(e):
        for r in range(len(reps)):
            e.ge_set(nf, r)
            e.alsd_set_mlp(params[0], lo, hi, rep=r)

    fp, rp, np_ = _run(reps, poly, nsteps, x0v0)
    fn, rn, nn = _run(reps, net, nsteps, x0v0)
    assert 0.0 < fp <= 100.0 and 0.0 < fn <= 100.0
    use_net = fn >= fp
    print(f"flatness polynomial {fp:.1f} % (max/min {rp:.2f}), network {fn:.1f} % (max/min {rn:.2f}); "
          f"network {'kept' if use_net else 'rejected'}")
    assert np_ > 0 and nn > 0
