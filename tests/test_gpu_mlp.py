"""The weight surrogate network on the GPU: forward and gradient against the float64 oracle,
batched training, its use in the McMD force scaling, and what it gains over the polynomial.

Tolerances: FP32 network against the float64 oracle -- outputs 1e-5 relative, gradient
entries 2e-3 of the largest entry, loss 1e-4 relative.
"""
import numpy as np
import pytest

import oracle
from oracle import mlp as ora
from j_presto_b200 import abi, ge, systems

pytestmark = pytest.mark.gpu

R_KCAL = 8.31451 / 4.184 * 1e-3


@pytest.fixture(scope="module")
def eng(engine_lib):
    from j_presto_b200 import engine
    return engine


def _data(seed, n=120):
    rng = np.random.default_rng(seed)
    x = np.sort(rng.uniform(0.0, 1.0, n))
    y = 1.0 / (R_KCAL * (280.0 + 420.0 * x)) + 0.01 * rng.normal(size=n)
    w = np.sqrt(rng.integers(1, 300, n).astype(float))
    return x, y, w


def test_forward_and_gradient_match_oracle(eng):
    x, y, w = _data(1)
    p0, loss, g = eng.mlp_train([(x, y, w)], epochs=0, grad=True)
    lo, go = ora.loss_grad(p0[0].astype(np.float64), x, y, w, 1, 1)
    np.testing.assert_allclose(loss[0], lo, rtol=1e-4)
    assert np.abs(g[0] - go).max() < 2e-3 * np.abs(go).max()
    f = eng.mlp_forward(p0[0], x)[:, 0]
    np.testing.assert_allclose(f, ora.forward(p0[0].astype(np.float64), x, 1, 1)[:, 0], rtol=1e-5)


def test_batched_training_equals_single_and_learns(eng):
    data = [_data(s) for s in (2, 3, 4)]
    p0, l0, _ = eng.mlp_train(data, epochs=0)            # initial parameters and loss
    pb, lb, _ = eng.mlp_train(data, epochs=1500, params=p0)
    for k, d in enumerate(data):
        p1, l1, _ = eng.mlp_train([d], epochs=1500, params=p0[k:k + 1])
        np.testing.assert_array_equal(pb[k], p1[0])      # deterministic, block-independent
        assert l1[0] == lb[k] and l1[0] < 0.05 * l0[k]


def test_network_weight_drives_the_force_scaling(eng):
    """A network that outputs 1.5 everywhere must give exactly the trajectory of the
    degree-0 polynomial weight 1.5 (same scale in double precision)."""
    top = dict(systems.solvated_polymer(20, 1500, seed=7))
    e0 = oracle.Oracle(top, method=abi.JP_METHOD_MICR).energy_grad()[0][0]
    const = dict(coef=np.array([[1.5]]), low=np.array([0.0]), high=np.array([1.0 + 1e-12]),
                 alphalw=1.5, alphaup=1.5, celw=e0 - 3000.0, ceup=e0 + 500.0, tempce=300.0)
    top["ge"] = const
    net = np.zeros(eng.mlp_nparam(1, 1), np.float32)
    L = ora.layout(1, 1)
    net[L["xs"][0]] = 1.0
    net[L["yo"][0]] = 1.5
    net[L["ys"][0]] = 1.0
    with eng.Engine(top, precision=abi.JP_PREC_MIXED, method=abi.JP_METHOD_GE) as e:
        e.step(1)
        e.set_state(0, top["cord"], top["vel"])
        e.rebuild()
        e.ge_set_mlp(net)
        pre = e.launch_counts()[0]
        e.step(11)
        x_net, _ = e.get_state()
    with eng.Engine(top, precision=abi.JP_PREC_MIXED, method=abi.JP_METHOD_GE) as e:
        e.step(1)
        e.set_state(0, top["cord"], top["vel"])
        e.rebuild()
        e.step(11)
        x_ref, _ = e.get_state()
    np.testing.assert_array_equal(x_net, x_ref)
    assert pre >= 4   # k_ge_scale joined the step


def _law(x):
    """Temperature rising steeply from 280 K to 700 K across the middle of the range (a
    transition): d lnN/dE = 1/(R T) is a sigmoid a degree-8 polynomial cannot follow."""
    return 280.0 + 420.0 / (1.0 + np.exp(-(np.clip(x, 0.0, 1.0) - 0.5) / 0.04))


def _histogram(old, emin, emax, nbin, nbor):
    """Expected counts of a McMD run sampled with `old` on the density of states of _law."""
    de = (emax - emin) / nbin
    e = emin - de * nbor + de * (np.arange(nbin + 2 * nbor) + 0.5)
    fine = np.linspace(e[0], e[-1], 40001)
    dlnn = 1.0 / (R_KCAL * _law((fine - emin) / (emax - emin)))
    xo = np.clip((fine - old["celw"]) / (old["ceup"] - old["celw"]), 0.0, 1.0)
    dw = ge.poly_values(old, xo)
    g = np.concatenate([[0.0], np.cumsum(0.5 * (dlnn[1:] + dlnn[:-1] - dw[1:] - dw[:-1]) * np.diff(fine))])
    lnp = np.interp(e, fine, g)
    p = np.exp(lnp - lnp.max())
    return np.round(2.0e6 * p / p.sum())


def test_network_gains_over_polynomial_on_a_transition(eng):
    """The run used the best degree-8 polynomial of the true law (the previous iteration's
    weight); refitting the polynomial cannot get closer, the network can, and the flatness it
    predicts for the next run is higher, so the iteration takes it."""
    emin, emax, nbin, nbor = -300.0, 300.0, 150, 0
    xg = np.linspace(0.0, 1.0, 401)
    c8 = np.polynomial.polynomial.polyfit(xg, 1.0 / (R_KCAL * _law(xg)), 8)
    old = dict(coef=c8.reshape(1, -1), low=np.array([0.0]), high=np.array([1.0 + 1e-12]),
               alphalw=1.0 / (R_KCAL * 280.0), alphaup=1.0 / (R_KCAL * 700.0), celw=emin,
               ceup=emax, tempce=300.0)
    hist = _histogram(old, emin, emax, nbin, nbor)
    out = ge.iterate(hist, old, emin, emax, nbin, nbor, emin, emax, 300.0, nwindow=1, ndeg=8,
                     epochs=6000)
    x, y, w = out["data"]
    m = w > 0
    truth = 1.0 / (R_KCAL * _law(x[m]))
    f_poly = ge.poly_values(out["poly"], x[m])
    f_mlp = eng.mlp_forward(out["mlp"], x[m])[:, 0]
    err_poly = np.sqrt((w[m] * (truth - f_poly) ** 2).sum() / w[m].sum())
    err_mlp = np.sqrt((w[m] * (truth - f_mlp) ** 2).sum() / w[m].sum())
    assert m.sum() > 100
    assert err_mlp < 0.3 * err_poly
    assert out["flat_mlp"] > out["flat_poly"] and out["use_mlp"]
