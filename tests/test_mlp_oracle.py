"""The float64 network oracle against central finite differences, and the predicted-flatness
measure of the McMD iteration policy (no GPU)."""
import numpy as np

from oracle import mlp as ora
from j_presto_b200 import ge


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    nin, nout = 2, 2
    L = ora.layout(nin, nout)
    p = rng.normal(0.0, 0.2, L["n"])
    p[slice(*L["xo"])] = [0.5, 0.7]
    p[slice(*L["xs"])] = [2.0, 1.5]
    p[slice(*L["yo"])] = [0.3, -0.1]
    p[slice(*L["ys"])] = [1.2, 0.8]
    x = rng.uniform(0.0, 1.0, (40, nin))
    y = np.stack([np.sin(3 * x[:, 0]), x[:, 0] * x[:, 1]], 1)
    w = rng.uniform(0.5, 2.0, 40)
    loss, grad = ora.loss_grad(p, x, y, w, nin, nout)
    for q in list(range(0, L["xo"][0], 97)) + [L["b3"][0], L["w3"][0] + 5]:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[q] += h
        pm[q] -= h
        fd = (ora.loss_grad(pp, x, y, w, nin, nout)[0] - ora.loss_grad(pm, x, y, w, nin, nout)[0]) / (2 * h)
        assert abs(fd - grad[q]) < 1e-7 + 1e-5 * abs(fd)
    assert not grad[L["xo"][0]:].any()


def test_predicted_flatness():
    x = np.linspace(0.0, 1.0, 50)
    y = 1.0 + x
    w = np.ones(50)
    assert abs(ge.predicted_flatness(x, y, w, y, 100.0) - 100.0) < 1e-9   # exact weight: flat
    assert ge.predicted_flatness(x, y, w, y + 0.05, 100.0) < 50.0          # biased weight
