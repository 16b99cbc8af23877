"""TEST INFRASTRUCTURE ONLY: float64 numpy restatement of the weight surrogate network
(layout and loss as documented for jp_mlp_train in include/jpgpu.h and csrc/jp_mlp.cuh).

Checks the GPU forward pass, the GPU gradient (jp_mlp_train with epochs = 0) and itself
against finite differences; the product never imports it.
"""
import numpy as np

H = 64


def layout(nin, nout):
    o = {}
    n = 0
    for name, size in (("w1", H * nin), ("b1", H), ("w2", H * H), ("b2", H), ("w3", nout * H),
                       ("b3", nout), ("xo", nin), ("xs", nin), ("yo", nout), ("ys", nout)):
        o[name] = (n, n + size)
        n += size
    o["n"] = n
    return o


def unpack(p, nin, nout):
    L = layout(nin, nout)
    g = {k: np.asarray(p[v[0]:v[1]], np.float64) for k, v in L.items() if k != "n"}
    g["w1"] = g["w1"].reshape(H, nin)
    g["w2"] = g["w2"].reshape(H, H)
    g["w3"] = g["w3"].reshape(nout, H)
    return g


def forward(p, x, nin, nout):
    """y[n][nout] = yo + ys * net((x - xo) * xs)."""
    g = unpack(p, nin, nout)
    xn = (np.asarray(x, np.float64).reshape(-1, nin) - g["xo"]) * g["xs"]
    h1 = np.tanh(xn @ g["w1"].T + g["b1"])
    h2 = np.tanh(h1 @ g["w2"].T + g["b2"])
    o = h2 @ g["w3"].T + g["b3"]
    return g["yo"] + g["ys"] * o


def loss_grad(p, x, y, w, nin, nout):
    """Weighted MSE of the normalised targets and its gradient (normalisation entries 0)."""
    g = unpack(p, nin, nout)
    L = layout(nin, nout)
    x = np.asarray(x, np.float64).reshape(-1, nin)
    y = np.asarray(y, np.float64).reshape(-1, nout)
    w = np.asarray(w, np.float64).reshape(-1)
    xn = (x - g["xo"]) * g["xs"]
    h1 = np.tanh(xn @ g["w1"].T + g["b1"])
    h2 = np.tanh(h1 @ g["w2"].T + g["b2"])
    o = h2 @ g["w3"].T + g["b3"]
    e = o - (y - g["yo"]) / g["ys"]
    isw = 1.0 / w.sum()
    loss = float((w[:, None] * e * e).sum() * isw)
    g3 = 2.0 * w[:, None] * e * isw
    d2 = (g3 @ g["w3"]) * (1.0 - h2 * h2)
    d1 = (d2 @ g["w2"]) * (1.0 - h1 * h1)
    grad = np.zeros(L["n"])
    grad[slice(*L["w1"])] = (d1.T @ xn).reshape(-1)
    grad[slice(*L["b1"])] = d1.sum(0)
    grad[slice(*L["w2"])] = (d2.T @ h1).reshape(-1)
    grad[slice(*L["b2"])] = d2.sum(0)
    grad[slice(*L["w3"])] = (g3.T @ h2).reshape(-1)
    grad[slice(*L["b3"])] = g3.sum(0)
    return loss, grad
