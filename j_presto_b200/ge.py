"""One McMD weight iteration with the surrogate network as a candidate.

GEprep fits d lnN/dE by windowed polynomials (jp_ge_fit).  Here the same data also trains a
64-64 tanh network on the GPU (jp_mlp_train); the polynomial remains the fallback and the
yardstick: the network is taken only if the flatness it predicts for the next run is no worse
than the polynomial's.

Predicted flatness.  With the data's d lnN/dE estimate y(x) and a candidate weight f(x), a
run with that weight samples ln P(x) = integral of (y - f) dE, so its histogram over the
data points is exp(ln P - max ln P); flatness is its mean in percent, the measure GEprep's
distrib_MULT reports (distrib_MULT.f90:298-302).
"""
import numpy as np

from . import engine


def write_nf(path, nf, alsd=False):
    """The weight as md_run reads it (inmcmd.f90:21-38, list-directed, one READ per line):
    nwindow ndeg / c(0..ndeg) of each window one per line, then its low high / alphalw
    alphaup / celw ceup / tempce / with ALSD (CLSTMETHOD= LMD*) the walls lower upper."""
    coef = np.atleast_2d(np.asarray(nf["coef"], np.float64))
    nwin, ndeg = coef.shape[0], coef.shape[1] - 1
    lines = [f"{nwin} {ndeg}"]
    for w in range(nwin):
        lines += [repr(float(v)) for v in coef[w]]
        lines.append(f"{float(nf['low'][w])!r} {float(nf['high'][w])!r}")
    lines.append(f"{float(nf['alphalw'])!r} {float(nf['alphaup'])!r}")
    lines.append(f"{float(nf['celw'])!r} {float(nf['ceup'])!r}")
    lines.append(repr(float(nf["tempce"])))
    if alsd:
        lines.append(f"{float(nf.get('lower', 0.0))!r} {float(nf.get('upper', 0.0))!r}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_nf(path, alsd=False):
    """A weight file as inmcmd.f90 reads it: each READ takes the first values of the next
    line (Fortran D exponents accepted); the dict has the keys jp_ge takes."""
    with open(path) as f:
        recs = [ln.replace("D", "E").replace("d", "e").replace(",", " ").split()
                for ln in f if ln.strip()]
    it = iter(recs)
    head = next(it)
    nwin, ndeg = int(head[0]), int(head[1])
    coef = np.zeros((nwin, ndeg + 1))
    low, high = np.zeros(nwin), np.zeros(nwin)
    for w in range(nwin):
        for j in range(ndeg + 1):
            coef[w, j] = float(next(it)[0])
        r = next(it)
        low[w], high[w] = float(r[0]), float(r[1])
    a = next(it)
    c = next(it)
    t = next(it)
    nf = dict(coef=coef, low=low, high=high, alphalw=float(a[0]), alphaup=float(a[1]),
              celw=float(c[0]), ceup=float(c[1]), tempce=float(t[0]))
    if alsd:
        wl = next(it)
        nf["lower"], nf["upper"] = float(wl[0]), float(wl[1])
    return nf


def predicted_flatness(x, y, w, f, e_span):
    """Flatness (percent) of the next run's histogram over the sampled points (w > 0,
    0 <= x <= 1) if it ran with weight values f at x.  e_span = ceup - celw."""
    m = (w > 0.0) & (x >= 0.0) & (x <= 1.0)
    xs, d = x[m], (y - f)[m]
    if len(xs) < 2:
        return 0.0
    lnp = np.concatenate([[0.0], np.cumsum(0.5 * (d[1:] + d[:-1]) * np.diff(xs) * e_span)])
    return float(np.exp(lnp - lnp.max()).mean() * 100.0)


def poly_values(nf, x):
    out = np.empty(len(x))
    for n, xv in enumerate(x):
        j = 0
        while j != len(nf["low"]) - 1 and xv >= nf["high"][j]:
            j += 1
        out[n] = np.polynomial.polynomial.polyval(xv - nf["low"][j], nf["coef"][j])
    return out


def iterate(hist, old_nf, emin, emax, nbin, nbor, next_emin, next_emax, next_temp, nwindow=1,
            ndeg=8, epochs=3000, lr=1e-3, seed=1, device=0, **kw):
    """Polynomial fit and network of the next McMD weight; returns a dict with both, their
    predicted flatness and `use_mlp` (the network wins only if it is no worse)."""
    nf, resid = engine.ge_fit(hist, old_nf, emin, emax, nbin, nbor, next_emin, next_emax,
                              next_temp, nwindow, ndeg, **kw)
    x, y, w = engine.ge_dlnn(hist, old_nf, emin, emax, nbin, nbor, next_emin, next_emax, **kw)
    keep = w > 0.0
    params, loss, _ = engine.mlp_train([(x[keep], y[keep], w[keep])], epochs=epochs, lr=lr,
                                       seed=seed, device=device)
    span = next_emax - next_emin
    f_poly = poly_values(nf, x)
    f_mlp = engine.mlp_forward(params[0], x, device=device)[:, 0].astype(np.float64)
    flat_poly = predicted_flatness(x, y, w, f_poly, span)
    flat_mlp = predicted_flatness(x, y, w, f_mlp, span)
    return dict(poly=nf, poly_resid=resid, mlp=params[0], mlp_loss=float(loss[0]),
                flat_poly=flat_poly, flat_mlp=flat_mlp, use_mlp=flat_mlp >= flat_poly,
                data=(x, y, w))
