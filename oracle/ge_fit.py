"""TEST INFRASTRUCTURE ONLY: numpy restatement of one GEprep McMD weight iteration.

Used by tests/ as the checker of the library's host fit (jp_ge_fit / jp_lstsq_windows); the
product never imports it.  Written 1-based, line for line after the reference so that it
can be read beside it:
  minver            src_GEprep/minver.f90:1-80
  lstsquare_final   src_GEprep/lstsquare_final.f90:1-253
  dlnn_data         src_GEprep/distrib_MULT.f90:60-68, 286-296, 322-420
  ge_fit            src_GEprep/distrib_MULT.f90:422-445
Parity against the reference itself is unpinned (Fortran, no compiler here); the tests pin
this restatement with closed-form cases (exact polynomials, converged flat histograms).
"""
import numpy as np


def ipow(x, j):
    """x**j for integer j >= 0 as j-1 successive products (Fortran's integer power)."""
    r = 1.0
    for _ in range(j):
        r *= x
    return r


def matvec(A, b):
    """A @ b summed in column order (Fortran matmul loop), no BLAS reordering."""
    out = np.zeros(A.shape[0])
    for i in range(A.shape[0]):
        s = 0.0
        for j in range(A.shape[1]):
            s += A[i, j] * b[j]
        out[i] = s
    return out


def minver(a):
    """Gauss-Jordan inverse with partial pivoting, pivots <= 1e-12 zero their row/column."""
    m = a.shape[0]
    A = np.zeros((m + 1, m + 1))
    A[1:, 1:] = a
    eps = 1.0e-12
    iwork = list(range(m + 1))
    for k in range(1, m + 1):
        wmax, lr = 0.0, k
        for i in range(k, m + 1):
            w = abs(A[i, k])
            if w > wmax:
                wmax, lr = w, i
        pivot = A[lr, k]
        api = abs(pivot)
        if lr != k:
            iwork[k], iwork[lr] = iwork[lr], iwork[k]
            A[[k, lr], 1:] = A[[lr, k], 1:]
        if api > eps:
            A[k, 1:] = A[k, 1:] / pivot
            for i in range(1, m + 1):
                if i != k:
                    w = A[i, k]
                    if w != 0.0:
                        for j in range(1, m + 1):
                            if j != k:
                                A[i, j] = A[i, j] - w * A[k, j]
                        A[i, k] = -w / pivot
            A[k, k] = 1.0 / pivot
        else:
            A[k, 1:] = 0.0
            A[1:, k] = 0.0
    for i in range(1, m + 1):
        while iwork[i] != i:
            k = iwork[i]
            iwork[k], iwork[i] = iwork[i], iwork[k]
            A[1:, [i, k]] = A[1:, [k, i]]
    return A[1:, 1:]


def _sums(X, Y, wei, imn, imx, x0, ndim):
    xs = np.zeros(2 * ndim + 1)
    xys = np.zeros(ndim + 1)
    swei = 1.0 / sum(wei[i] for i in range(imn, imx + 1))
    for i in range(imn, imx + 1):
        dx = X[i] - x0
        for j in range(1, 2 * ndim + 1):
            xs[j] += ipow(dx, j) * wei[i]
        for j in range(0, ndim + 1):
            xys[j] += Y[i] * ipow(dx, j) * wei[i]
    xs[1:] *= swei
    xys *= swei
    return xs, xys, swei


def lstsquare_final(nwindow, ndim, minv, maxv, x, y, w):
    """Returns coe[nwindow][ndim+1], low[nwindow], high[nwindow], (resierr, resierr2)."""
    ndat = len(x)
    X = np.concatenate([[0.0], x]); Y = np.concatenate([[0.0], y]); wei = np.concatenate([[0.0], w])
    COE = np.zeros((ndim + 1, nwindow + 1))
    low = np.zeros(nwindow + 1); high = np.zeros(nwindow + 1)
    nmx = [ndat] * (nwindow + 1)
    rrange = (maxv - minv) / nwindow
    rtmp = rrange + minv
    j = 1
    rtmp2 = rrange * 0.00001
    low[1] = minv
    for i in range(1, ndat + 1):
        if rtmp - X[i] < rtmp2:
            high[j] = X[i]
            nmx[j] = i
            j += 1
            rtmp = rrange * j + minv
            if j == nwindow + 1:
                break
            low[j] = X[i]
    high[nwindow] = maxv
    nmx[nwindow] = ndat
    itole = ndat // (2 * nwindow)
    ndw = np.zeros(nwindow + 1)
    k = 1
    for i in range(1, nwindow + 1):
        for jj in range(k, nmx[i] + 1):
            ndw[i] += wei[jj] * wei[jj]
        k = nmx[i] + 1
    maxw = 1
    for i in range(2, nwindow + 1):
        if ndw[i] > ndw[maxw]:
            maxw = i
    ii = nmx[maxw - 1] if maxw != 1 else 1
    imn, imx = max(1, ii - itole), min(nmx[maxw] + itole, ndat)
    xs, xys, _ = _sums(X, Y, wei, imn, imx, low[maxw], ndim)
    A = np.array([[xs[i + j] - xs[i] * xs[j] for j in range(1, ndim + 1)] for i in range(1, ndim + 1)])
    B = np.array([xys[i] - xys[0] * xs[i] for i in range(1, ndim + 1)])
    C = matvec(minver(A), B)
    dot = 0.0
    for a in range(ndim):
        dot += C[a] * xs[a + 1]
    COE[0, maxw] = -dot + xys[0]
    COE[1:, maxw] = C
    for i in range(maxw + 1, nwindow + 1):
        p = i - 1
        dx = high[p] - low[p]
        COE[0, i] = COE[0, p]
        for jj in range(1, ndim + 1):
            COE[0, i] += COE[jj, p] * ipow(dx, jj)
        COE[1, i] = COE[1, p]
        for jj in range(2, ndim + 1):
            COE[1, i] += jj * COE[jj, p] * ipow(dx, jj - 1)
        imn, imx = max(1, nmx[i - 1] - itole), min(nmx[i] + itole, ndat)
        xs, xys, _ = _sums(X, Y, wei, imn, imx, low[i], ndim)
        if ndim >= 2:
            A = np.array([[xs[a + b] for b in range(2, ndim + 1)] for a in range(2, ndim + 1)])
            B = np.array([xys[a] - COE[0, i] * xs[a] - COE[1, i] * xs[a + 1] for a in range(2, ndim + 1)])
            COE[2:, i] = matvec(minver(A), B)
    for i in range(maxw - 1, 0, -1):
        ii = nmx[i - 1] if i != 1 else 1
        imn, imx = max(1, ii - itole), min(nmx[i] + itole, ndat)
        xs, xys, swei = _sums(X, Y, wei, imn, imx, low[i], ndim)
        xs[0] = 1.0
        nu = i + 1
        dx = high[i] - low[i]
        m = ndim + 3
        Ac = np.zeros((m, m))
        for a in range(ndim + 1):
            for b in range(ndim + 1):
                Ac[a, b] = xs[a + b]
            Ac[a, ndim + 1] = -ipow(dx, a) * swei * 0.5
            Ac[ndim + 1, a] = ipow(dx, a)
        for a in range(1, ndim + 1):
            Ac[a, ndim + 2] = -(a * ipow(dx, a - 1)) * swei * 0.5
            Ac[ndim + 2, a] = a * ipow(dx, a - 1)
        Bc = np.concatenate([xys, [COE[0, nu], COE[1, nu]]])
        COE[:, i] = matvec(minver(Ac), Bc)[:ndim + 1]
    r1 = r2 = 0.0

    def acc(i, wdw):
        nonlocal r1, r2
        dxx = X[i] - low[wdw]
        ex = 0.0
        for a in range(ndim + 1):
            ex += COE[a, wdw] * ipow(dxx, a)
        ex = Y[i] - ex
        ex2 = ex * ex
        ex = ex2 * wei[i]
        ex2 = ex * ex2
        r1 += ex
        r2 += ex2
    for i in range(1, nmx[1] + 1):
        acc(i, 1)
    if nwindow > 1:
        for i in range(nmx[nwindow - 1] + 1, ndat + 1):
            acc(i, nwindow)
        for wdw in range(2, nwindow):
            for i in range(nmx[wdw - 1] + 1, nmx[wdw] + 1):
                acc(i, wdw)
    sw = 0.0
    for i in range(1, ndat + 1):
        sw += wei[i]
    swei = 1.0 / sw
    r1 *= swei
    r2 = np.sqrt(r2 * swei)
    res2 = np.sqrt(r2 - r1) if r2 >= r1 else float("nan")
    return COE[:, 1:].T.copy(), low[1:].copy(), high[1:].copy(), (np.sqrt(r1), res2)


def poly_old(nf, xs):
    """d lnN/dE of a weight at reduced energy xs (rr/ss outside [0, 1])."""
    if xs < 0.0:
        return nf["alphalw"]
    if xs > 1.0:
        return nf["alphaup"]
    nw = len(nf["low"])
    j = 0
    while j != nw - 1 and xs >= nf["high"][j]:
        j += 1
    dx = xs - nf["low"][j]
    p = nf["coef"][j][0]
    for k in range(1, len(nf["coef"][j])):
        p += nf["coef"][j][k] * ipow(dx, k)
    return p


def dlnn_data(hist, old, emin, emax, nbin, nbor, next_emin, next_emax, ignore_empty=True,
              neglect_low=False, neglect_high=False):
    """(X, Y, W) handed to the fit by distrib_MULT."""
    nab = nbin + 2 * nbor
    de = (emax - emin) / nbin
    minec = emin - de * nbor
    P = np.concatenate([[0.0], np.asarray(hist, float)])
    EE = np.array([0.0] + [minec + de * (i - 1 + 0.5) for i in range(1, nab + 1)])
    lmax = np.log(P[1:].max())
    lnP = np.array([0.0] + [1.0 if P[i] == 0.0 else np.log(P[i]) - lmax for i in range(1, nab + 1)])
    dlnN = np.zeros(nab + 1)
    # the old weight's window pointer runs monotonically, as in the reference loop
    j = 0
    nw = len(old["low"])
    for i in range(1, nab):
        xs = (EE[i] + 0.5 * de - old["celw"]) / (old["ceup"] - old["celw"])
        if xs < 0.0:
            p = old["alphalw"]
        elif xs > 1.0:
            p = old["alphaup"]
        else:
            while j != nw - 1 and xs >= old["high"][j]:
                j += 1
            dx = xs - old["low"][j]
            p = old["coef"][j][0]
            for k in range(1, len(old["coef"][j])):
                p += old["coef"][j][k] * ipow(dx, k)
        if lnP[i] != 1.0 and lnP[i + 1] != 1.0:
            dlnN[i] = (lnP[i + 1] - lnP[i]) / de + p
        else:
            dlnN[i] = p if 0.0 <= xs <= 1.0 else 0.0
    ist = nbor + 1 if neglect_low else 1
    ien = nbor + nbin if neglect_high else nab - 1
    X, Y, W = [], [], []
    for i in range(ist, ien + 1):
        x2 = (EE[i] + 0.5 * de - next_emin) / (next_emax - next_emin)
        if ignore_empty:
            if dlnN[i] == 0.0:
                continue
            W.append(np.sqrt(P[i] + P[i + 1]))
        else:
            if dlnN[i] == 0.0 and (x2 < old["celw"] or x2 > old["ceup"]):
                continue
            W.append(max(np.sqrt(P[i] + P[i + 1]), 1.0))
        X.append(x2)
        Y.append(dlnN[i])
    return np.array(X), np.array(Y), np.array(W)


def ge_fit(hist, old, emin, emax, nbin, nbor, next_emin, next_emax, next_temp, nwindow, ndeg,
           **kw):
    X, Y, W = dlnn_data(hist, old, emin, emax, nbin, nbor, next_emin, next_emax, **kw)
    coe, low, high, res = lstsquare_final(nwindow, ndeg, 0.0, 1.0, X, Y, W)
    upd = coe[-1, 0]
    for k in range(1, ndeg + 1):
        upd += coe[-1, k] * ipow(1.0 - low[-1], k)
    nf = dict(coef=coe, low=low, high=high, alphalw=coe[0, 0], alphaup=upd, celw=next_emin,
              ceup=next_emax, tempce=next_temp, lower=old.get("lower", 0.0),
              upper=old.get("upper", 0.0))
    return nf, res
