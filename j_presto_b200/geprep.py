"""GEprep's McMD distribution step (src_GEprep/distrib_MULT.f90) on energy histograms.

The reference's GEprep reads the `.ene` files of a set of McMD runs, bins their energies,
and writes: the distribution (`.dist`), the bar graph of each set's sampled range (`.bar`),
the new weight (`.nf`), d lnN/dE with its fit (`.dlnN`), the temperature at each energy
(`.et`), the specific heat (`.sph`), the canonical distribution and probability at a
temperature (`_T.cdist`, `_T.prob`) and the per-bin count of sets reaching ln P >= 0,
-1.5, -0.5 (`.TTPdist`), and prints the flatness.  Here the histograms come from the
engine (jp_ge_hist_get: one per replica, distrib_MULT's binning) and the same quantities are
computed and written in the reference's layout:

* runs are grouped in sets (`sets`, a run's set index; default one set per run) and each
  run has a weight fw (default 1): trP = sum over the set's runs of counts, tP = sum of
  fw * counts; with flatness acceleration (accele) tP is divided by the set's flatness to
  the power accrat before it enters P (distrib_MULT.f90:80-210);
* rlnP = ln(rP / max rP), lnP = ln(P / max P), 1.0 marking an empty bin as the reference
  does; flatness = 100 * sum over the nBIN inner bins of exp(ln P) / nBIN (:216-247);
* d lnN/dE = d lnP/dE + the old weight's d lnN/dE, by forward differences between bins
  (:322-370), accelerated by accrt2 inside the old range when accel2 is set;
* the fit points are the reduced energies of the next range with weights sqrt(P_i + P_i+1)
  (:380-420) and the fit is lstsquare_final (engine.lstsq_windows, jp_lstsq_windows).
With one run, fw = 1 and no acceleration this is exactly what jp_ge_fit computes.
"""
import numpy as np

from . import engine

R_GAS = 8.31451 / 4184.0   # kcal/mol/K (GEprep's R)
EMPTY = 1.0                # ln P marker of an empty bin (distrib_MULT.f90:214, :222)


def bin_centres(emin, emax, nbin, nbor):
    """EE(i) = minEc + EbinSZ (i - 1/2), minEc = minE - EbinSZ nBOR (distrib_MULT.f90:58-63)."""
    de = (emax - emin) / nbin
    nab = nbin + 2 * nbor
    return emin - de * nbor + de * (np.arange(nab) + 0.5), de


def _lnp(p):
    out = np.full(len(p), EMPTY)
    nz = p != 0.0
    if nz.any():
        out[nz] = np.log(p[nz]) - np.log(p.max())
    return out


def _flatness(lnp, nbor, nbin):
    inner = lnp[nbor:nbor + nbin]
    return float(np.exp(inner[inner != EMPTY]).sum() / nbin * 100.0)


def distribution(counts, emin, emax, nbin, nbor, fw=None, sets=None, accele=False, accrat=1.0):
    """The distribution of a group of runs.  counts [nrun][nBIN + 2 nBOR] histogram counts;
    fw [nrun] run weights; sets [nrun] set index of each run (runs of a set contiguous).
    Returns a dict with EE, rP, P, rlnP, lnP, the overall flatness (rlnP; `flat_acc` from
    lnP), per-set flatness `flt`, per-set energy ranges `erange` [nset][2], the `.bar` rows,
    TTPdist [nAB][3], and the counts inside [minE, maxE] against all counts."""
    counts = np.atleast_2d(np.asarray(counts, np.float64))
    nrun, nab = counts.shape
    assert nab == nbin + 2 * nbor
    fw = np.ones(nrun) if fw is None else np.asarray(fw, np.float64)
    sets = np.arange(nrun) if sets is None else np.asarray(sets)
    EE, de = bin_centres(emin, emax, nbin, nbor)
    rP, P = np.zeros(nab), np.zeros(nab)
    flt, erange, bar = [], [], []
    ttp = np.zeros((nab, 3), np.int64)
    for s in np.unique(sets):
        runs = np.flatnonzero(sets == s)
        trP = counts[runs].sum(axis=0)
        tP = (counts[runs] * fw[runs, None]).sum(axis=0)
        rP += trP
        if trP.max() == 0.0:
            continue
        tlnp = _lnp(trP)
        f = _flatness(tlnp, nbor, nbin)
        flt.append(f if f != 0.0 else 0.01)
        ttp[:, 0] += tlnp <= 0.0
        ttp[:, 1] += (tlnp <= 0.0) & (tlnp >= -1.5)
        ttp[:, 2] += (tlnp <= 0.0) & (tlnp >= -0.5)
        if accele:
            tP = tP / flt[-1] ** accrat
        P += tP
        occ = np.flatnonzero(tlnp != EMPTY)
        i1, il = occ[0], occ[-1]
        i2 = i1 + np.flatnonzero(tlnp[i1:] >= -1.5)[0]
        l2 = np.flatnonzero(tlnp[:il + 1] >= -1.5)[-1]
        bar.append((EE[i1], len(flt), EE[i2]))
        bar.append((EE[il], len(flt), EE[l2]))
        erange.append((EE[il] - EE[i1] + de, EE[l2] - EE[i2] + de))
    rlnP, lnP = _lnp(rP), _lnp(P)
    inside = counts[:, nbor:nbor + nbin].sum()
    return dict(EE=EE, de=de, emin=emin, emax=emax, nbin=nbin, nbor=nbor, rP=rP, P=P, rlnP=rlnP,
                lnP=lnP, flat=_flatness(rlnP, nbor, nbin), flat_acc=_flatness(lnP, nbor, nbin),
                flt=np.array(flt), erange=np.array(erange), bar=bar, ttpdist=ttp,
                counted=(float(inside), float(counts.sum())), fwflg=bool(accele or (fw != 1.0).any()))


def _poly(nf, xs):
    """A windowed weight polynomial at reduced energy xs, summed as the reference sums it:
    c0 + c1 dx + c2 dx^2 + ..., dx^k as k - 1 successive products."""
    j = 0
    nw = len(nf["low"])
    while j != nw - 1 and xs >= nf["high"][j]:
        j += 1
    c = nf["coef"][j]
    dx = xs - nf["low"][j]
    p = float(c[0])
    pw = 1.0
    for k in range(1, len(c)):
        pw = pw * dx if k > 1 else dx
        p += float(c[k]) * pw
    return p


def dlnn(dist, old, accel2=False, accrt2=1.0):
    """rdlnN (from rlnP) and dlnN (from lnP) at the nBIN + 2 nBOR - 1 bin boundaries:
    forward differences plus the old weight's d lnN/dE (alphalw / alphaup outside its range);
    0 where a bin is empty outside the old range (distrib_MULT.f90:322-370)."""
    EE, de, lnP, rlnP = dist["EE"], dist["de"], dist["lnP"], dist["rlnP"]
    nab = len(EE)
    rd, d = np.zeros(nab - 1), np.zeros(nab - 1)
    for i in range(nab - 1):
        xs = (EE[i] + 0.5 * de - old["celw"]) / (old["ceup"] - old["celw"])
        if xs < 0.0:
            p = old["alphalw"]
        elif xs > 1.0:
            p = old["alphaup"]
        else:
            p = _poly(old, xs)
        if lnP[i] != EMPTY and lnP[i + 1] != EMPTY:
            rd[i] = (rlnP[i + 1] - rlnP[i]) / de + p
            a = accrt2 if (accel2 and 0.0 <= xs <= 1.0) else 1.0
            d[i] = a * (lnP[i + 1] - lnP[i]) / de + p
        elif 0.0 <= xs <= 1.0:
            rd[i] = d[i] = p
    return rd, d


def fit_data(dist, d, old, next_emin, next_emax, ignore_empty=True, neglect_low=False,
             neglect_high=False):
    """The points lstsquare_final fits (distrib_MULT.f90:380-420): reduced energies of the
    next range, d lnN/dE, weights sqrt(P_i + P_i+1) (at least 1 without igndat)."""
    EE, de, P = dist["EE"], dist["de"], dist["P"]
    nbin, nbor = dist["nbin"], dist["nbor"]
    nab = len(EE)
    ist = nbor if neglect_low else 0
    ien = nbor + nbin - 1 if neglect_high else nab - 2
    X, Y, W = [], [], []
    for i in range(ist, ien + 1):
        x2 = (EE[i] + 0.5 * de - next_emin) / (next_emax - next_emin)
        if ignore_empty:
            if d[i] == 0.0:
                continue
            W.append(np.sqrt(P[i] + P[i + 1]))
        else:
            if d[i] == 0.0 and (x2 < old["celw"] or x2 > old["ceup"]):
                continue
            W.append(max(np.sqrt(P[i] + P[i + 1]), 1.0))
        X.append(x2)
        Y.append(d[i])
    return np.array(X), np.array(Y), np.array(W)


def fit(X, Y, W, next_emin, next_emax, next_temp, nwindow, ndeg, old=None):
    """lstsquare_final over [0, 1] and the .nf record (distrib_MULT.f90:422-445)."""
    coef, low, high, resid = engine.lstsq_windows(X, Y, W, nwindow, ndeg)
    lowd = coef[0, 0]
    upd = _poly(dict(coef=coef[-1:], low=low[-1:], high=high[-1:]), 1.0)
    old = old or {}
    nf = dict(coef=coef, low=low, high=high, alphalw=lowd, alphaup=upd, celw=next_emin,
              ceup=next_emax, tempce=next_temp, lower=old.get("lower", 0.0), upper=old.get("upper", 0.0))
    return nf, resid


def temperatures(dist, nf):
    """The `.et` table: (E, 1 / (R d lnN/dE)) at minE, at each inner bin centre and at maxE
    (distrib_MULT.f90:615-665), and the `.sph` pairs (T step / 2, EbinSZ / T step)."""
    EE, nbin, nbor = dist["EE"], dist["nbin"], dist["nbor"]
    span = nf["ceup"] - nf["celw"]
    rows = [(dist["emin"], 1.0 / (_poly(nf, (dist["emin"] - nf["celw"]) / span) * R_GAS))]
    TT = np.zeros(len(EE))
    for i in range(nbor, nbor + nbin):
        TT[i] = 1.0 / (_poly(nf, (EE[i] - nf["celw"]) / span) * R_GAS)
        rows.append((EE[i], TT[i]))
    rows.append((dist["emax"], 1.0 / (_poly(nf, (dist["emax"] - nf["celw"]) / span) * R_GAS)))
    sph = [(0.5 * (TT[i] - TT[i - 1]), dist["de"] / (TT[i] - TT[i - 1])) for i in range(nbor + 1, nbor + nbin)]
    return rows, sph


def canonical(dist, nf, temp):
    """ln Pc(E) = ln N(E) - E / (R T) on nBIN bins spanning where the first pass has
    ln Pc >= -7 (distrib_MULT.f90:503-560): (E, ln Pc) rows and the `.prob` header."""
    EE, de, rlnP, nbin = dist["EE"], dist["de"], dist["rlnP"], dist["nbin"]
    span = nf["ceup"] - nf["celw"]
    beta = 1.0 / (R_GAS * temp)
    lnpc = np.zeros(len(EE))
    acc = 0.0
    occ = rlnP != EMPTY
    for i in range(len(EE)):
        if occ[i]:
            acc += _poly(nf, (EE[i] - nf["celw"]) / span) * de
            lnpc[i] = acc - EE[i] * beta
    lnpc[occ] -= lnpc[occ].max()
    keep = np.flatnonzero(occ & (lnpc >= -7.0))
    lo, hi = keep[0], keep[-1]
    ebin = (EE[hi] - EE[lo] + de) / nbin
    emin_c = EE[lo] - 0.5 * ebin
    ee = emin_c + ebin * (np.arange(nbin) + 0.5)
    out = np.zeros(nbin)
    acc = 0.0
    for i in range(nbin):
        acc += _poly(nf, (ee[i] - nf["celw"]) / span) * ebin
        out[i] = acc - ee[i] * beta
    out -= out.max()
    return ee, out, (nbin, ebin, emin_c)


# ---- files in the reference's layout (list-directed numbers, one record per line) --------
def _rows(path, rows, fmt=None):
    with open(path, "w") as f:
        for r in rows:
            if r is None:
                f.write("\n")
            elif fmt:
                f.write(fmt % tuple(r) + "\n")
            else:
                f.write(" ".join(repr(float(v)) if not isinstance(v, (int, np.integer)) else str(int(v))
                                 for v in r) + "\n")


def write_outputs(prefix, dist, rd, d, nf, smp_temp=None):
    """PROJNM.dist, .bar, .dlnN, .TTPdist, and with smp_temp also .et, .sph, _T.cdist and
    _T.prob, as distrib_MULT writes them."""
    EE, de = dist["EE"], dist["de"]
    emin, emax = dist["emin"], dist["emax"]
    if dist["fwflg"]:
        rows = [(EE[i], dist["rlnP"][i], dist["lnP"][i]) for i in range(len(EE)) if dist["rlnP"][i] != EMPTY]
        rows += [None, (emin, 0.0, 0.0), (emin, -3.0, -3.0), None, (emax, 0.0, 0.0), (emax, -3.0, -3.0)]
    else:
        rows = [(EE[i], dist["lnP"][i]) for i in range(len(EE)) if dist["lnP"][i] != EMPTY]
        rows += [None, (emin, 0.0), (emin, -3.0), None, (emax, 0.0), (emax, -3.0)]
    _rows(prefix + ".dist", rows)
    nset = len(dist["flt"])
    bar = []
    for k in range(0, len(dist["bar"]), 2):
        bar += [dist["bar"][k], dist["bar"][k + 1], None]
    bar += [(emin, 0), (emin, nset + 1), None, (emax, 0), (emax, nset + 1)]
    _rows(prefix + ".bar", bar)
    span = nf["ceup"] - nf["celw"]
    lowd, upd = nf["alphalw"], nf["alphaup"]
    rows = []
    for i in range(len(EE) - 1):
        if d[i] == 0.0:
            continue
        fitv = _poly(nf, (EE[i] + 0.5 * de - nf["celw"]) / span)
        rows.append((EE[i] + 0.5 * de, d[i], fitv) + ((rd[i],) if dist["fwflg"] else ()))
    k = 4 if dist["fwflg"] else 3
    lo, hi = nf["celw"], nf["ceup"]
    rows += [None, (lo,) + (lowd,) * (k - 1), (lo,) + (upd,) * (k - 1), None,
             (hi,) + (lowd,) * (k - 1), (hi,) + (upd,) * (k - 1)]
    _rows(prefix + ".dlnN", rows)
    _rows(prefix + ".TTPdist", [(EE[i] + 0.5 * de, *dist["ttpdist"][i]) for i in range(len(EE))
                                if dist["ttpdist"][i, 0] != 0])
    if smp_temp is not None:
        et, sph = temperatures(dist, nf)
        _rows(prefix + ".et", et)
        _rows(prefix + ".sph", sph)
        ee, lnpc, (nb, eb, e0) = canonical(dist, nf, smp_temp)
        tag = f"{prefix}_{int(smp_temp)}"
        _rows(tag + ".cdist", zip(ee, lnpc))
        with open(tag + ".prob", "w") as f:
            f.write("MULT\n%d\n%r\n%r\n\n" % (nb, float(eb), float(e0)))
            for v in np.exp(lnpc):
                f.write(repr(float(v)) + "\n")


def iterate(counts, old, emin, emax, nbin, nbor, next_emin, next_emax, next_temp, nwindow=1,
            ndeg=8, fw=None, sets=None, accele=False, accrat=1.0, accel2=False, accrt2=1.0,
            ignore_empty=True, neglect_low=False, neglect_high=False, prefix=None, smp_temp=None):
    """One GEprep McMD iteration from the runs' histograms: the distribution, d lnN/dE, the
    new weight; with `prefix` the reference's output files are written.  Returns a dict with
    the new weight (`nf`), its fit residuals, the distribution and the fit data."""
    dist = distribution(counts, emin, emax, nbin, nbor, fw=fw, sets=sets, accele=accele, accrat=accrat)
    rd, d = dlnn(dist, old, accel2=accel2, accrt2=accrt2)
    X, Y, W = fit_data(dist, d, old, next_emin, next_emax, ignore_empty, neglect_low, neglect_high)
    nf, resid = fit(X, Y, W, next_emin, next_emax, next_temp, nwindow, ndeg, old)
    if prefix:
        write_outputs(prefix, dist, rd, d, nf, smp_temp)
    return dict(nf=nf, resid=resid, dist=dist, rdlnN=rd, dlnN=d, data=(X, Y, W))


# ---- ALSD: the weight in lambda (src_GEprep/distrib_ALSD.f90) ----------------------------
def alsd_distribution(counts, dedl, lmin, lmax, nbin, nbor, temp, fw=None, sets=None, accele=False,
                      accrat=1.0):
    """distrib_ALSD's distribution in lambda and mean force.  counts, dedl [nrun][nBIN + 2 nBOR]:
    per lambda bin the visits and the sum of dE/dlambda of the cluster energy (the engine's
    jp_alsd_hist_get).  Per set (onend_data, distrib_ALSD.f90:675-706): flatness of its own
    visits; F += fw * dedl and w += fw * counts, divided by flatness^accrat with acceleration.
    P = all visits.  F(i) = -F / w / (R T), rF(i) = -(sum of dedl) / P / (R T) where P != 0
    (:405-412).  Returns EE (bin centres), P, lnP, F, rF, flatness (overall and per set),
    the max/min visit ratio over the inner bins, and the lambda ranges per set."""
    counts = np.atleast_2d(np.asarray(counts, np.float64))
    dedl = np.atleast_2d(np.asarray(dedl, np.float64))
    nrun, nab = counts.shape
    fw = np.ones(nrun) if fw is None else np.asarray(fw, np.float64)
    sets = np.arange(nrun) if sets is None else np.asarray(sets)
    EE, dl = bin_centres(lmin, lmax, nbin, nbor)
    P, F, w, rF = np.zeros(nab), np.zeros(nab), np.zeros(nab), np.zeros(nab)
    flt, lrange = [], []
    for s in np.unique(sets):
        runs = np.flatnonzero(sets == s)
        tP = counts[runs].sum(axis=0)
        tF = (dedl[runs] * fw[runs, None]).sum(axis=0)
        tw = (counts[runs] * fw[runs, None]).sum(axis=0)
        rF += dedl[runs].sum(axis=0)
        P += tP
        if tP.max() == 0.0:
            continue
        tlnp = _lnp(tP)
        f = _flatness(tlnp, nbor, nbin)
        flt.append(f if f != 0.0 else 0.01)
        a = 1.0 / flt[-1] ** accrat if accele else 1.0
        F += tF * a
        w += tw * a
        occ = np.flatnonzero(tlnp != EMPTY)
        sub = occ[tlnp[occ] >= -1.5]
        lrange.append((EE[occ[-1]] - EE[occ[0]] + dl, EE[sub[-1]] - EE[sub[0]] + dl))
    lnP = _lnp(P)
    rt = 1.0 / (R_GAS * temp)
    nz = P != 0.0
    Fo, rFo = np.zeros(nab), np.zeros(nab)
    Fo[nz] = -F[nz] / w[nz] * rt
    rFo[nz] = -rF[nz] / P[nz] * rt
    inner = P[nbor:nbor + nbin]
    ratio = float(inner.max() / inner.min()) if inner.min() > 0 else float("inf")
    return dict(EE=EE, de=dl, lmin=lmin, lmax=lmax, nbin=nbin, nbor=nbor, P=P, lnP=lnP, F=Fo, rF=rFo,
                flat=_flatness(lnP, nbor, nbin), flt=np.array(flt), maxmin=ratio,
                lrange=np.array(lrange))


def alsd_fit(dist, next_lmin, next_lmax, next_temp, nwindow, ndeg, force_low, force_high,
             neglect_low=False, neglect_high=False):
    """The lambda weight (distrib_ALSD.f90:415-475): F at the bin centres of the occupied bins,
    weights sqrt(P), fitted by lstsquare_final on [next_lmin, next_lmax] in lambda itself;
    lowd = c0 of window 1, upd = the last window at next_lmax, the walls -force_low and
    force_high.  Returns the weight dict (jp_ge / .nf with lower, upper) and the residuals."""
    EE, P, F = dist["EE"], dist["P"], dist["F"]
    nbin, nbor = dist["nbin"], dist["nbor"]
    ist = nbor if neglect_low else 0
    ien = nbor + nbin - 1 if neglect_high else len(EE) - 2
    keep = [i for i in range(ist, ien + 1) if P[i] != 0.0]
    X, Y, W = EE[keep], F[keep], np.sqrt(P[keep])
    coef, low, high, resid = engine.lstsq_windows(X, Y, W, nwindow, ndeg, next_lmin, next_lmax)
    upd = _poly(dict(coef=coef[-1:], low=low[-1:], high=high[-1:]), next_lmax)
    nf = dict(coef=coef, low=low, high=high, alphalw=float(coef[0, 0]), alphaup=upd, celw=next_lmin,
              ceup=next_lmax, tempce=next_temp, lower=-float(force_low), upper=float(force_high))
    return nf, resid, (X, Y, W)


def alsd_net_data(counts2, dedl2, emin, emax, lmin, lmax, nbin, nbor, temp):
    """Training data of the (E, lambda) network from the (E, lambda) histograms [ne][nl]
    (jp_alsd_hist_get): at each visited cell x = (reduced E, lambda) and two targets, the
    cell's mean d lnP/dlambda = -<dE/dlambda> / (R T) (the lambda weight distrib_ALSD fits,
    here also resolved in E) and d lnN/dE = d ln(visits)/dE + 1 / (R T) at fixed lambda
    (the canonical distribution in E of a lambda bin; a cell without a visited E neighbour
    takes its lambda column's mean); weights sqrt(visits)."""
    c2 = np.asarray(counts2, np.float64)
    f2 = np.asarray(dedl2, np.float64)
    ne, nl = c2.shape
    de = (emax - emin) / ne
    EEc = emin + de * (np.arange(ne) + 0.5)
    LL, _ = bin_centres(lmin, lmax, nbin, nbor)
    rt = 1.0 / (R_GAS * temp)
    X, Y, W = [], [], []
    for i in range(nl):
        col = c2[:, i]
        occ = np.flatnonzero(col > 0)
        if len(occ) == 0:
            continue
        slopes = {}
        for a in occ:
            if a + 1 < ne and col[a + 1] > 0:
                slopes[a] = (np.log(col[a + 1]) - np.log(col[a])) / de + rt
        mean_slope = float(np.mean(list(slopes.values()))) if slopes else rt
        for a in occ:
            X.append(((EEc[a] - emin) / (emax - emin), LL[i]))
            Y.append((-f2[a, i] / col[a] * rt, slopes.get(a, mean_slope)))
            W.append(np.sqrt(col[a]))
    return np.array(X), np.array(Y), np.array(W)
