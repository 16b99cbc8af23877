"""Generate tests/golden/kat.json: known-answer vectors for md_run's force field.

The reference (j_presto md_run) ships no tests, golden vectors or fixtures, and cannot be
compiled here (no Fortran compiler).  These vectors are closed-form evaluations of the
formulas md_run implements, written independently of oracle/oracle.cpp and of the CUDA
engine:

  ZD pair   E = 332.06378*qi*qj*(1/r + r^2/(2 rc^3) - 1.5/rc), co = [r <= rc]
            (enear.f90:132-141 with incel.f90:655-658)
  self      dself = -(1.5/rc)/2 * 332.06378 * sum_i qi*(qi + sum_{excl j} qj)
            (incel.f90:631-662), excluded pairs add qi*qj*332.06378*r^2/(2 rc^3)
            (enear.f90:518-555)
  LJ        E = C12/r^12 - C6/r^6, AMBER mixing (inptpl.f90:409-425)
  bond      K (r - r0)^2; angle K (theta - theta0)^2; torsion K (1 + cos(n phi + d))/div
  1-4       s_vdw*(C12/r^12 - C6/r^6) + s_ele*332.06378*qi*qj/r (dnergv.f90:440-516)

Gradients are central differences (h = 1e-6 A) of the closed-form energy.

    python tests/golden/make_golden.py      # rewrites kat.json
"""
import json
import math
import os

import numpy as np

CC = 332.06378
HERE = os.path.dirname(os.path.abspath(__file__))

# two LJ types: 0 = no LJ, 1 = TIP3P-like oxygen (Rmin/2 1.76827 A, eps 0.1521)
R = np.array([0.0, 1.76827])
EPS = np.array([0.0, 0.1521])
C6 = 2.0 * np.sqrt(np.outer(EPS, EPS)) * np.add.outer(R, R) ** 6
C12 = np.sqrt(np.outer(EPS, EPS)) * np.add.outer(R, R) ** 12


def mimg(d, box):
    return d - box * np.round(d / box)


def base_system(x, q, t, box):
    n = len(q)
    return dict(natom=n, box=[box] * 3, cord=np.asarray(x, float).tolist(), mass=[12.0] * n,
                charge=list(map(float, q)), atype=list(map(int, t)), ntype=2,
                c6=C6.tolist(), c12=C12.tolist(), s14_vdw=[0.5, 0.5], s14_ele=[1 / 1.2, 1 / 1.2],
                excl=[[] for _ in range(n)], bond=[], bond_k=[], bond_r0=[], angle=[],
                angle_k=[], angle_theta0=[], tors=[], tors_k=[], tors_nrot=[], tors_phase=[],
                tors_div=[], tors_nbf=[], impr=[], impr_k=[], impr_nrot=[], impr_phase=[],
                impr_div=[])


def energy_nonbonded(x, sysd, rc, inside=None):
    """ZD + LJ over all non-excluded pairs (minimum image) + excess + self, by slot.
    `inside` (set of pairs) freezes which pairs count as r <= rc, so that finite
    differences at a pair sitting exactly on the cut-off see one smooth branch."""
    x = np.asarray(x)
    q = np.array(sysd["charge"])
    t = sysd["atype"]
    box = sysd["box"][0]
    n = len(q)
    ex = [set(e) for e in sysd["excl"]]
    el = vdw = 0.0
    for i in range(n):
        for j in range(i + 1, n):
            if j in ex[i]:
                continue
            r = np.linalg.norm(mimg(x[i] - x[j], box))
            if (r <= rc) if inside is None else ((i, j) in inside):
                el += CC * q[i] * q[j] * (1 / r + r * r / (2 * rc ** 3) - 1.5 / rc)
                vdw += C12[t[i], t[j]] / r ** 12 - C6[t[i], t[j]] / r ** 6
    # excess: every bond, angle 1-3 and nbf torsion pair
    pairs = [tuple(b) for b in sysd["bond"]] + [(a[0], a[2]) for a in sysd["angle"]] + \
        [(tt[0], tt[3]) for tt, f in zip(sysd["tors"], sysd["tors_nbf"]) if f == 1]
    dw = q.copy()
    for a, b in pairs:
        r = np.linalg.norm(mimg(x[a] - x[b], box))
        el += CC * q[a] * q[b] * r * r / (2 * rc ** 3)
        dw[a] += q[b]
        dw[b] += q[a]
    el += -(1.5 / rc) * 0.5 * CC * float(np.dot(q, dw))
    return el, vdw


def dihedral(a, b, c, d):
    b0, b1, b2 = a - b, c - b, d - c
    n1 = np.cross(-b0, b1)
    n2 = np.cross(b1, b2)
    return math.atan2(np.dot(np.cross(n1, n2), b1 / np.linalg.norm(b1)), np.dot(n1, n2))


def energy_bonded(x, sysd):
    x = np.asarray(x)
    q = np.array(sysd["charge"])
    t = sysd["atype"]
    e = dict(bond=0.0, angle=0.0, tors=0.0, vdw14=0.0, ele14=0.0)
    for (a, b), k, r0 in zip(sysd["bond"], sysd["bond_k"], sysd["bond_r0"]):
        e["bond"] += k * (np.linalg.norm(x[a] - x[b]) - r0) ** 2
    for (a, b, c), k, t0 in zip(sysd["angle"], sysd["angle_k"], sysd["angle_theta0"]):
        u, v = x[a] - x[b], x[c] - x[b]
        th = math.acos(np.dot(u, v) / np.linalg.norm(u) / np.linalg.norm(v))
        e["angle"] += k * (th - t0) ** 2
    for tt, k, n, ph, dv, nbf in zip(sysd["tors"], sysd["tors_k"], sysd["tors_nrot"],
                                     sysd["tors_phase"], sysd["tors_div"], sysd["tors_nbf"]):
        phi = dihedral(*[x[i] for i in tt])
        e["tors"] += k * (1 + math.cos(n * phi + ph)) / dv
        if nbf == 1:
            a, d = tt[0], tt[3]
            r = np.linalg.norm(x[a] - x[d])
            sv = min(sysd["s14_vdw"][t[a]], sysd["s14_vdw"][t[d]])
            se = min(sysd["s14_ele"][t[a]], sysd["s14_ele"][t[d]])
            e["vdw14"] += sv * (C12[t[a], t[d]] / r ** 12 - C6[t[a], t[d]] / r ** 6)
            e["ele14"] += se * CC * q[a] * q[d] / r
    return e


def all_energy(x, sysd, rc, inside=None):
    el, vdw = energy_nonbonded(x, sysd, rc, inside)
    b = energy_bonded(x, sysd)
    ene = [0.0] * 15
    ene[1], ene[2], ene[3] = b["bond"], b["angle"], b["tors"]
    ene[5], ene[6], ene[7], ene[8] = b["vdw14"], b["ele14"], vdw, el
    ene[0] = sum(ene[1:])
    return ene


def inside_pairs(x, sysd, rc):
    x = np.asarray(x)
    box = sysd["box"][0]
    n = len(x)
    return {(i, j) for i in range(n) for j in range(i + 1, n)
            if np.linalg.norm(mimg(x[i] - x[j], box)) <= rc}


def fd_grad(x, sysd, rc, h=1e-6):
    x = np.asarray(x, float)
    g = np.zeros_like(x)
    ins = inside_pairs(x, sysd, rc)
    for i in range(x.shape[0]):
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[i, k] += h
            xm[i, k] -= h
            g[i, k] = (all_energy(xp, sysd, rc, ins)[0] - all_energy(xm, sysd, rc, ins)[0]) / (2 * h)
    return g


def cases():
    rc = 12.0
    out = {}
    # 1. two charges at 3 A, no LJ
    s = base_system([[5, 5, 5], [8, 5, 5]], [0.5, -0.7], [0, 0], 40.0)
    out["zd_pair"] = s
    # 2. LJ pair (neutral oxygens) at 3.5 A
    out["lj_pair"] = base_system([[5, 5, 5], [5, 8.5, 5]], [0.0, 0.0], [1, 1], 40.0)
    # 3. cut-off edge: r = rc exactly interacts (co = 1 at equality), r = 12.5 is listed
    #    (< rc + 1.5) but contributes nothing, r = 14 is not listed
    out["cutoff_edge"] = base_system([[1, 1, 1], [13, 1, 1], [1, 13.5, 1], [1, 1, 15]],
                                     [0.4, -0.3, 0.2, 0.1], [1, 1, 1, 1], 40.0)
    # 4. minimum image across the box face
    out["min_image"] = base_system([[0.5, 10, 10], [27.3, 10, 10]], [0.6, -0.6], [1, 1], 30.0)
    # 5. bonded chain A-B-C-D with every pair excluded (1-2, 1-3, 1-4)
    phi = math.radians(150.0)
    x = [[0, 2.0, 0], [0, 0, 0], [1.5, 0, 0], [1.5, 2.0 * math.cos(phi), 2.0 * math.sin(phi)]]
    s = base_system(x, [0.3, -0.2, 0.25, -0.35], [1, 0, 0, 1], 40.0)
    s["excl"] = [[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]]
    s["bond"], s["bond_k"], s["bond_r0"] = [[0, 1], [1, 2], [2, 3]], [300.0, 340.0, 280.0], [1.1, 1.05, 1.25]
    s["angle"], s["angle_k"], s["angle_theta0"] = [[0, 1, 2], [1, 2, 3]], [50.0, 60.0], [1.745, 1.9]
    s["tors"], s["tors_k"], s["tors_nrot"] = [[0, 1, 2, 3]], [1.4], [3.0]
    s["tors_phase"], s["tors_div"], s["tors_nbf"] = [0.0], [1], [1]
    out["bonded_chain"] = s
    # 6. torsion with phase pi and n = 2, second torsion term on the same 1-4 pair (nbf 0)
    s2 = json.loads(json.dumps(s))
    s2["tors"] = [[0, 1, 2, 3], [0, 1, 2, 3]]
    s2["tors_k"], s2["tors_nrot"] = [1.4, 0.7], [3.0, 2.0]
    s2["tors_phase"], s2["tors_div"], s2["tors_nbf"] = [0.0, math.pi], [1, 2], [1, 0]
    out["torsion_multi"] = s2
    # 7. one rigid water: all three atoms mutually excluded, neutral -> dself = 0
    roh, th = 0.9572, math.radians(104.52)
    w = [[3, 3, 3], [3 + roh, 3, 3], [3 + roh * math.cos(th), 3 + roh * math.sin(th), 3]]
    s = base_system(w, [-0.834, 0.417, 0.417], [1, 0, 0], 40.0)
    s["excl"] = [[1, 2], [0, 2], [0, 1]]
    s["bond"], s["bond_k"], s["bond_r0"] = [[0, 1], [0, 2]], [553.0, 553.0], [roh, roh]
    s["angle"], s["angle_k"], s["angle_theta0"] = [[1, 0, 2]], [100.0], [th]
    out["water"] = s
    res = {}
    for name, sysd in out.items():
        ene = all_energy(sysd["cord"], sysd, rc)
        g = fd_grad(sysd["cord"], sysd, rc)
        res[name] = dict(system=sysd, cutoff=rc, energy=ene, grad=g.tolist())
    res["_meta"] = dict(generator="tests/golden/make_golden.py", eekcal=CC,
                        note="closed-form md_run force-field energies; FD gradients h=1e-6")
    # McMD weight: R*T0*P(x) with P a polynomial in x = (E-celw)/(ceup-celw)
    coef = [0.9, -0.3, 0.05]
    ge = dict(nwindow=1, ndeg=2, coef=[coef], low=[0.0], high=[1.0 + 1e-12], alphalw=1.2,
              alphaup=0.4, celw=-100.0, ceup=100.0, tempce=300.0)
    pts = [-150.0, -100.0, -20.0, 0.0, 55.0, 100.0, 130.0]
    Rk = 8.31451 / 4.184 * 1e-3
    vals = []
    for e in pts:
        if e <= ge["celw"]:
            p = ge["alphalw"]
        elif e >= ge["ceup"]:
            p = ge["alphaup"]
        else:
            xx = (e - ge["celw"]) / (ge["ceup"] - ge["celw"])
            p = sum(c * xx ** k for k, c in enumerate(coef))
        vals.append(Rk * ge["tempce"] * p)
    res["_mcmd"] = dict(ge=ge, energies=pts, scale=vals)
    return res


if __name__ == "__main__":
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(cases(), f, indent=1)
    print("wrote", os.path.join(HERE, "kat.json"))
