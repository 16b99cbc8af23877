"""Seeded synthetic MD systems in md_run's topology model.

The reference benchmarks on no public dataset; these generators produce the five workloads
(water box, solvated polymer, large water/ion box, uneven McMD replicas, ALSD replicas)
from a seed, with md_run's conventions:

* LJ parameters in AMBER form (Rmin/2, epsilon) mixed as C6 = 2*sqrt(ei*ej)*(Ri+Rj)^6,
  C12 = sqrt(ei*ej)*(Ri+Rj)^12 (md_run inptpl.f90:409-425), 1-4 scales per type;
* exclusions = 1-2, 1-3 and 1-4 partners (the TPL ix14lt list);
* torsions enumerated over every bond, the first torsion of each 1-4 pair flagged nbf=1;
* SHAKE groups as in a .shk file: a heavy atom with its hydrogens, all pair distances
  constrained, in md_run pair order (1,2),(2,3),(3,1),(4,1),(3,4),(2,4).

Every topology is a dict of numpy arrays consumed by `abi.make_system`.
"""
import math

import numpy as np

# --- atom types: (name, Rmin/2 [A], epsilon [kcal/mol], mass) -------------------------
TYPES = [
    ("OW", 1.76827, 0.1521, 15.9994),   # TIP3P-like oxygen: sigma 3.15061 A
    ("HW", 0.0, 0.0, 1.008),
    ("C", 1.9080, 0.0860, 12.011),
    ("N", 1.8240, 0.1700, 14.007),
    ("O", 1.6612, 0.2100, 15.9994),
    ("H", 0.6000, 0.0157, 1.008),
    ("HC", 1.4870, 0.0157, 1.008),
    ("NA", 1.3470, 0.1000, 22.990),     # sigma 2.4 A
    ("CL", 2.4690, 0.1000, 35.453),     # sigma 4.4 A
]
T_OW, T_HW, T_C, T_N, T_O, T_H, T_HC, T_NA, T_CL = range(len(TYPES))
S14_VDW, S14_ELE = 0.5, 1.0 / 1.2       # AMBER 1-4 scales

Q_OW, Q_HW = -0.834, 0.417
R_OH, ANG_HOH = 0.9572, math.radians(104.52)
R_HH = 2.0 * R_OH * math.sin(ANG_HOH / 2.0)
WATER_DENSITY = 0.0334                  # molecules / A^3

MOL_SOLUTE, MOL_WATER, MOL_NA, MOL_CL = 0, 1, 2, 3


def lj_tables():
    nt = len(TYPES)
    R = np.array([t[1] for t in TYPES])
    E = np.array([t[2] for t in TYPES])
    rr = (R[:, None] + R[None, :]) ** 6
    ee = np.sqrt(E[:, None] * E[None, :])
    c6 = 2.0 * ee * rr
    c12 = ee * rr * rr
    return nt, c6, c12


class _Top:
    def __init__(self, rng):
        self.rng = rng
        self.pos, self.mass, self.chg, self.typ, self.mol = [], [], [], [], []
        self.bonds, self.bond_k = [], []
        self.shake = []          # (atoms tuple)
        self.impr = []           # (a,b,c,d,k,n,phase)
        self.water_first = None

    def add(self, p, t, q, mol):
        self.pos.append(np.asarray(p, float))
        self.typ.append(t)
        self.chg.append(q)
        self.mass.append(TYPES[t][3])
        self.mol.append(mol)
        return len(self.pos) - 1


def _perp(v, rng):
    a = rng.normal(size=3)
    a -= a.dot(v) / v.dot(v) * v
    return a / np.linalg.norm(a)


def _serpentine(npts, step, lo, hi, rowgap):
    """`npts` points spaced `step` (arc length) along a 3-D boustrophedon inside the box
    [lo, hi]^3: rows along x, stepped by `rowgap` in y, layers stepped by `rowgap` in z,
    the y order reversed on every other layer so each turn is one short straight leg."""
    nrow = max(1, int((hi - lo) // rowgap))
    rows = lo + 0.5 * rowgap + rowgap * np.arange(nrow)
    way = []
    k = 0
    for iz, z in enumerate(rows):
        for y in (rows if iz % 2 == 0 else rows[::-1]):
            xa, xb = (lo, hi) if k % 2 == 0 else (hi, lo)
            way += [(xa, y, z), (xb, y, z)]
            k += 1
    way = np.array(way, float)
    seg = np.diff(way, axis=0)
    slen = np.linalg.norm(seg, axis=1)
    keep = slen > 1e-9
    seg, slen, base = seg[keep], slen[keep], way[:-1][keep]
    cum = np.concatenate([[0.0], np.cumsum(slen)])
    s_at = step * np.arange(npts)
    if s_at[-1] > cum[-1]:
        raise ValueError("polymer does not fit in the box")
    i = np.minimum(np.searchsorted(cum, s_at, side="right") - 1, len(slen) - 1)
    t = (s_at - cum[i]) / slen[i]
    return base[i] + t[:, None] * seg[i]


def _build_polymer(top, nres, lo, hi, rng, box):
    """Generic amino-acid-like chain: backbone N-CA-C(=O) with H on N and CA, plus a side
    chain of 1-10 atoms (heavy atoms carrying up to 2-3 hydrogens) per residue.  The
    backbone follows a boustrophedon path; side-chain atoms are placed by a tetrahedral
    random walk, each the least crowded of many trial positions."""
    step = 1.26
    path = _serpentine(3 * nres, step, lo, hi, rowgap=12.0)
    buf = np.zeros((16 * nres + 16, 3))
    nbuf = [0]
    first = len(top.pos)

    def place(p, t):
        a = top.add(p, t, 0.0, MOL_SOLUTE)
        buf[nbuf[0]] = p
        nbuf[0] += 1
        return a

    def crowd(cands, skip):
        """min distance of each candidate to placed solute atoms, ignoring `skip`."""
        P = buf[:nbuf[0]]
        dv = cands[:, None, :] - P[None, :, :]
        dv -= box * np.round(dv / box)
        d = np.linalg.norm(dv, axis=2)
        for s_ in skip:
            d[:, s_ - first] = np.inf
        return d.min(axis=1) if P.shape[0] else np.full(len(cands), np.inf)

    def tetra_dirs(prev, ntry):
        """unit vectors at ~109.5 deg from -prev (random azimuth)."""
        ca, sa = math.cos(math.radians(70.5)), math.sin(math.radians(70.5))
        out = []
        for _ in range(ntry):
            pp = _perp(prev, rng)
            out.append(ca * prev + sa * pp)
        return np.array(out)

    res = []
    prev_c = None
    for r in range(nres):
        idx = {}
        tang = path[min(3 * r + 3, len(path) - 1)] - path[max(3 * r - 1, 0)]
        tang /= np.linalg.norm(tang)
        zz = np.array([0.0, 0.0, 1.0]) if abs(tang[2]) < 0.9 else np.array([1.0, 0.0, 0.0])
        off = np.cross(tang, zz)
        off /= np.linalg.norm(off)
        # zig-zag: path atom i sits at (-1)^i * 0.41 A off the path
        sg = [1.0 if (3 * r + k) % 2 == 0 else -1.0 for k in range(3)]
        idx["N"] = place(path[3 * r] + sg[0] * 0.41 * off, T_N)
        idx["CA"] = place(path[3 * r + 1] + sg[1] * 0.41 * off, T_C)
        idx["C"] = place(path[3 * r + 2] + sg[2] * 0.41 * off, T_C)
        idx["atoms"] = [idx["N"], idx["CA"], idx["C"]]
        if prev_c is not None:
            top.bonds.append((prev_c, idx["N"]))
        top.bonds += [(idx["N"], idx["CA"]), (idx["CA"], idx["C"])]
        idx["off"], idx["zz"], idx["sg"] = off, zz, sg
        res.append(idx)
        prev_c = idx["C"]
    for idx in res:
        off, zz, sg = idx["off"], idx["zz"], idx["sg"]
        p_c, p_n, p_ca = top.pos[idx["C"]], top.pos[idx["N"]], top.pos[idx["CA"]]
        # substituents point away from the zig-zag: O and HN of one peptide bond end up
        # on opposite sides (trans), HA below the plane, the side chain above it
        idx["O"] = place(p_c + 1.23 * sg[2] * off, T_O)
        top.bonds.append((idx["C"], idx["O"]))
        idx["HN"] = place(p_n + 1.01 * sg[0] * off, T_H)
        top.bonds.append((idx["N"], idx["HN"]))
        top.shake.append((idx["N"], idx["HN"]))
        idx["HA"] = place(p_ca + 1.09 * (0.5 * sg[1] * off - 0.866 * zz), T_HC)
        idx["atoms"] += [idx["O"], idx["HN"], idx["HA"]]
        top.bonds.append((idx["CA"], idx["HA"]))
        top.shake.append((idx["CA"], idx["HA"]))
    for idx in res:
        off, zz, sg = idx["off"], idx["zz"], idx["sg"]
        k = int(rng.integers(1, 11))
        m = max(1, (k + 2) // 3)
        nh = k - m
        heavy = []
        anchor = idx["CA"]
        prev_dir = -(0.5 * sg[1] * off + 0.866 * zz)
        nbrs = [idx["N"], idx["C"], idx["HA"]]
        for _ in range(m):
            cands = top.pos[anchor] + 1.53 * tetra_dirs(prev_dir, 48)
            score = crowd(cands, [anchor] + nbrs)
            best = int(np.argmax(score))
            a = place(cands[best], T_C)
            top.bonds.append((anchor, a))
            prev_dir = (cands[best] - top.pos[anchor]) / 1.53
            nbrs = [anchor]
            heavy.append(a)
            idx["atoms"].append(a)
            anchor = a
        # hydrogens: CH3 on the last heavy atom first, then CH2 down the chain
        caps = [2] * (len(heavy) - 1) + [3]
        hs = {a: [] for a in heavy}
        for i in reversed(range(len(heavy))):
            a = heavy[i]
            while nh > 0 and len(hs[a]) < caps[i]:
                bonded = [b2 for (x1, b2) in top.bonds if x1 == a] + [x1 for (x1, b2) in top.bonds if b2 == a]
                dirs = rng.normal(size=(64, 3))
                dirs /= np.linalg.norm(dirs, axis=1)[:, None]
                ok = np.ones(64, bool)
                for b2 in bonded:
                    u = top.pos[b2] - top.pos[a]
                    u /= np.linalg.norm(u)
                    ok &= dirs @ u < math.cos(math.radians(100.0))
                if not ok.any():
                    ok[:] = True
                cands = top.pos[a] + 1.09 * dirs[ok]
                score = crowd(cands, [a] + bonded)
                h = place(cands[int(np.argmax(score))], T_HC)
                top.bonds.append((a, h))
                hs[a].append(h)
                idx["atoms"].append(h)
                nh -= 1
        for a in heavy:
            if hs[a]:
                top.shake.append(tuple([a] + hs[a]))
    for r, idx in enumerate(res):
        if r + 1 < len(res):
            top.impr.append((idx["CA"], res[r + 1]["N"], idx["C"], idx["O"], 10.5, 2.0, math.pi))
    _relax_solute(top, first, len(top.pos), box)
    return res


def _relax_solute(top, first, last, box, iters=3000):
    """Position-based relaxation of the solute: bonds keep their built lengths, every 1-3
    pair is pulled to the distance of an ideal valence angle at its centre (120 deg at N
    and at the carbonyl C, 109.47 deg elsewhere), and every other pair is kept at
    >= 2.9 A between heavy atoms, >= 2.3 A with a hydrogen.  Bonded equilibrium values are
    taken from the relaxed geometry afterwards, so the start carries no bonded strain and
    no angle sits near 180 deg (where torsion gradients are singular)."""
    n = last - first
    if n < 2:
        return
    X = np.array(top.pos[first:last])
    isH = np.array([TYPES[t][0].startswith("H") for t in top.typ[first:last]])
    bonds = np.array([(a - first, b - first) for a, b in top.bonds
                      if first <= a < last and first <= b < last], int).reshape(-1, 2)
    L0 = np.linalg.norm(X[bonds[:, 0]] - X[bonds[:, 1]], axis=1)
    # heavy-atom bonds of the path's corners come out stretched or squeezed
    heavy_bond = ~isH[bonds[:, 0]] & ~isH[bonds[:, 1]]
    L0 = np.where(heavy_bond, np.clip(L0, 1.33, 1.53), L0)
    nbr = [set() for _ in range(n)]
    for a, b in bonds:
        nbr[a].add(b); nbr[b].add(a)
    blen = {}
    for (a, b), l0 in zip(bonds, L0):
        blen[(a, b)] = blen[(b, a)] = l0
    typ = [top.typ[first + i] for i in range(n)]
    sp2 = [typ[j] == T_N or (typ[j] == T_C and any(typ[b] == T_O for b in nbr[j]))
           for j in range(n)]
    t13 = {}
    for j in range(n):
        nb = sorted(nbr[j])
        c = math.cos(math.radians(120.0 if sp2[j] else 109.47))
        for x in range(len(nb)):
            for y in range(x + 1, len(nb)):
                la, lc = blen[(nb[x], j)], blen[(nb[y], j)]
                t13[(nb[x], nb[y])] = math.sqrt(la * la + lc * lc - 2.0 * la * lc * c)
    p13 = np.array(sorted(t13), int).reshape(-1, 2)
    d13 = np.array([t13[tuple(k)] for k in p13]) if len(p13) else np.zeros(0)
    from scipy.spatial import cKDTree
    ex_codes = np.unique(np.concatenate([np.minimum(bonds[:, 0], bonds[:, 1]) * n + np.maximum(bonds[:, 0], bonds[:, 1]),
                                         np.minimum(p13[:, 0], p13[:, 1]) * n + np.maximum(p13[:, 0], p13[:, 1])]))
    boxv = np.full(3, float(box)) if np.ndim(box) == 0 else np.asarray(box, float)
    iu = ju = dmin = None
    for it in range(iters):
        if it % 8 == 0:   # neighbour candidates within 3.5 A, periodic, 1-2/1-3 pairs removed
            tree = cKDTree(np.mod(X, boxv), boxsize=boxv)
            pr = tree.query_pairs(3.5, output_type="ndarray")
            if len(pr):
                a, b = np.minimum(pr[:, 0], pr[:, 1]), np.maximum(pr[:, 0], pr[:, 1])
                keep = ~np.isin(a * n + b, ex_codes)
                iu, ju = a[keep], b[keep]
            else:
                iu = ju = np.zeros(0, int)
            dmin = np.where(isH[iu] | isH[ju], 2.3, 2.9)
        moved = False
        # non-bonded minimum distances
        d = X[iu] - X[ju]
        d -= box * np.round(d / box)
        r = np.linalg.norm(d, axis=1)
        bad = r < dmin
        if bad.any():
            moved = True
            f = (0.5 * (dmin[bad] - r[bad]) / np.maximum(r[bad], 1e-6))[:, None] * d[bad]
            np.add.at(X, iu[bad], 0.5 * f)
            np.add.at(X, ju[bad], -0.5 * f)
        # 1-3 distances of the ideal valence angles
        if len(p13):
            d = X[p13[:, 0]] - X[p13[:, 1]]
            d -= box * np.round(d / box)
            r = np.linalg.norm(d, axis=1)
            bad = np.abs(r - d13) > 1e-3
            if bad.any():
                moved = True
                f = (0.25 * (d13[bad] - r[bad]) / np.maximum(r[bad], 1e-6))[:, None] * d[bad]
                np.add.at(X, p13[bad, 0], f)
                np.add.at(X, p13[bad, 1], -f)
        # bond lengths
        d = X[bonds[:, 0]] - X[bonds[:, 1]]
        r = np.linalg.norm(d, axis=1)
        f = (0.5 * (L0 - r) / r)[:, None] * d
        np.add.at(X, bonds[:, 0], f)
        np.add.at(X, bonds[:, 1], -f)
        if not moved and it > 10:
            break
    for i in range(n):
        top.pos[first + i] = X[i]


def _charges_polymer(top, first, last, residues, rng):
    """Partial charges ~N(0, 0.3 e) renormalised so each residue carries an integer charge.
    Hydrogens get small positive charges (|N(0, 0.15)| + 0.05): TIP3P water hydrogens carry
    no Lennard-Jones repulsion, so a negatively charged solute hydrogen would let a water
    hydrogen collapse onto it.  The heavy atoms absorb the renormalisation."""
    total = 0
    for res in residues:
        ids = np.array(res["atoms"])
        isH = np.array([TYPES[top.typ[a]][0].startswith("H") for a in ids])
        q = rng.normal(0.0, 0.3, size=len(ids))
        q[isH] = np.abs(rng.normal(0.0, 0.15, size=int(isH.sum()))) + 0.05
        target = int(max(-1, min(1, round(q.sum()))))
        heavy = ~isH
        q[heavy] += (target - q.sum()) / int(heavy.sum())
        for a, v in zip(ids, q):
            top.chg[a] = float(v)
        total += target
    return total


def _place_water(top, o_pos, rng):
    bis = rng.normal(size=3)
    bis /= np.linalg.norm(bis)
    p = _perp(bis, rng)
    h = 0.5 * ANG_HOH
    h1 = o_pos + R_OH * (math.cos(h) * bis + math.sin(h) * p)
    h2 = o_pos + R_OH * (math.cos(h) * bis - math.sin(h) * p)
    o = top.add(o_pos, T_OW, Q_OW, MOL_WATER)
    a = top.add(h1, T_HW, Q_HW, MOL_WATER)
    b = top.add(h2, T_HW, Q_HW, MOL_WATER)
    top.bonds += [(o, a), (o, b)]
    top.shake.append((o, a, b))


def _lattice(box, nsites_min):
    n = int(math.ceil(nsites_min ** (1.0 / 3.0) - 1e-9))
    a = box / n
    g = (np.arange(n) + 0.5) * a
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1), a


def _finalize(top, box, temp, rng, with_bonded_params=True):
    n = len(top.pos)
    cord = np.array(top.pos)
    # bond graph
    nbr = [[] for _ in range(n)]
    for a, b in top.bonds:
        nbr[a].append(b)
        nbr[b].append(a)
    bonds = np.array(top.bonds, np.int32).reshape(-1, 2)
    # angles: every pair of neighbours around a centre atom
    angles = []
    for j in range(n):
        nb = sorted(nbr[j])
        for x in range(len(nb)):
            for y in range(x + 1, len(nb)):
                angles.append((nb[x], j, nb[y]))
    angles = np.array(angles, np.int32).reshape(-1, 3)
    # torsions over every bond j-k
    tors = []
    for j, k in top.bonds:
        for i in nbr[j]:
            if i == k:
                continue
            for l in nbr[k]:
                if l == j or l == i:
                    continue
                tors.append((i, j, k, l))
    tors = np.array(tors, np.int32).reshape(-1, 4)
    # exclusions: 1-2, 1-3, 1-4
    ex = [set() for _ in range(n)]
    for a, b in bonds:
        ex[a].add(b); ex[b].add(a)
    for a, _, c in angles:
        ex[a].add(c); ex[c].add(a)
    nbf = np.zeros(len(tors), np.int32)
    seen = set()
    for t, (a, _, _, d) in enumerate(tors):
        key = (min(a, d), max(a, d))
        if key in seen or d in ex[a]:
            continue
        seen.add(key)
        nbf[t] = 1
    for a, _, _, d in tors:
        ex[a].add(d); ex[d].add(a)
    excl_ptr = np.zeros(n + 1, np.int32)
    for i in range(n):
        excl_ptr[i + 1] = excl_ptr[i] + len(ex[i])
    excl_idx = np.array([j for i in range(n) for j in sorted(ex[i])], np.int32)
    # bonded parameters: equilibrium values from the built geometry, force constants
    # drawn from typical AMBER ranges
    def vec(i, j):
        d = cord[i] - cord[j]
        return d - box * np.round(d / box)
    r0 = np.array([np.linalg.norm(vec(a, b)) for a, b in bonds]) if len(bonds) else np.zeros(0)
    bk = rng.uniform(300.0, 570.0, size=len(bonds))
    wat = np.array([top.typ[a] == T_OW for a, _ in bonds]) if len(bonds) else np.zeros(0, bool)
    bk[wat] = 553.0
    th0 = []
    for a, j, c in angles:
        u, v = vec(a, j), vec(c, j)
        th0.append(math.acos(max(-1.0, min(1.0, u.dot(v) / np.linalg.norm(u) / np.linalg.norm(v)))))
    th0 = np.array(th0)
    ak = rng.uniform(35.0, 80.0, size=len(angles))
    if len(angles):
        wang = np.array([top.typ[j] == T_OW for _, j, _ in angles])
        ak[wang] = 100.0
    tk = rng.uniform(0.1, 2.0, size=len(tors))
    tn = rng.integers(1, 4, size=len(tors)).astype(float)
    tph = rng.choice([0.0, math.pi], size=len(tors))
    impr = np.array([x[:4] for x in top.impr], np.int32).reshape(-1, 4)
    ik = np.array([x[4] for x in top.impr])
    inr = np.array([x[5] for x in top.impr])
    iph = np.array([x[6] for x in top.impr])
    # SHAKE groups
    sh_n = np.array([len(g) for g in top.shake], np.int32)
    sh_a = np.full((len(top.shake), 4), -1, np.int32)
    sh_d = np.zeros((len(top.shake), 6))
    pairs = [(0, 1), (1, 2), (2, 0), (3, 0), (2, 3), (1, 3)]
    for g, atoms in enumerate(top.shake):
        sh_a[g, :len(atoms)] = atoms
        nc = len(atoms) * (len(atoms) - 1) // 2
        for q in range(nc):
            x, y = pairs[q]
            sh_d[g, q] = np.linalg.norm(vec(atoms[x], atoms[y]))
    # water groups get their exact model geometry
    for g, atoms in enumerate(top.shake):
        if len(atoms) == 3 and top.typ[atoms[0]] == T_OW:
            sh_d[g, :3] = (R_OH, R_HH, R_OH)
    nt, c6, c12 = lj_tables()
    mass = np.array(top.mass)
    # Maxwell-Boltzmann velocities (Angstrom/fs): variance R*T/m in (A/fs)^2
    sig = np.sqrt(8.31451e-7 * temp / mass)
    vel = rng.normal(size=(n, 3)) * sig[:, None]
    vel -= (mass[:, None] * vel).sum(0) / mass.sum()
    return dict(
        natom=n, box=np.asarray(box, float).reshape(3) if np.ndim(box) else np.full(3, float(box)),
        cord=cord, vel=vel, mass=mass, charge=np.array(top.chg), atype=np.array(top.typ, np.int32),
        molecule=np.array(top.mol, np.int32), ntype=nt, c6=c6, c12=c12,
        s14_vdw=np.full(nt, S14_VDW), s14_ele=np.full(nt, S14_ELE),
        excl_ptr=excl_ptr, excl_idx=excl_idx,
        bond=bonds, bond_k=bk, bond_r0=r0,
        angle=angles, angle_k=ak, angle_theta0=th0,
        tors=tors, tors_k=tk, tors_nrot=tn, tors_phase=tph,
        tors_div=np.ones(len(tors), np.int32), tors_nbf=nbf,
        impr=impr, impr_k=ik, impr_nrot=inr, impr_phase=iph,
        impr_div=np.ones(len(impr), np.int32),
        shake_n=sh_n, shake_atoms=sh_a, shake_dist=sh_d,
    )


def water_box(nwat, box, seed=1, jitter=0.3, temp=300.0):
    """`nwat` rigid 3-site waters; O on a simple-cubic lattice (+-jitter uniform)."""
    rng = np.random.default_rng(seed)
    top = _Top(rng)
    sites, _ = _lattice(box, nwat)
    pick = np.sort(rng.choice(len(sites), size=nwat, replace=False))
    for s in sites[pick]:
        _place_water(top, s + rng.uniform(-jitter, jitter, size=3), rng)
    return _finalize(top, np.full(3, float(box)), temp, rng)


def solvated_polymer(nres, nwat, box=None, seed=2, nion_pairs=0, temp=300.0, sphere=None):
    """A `nres`-residue chain plus `nwat` waters and Na+/Cl- (neutralising, plus
    `nion_pairs` extra pairs) in a cubic PBC box; with `sphere` (a radius) the chain is
    built inside a cube of half-edge 0.8 radius and the solvent fills the sphere only (a
    droplet around the box centre)."""
    rng = np.random.default_rng(seed)
    top = _Top(rng)
    if box is None:
        vol = (nwat + 4.0 * nres) / WATER_DENSITY
        # a unique minimum image needs box > 2 (rc + 1.5) = 27 A at the 12 A ZD cut-off
        box = max(vol ** (1.0 / 3.0), 28.0)
    pad = 2.0
    lo, hi = pad, box - pad
    if sphere is not None:
        lo, hi = 0.5 * box - 0.8 * sphere, 0.5 * box + 0.8 * sphere
    residues = _build_polymer(top, nres, lo, hi, rng, box) if nres else []
    nsol = len(top.pos)
    net = _charges_polymer(top, 0, nsol, residues, rng) if nres else 0
    n_na = nion_pairs + max(0, -net)
    n_cl = nion_pairs + max(0, net)
    need = nwat + n_na + n_cl
    sol = np.array(top.pos) if nsol else np.zeros((0, 3))
    ncube = need
    while True:
        sites, a = _lattice(box, ncube)
        if sphere is not None:
            sites = sites[np.linalg.norm(sites - 0.5 * box, axis=1) < sphere - 1.0]
        if nsol:
            ok = np.ones(len(sites), bool)
            for c0 in range(0, len(sites), 4096):
                d = sites[c0:c0 + 4096, None, :] - sol[None, :, :]
                d -= box * np.round(d / box)
                ok[c0:c0 + 4096] = (np.einsum("ijk,ijk->ij", d, d) > 2.6 ** 2).all(1)
            sites = sites[ok]
        if len(sites) >= need:
            break
        ncube = int(ncube * 1.1) + 1
    pick = rng.choice(len(sites), size=need, replace=False)
    jit = min(0.3, 0.1 * a)
    kinds = np.array([0] * nwat + [1] * n_na + [2] * n_cl)
    rng.shuffle(kinds)
    for s, kd in zip(sites[np.sort(pick)], kinds):
        p = s + rng.uniform(-jit, jit, size=3)
        if kd == 0:
            _place_water(top, p, rng)
        elif kd == 1:
            top.add(p, T_NA, 1.0, MOL_NA)
        else:
            top.add(p, T_CL, -1.0, MOL_CL)
    out = _finalize(top, np.full(3, float(box)), temp, rng)
    out["residues"] = [np.array(sorted(r["atoms"]), np.int32) for r in residues]
    return out


def droplet(nres, nwat, seed=6, temp=300.0):
    """A chain and `nwat` waters in a sphere at water density, for BOUNDA= NO (the box only
    holds the construction: periodic images are never near)."""
    vol = (nwat + 4.0 * nres) / WATER_DENSITY
    radius = (3.0 * vol / (4.0 * math.pi)) ** (1.0 / 3.0) + 1.5
    box = 2.0 * radius + 30.0
    return solvated_polymer(nres, nwat, box=box, seed=seed, temp=temp, sphere=radius)


HBOND_PAIRS = ((T_H, T_O), (T_H, T_OW), (T_HW, T_O))   # donor H -- acceptor O


def with_hbond(top, pairs=HBOND_PAIRS, r0=1.9, depth=0.5):
    """A copy of `top` whose type pairs `pairs` take the 10-12 H-bond term
    E = C12h/r^12 - C10/r^10 (iyppid = 2), with its minimum -depth kcal/mol at r0 A:
    C10 = 6 depth r0^10, C12h = C10 r0^2 / 1.2."""
    nt = int(top["ntype"])
    hb = np.zeros((nt, nt), np.int32)
    c10 = np.zeros((nt, nt))
    c12h = np.zeros((nt, nt))
    a10 = 6.0 * depth * r0 ** 10
    for i, j in pairs:
        for p, q in ((i, j), (j, i)):
            hb[p, q] = 1
            c10[p, q] = a10
            c12h[p, q] = a10 * r0 * r0 / 1.2
    return dict(top, hbond=hb, c10=c10, c12h=c12h)


def with_restraints(top, seed=3, cap=False, kt=0.596):
    """A copy of `top` with restraints on its solute, as psr/dsr/dhr files would give them
    (constants folded as md_run folds them, kt = boltzk * 300 K): position restraints on
    the first heavy atoms, pulled 0.3 A off their reference; distance restraints between
    solute atoms and atom pairs, half of them violated; dihedral restraints on backbone-like
    quadruples whose [lo, up] misses the current angle.  cap=True adds the sphere CAP of
    the included waters (centre of mass of each O-H-H triple) and of the solute heavy atoms
    around the centroid, for BOUNDA= NO."""
    rng = np.random.default_rng(seed)
    x = np.asarray(top["cord"], float)
    t = np.asarray(top["atype"])
    heavy = np.flatnonzero(np.isin(t, (T_C, T_N, T_O)))
    pos_atoms = heavy[:12]
    ref = x[pos_atoms] + rng.normal(size=(len(pos_atoms), 3)) * 0.3
    rd = dict(pos=(pos_atoms.astype(np.int32), np.full(len(pos_atoms), 5.0), ref))
    ig, jg, lo, up = [], [], [], []
    for k in range(6):
        a, b = heavy[3 * k], heavy[3 * k + 10]
        grp_i = [a] if k % 2 == 0 else [a, heavy[3 * k + 1]]
        grp_j = [b]
        r = np.linalg.norm(x[a] - x[b])
        ig.append(grp_i)
        jg.append(grp_j)
        if k % 3 == 0:
            lo.append(r + 1.0); up.append(r + 3.0)       # too short: the lower wall
        elif k % 3 == 1:
            lo.append(r - 4.0); up.append(r - 1.0)       # too long: the upper wall
        else:
            lo.append(r - 1.0); up.append(r + 1.0)       # satisfied
    nd = len(ig)
    dscc = kt * 0.5
    rd["dist"] = (ig, jg, np.array(lo), np.array(up), np.full(nd, dscc * 0.2), np.full(nd, dscc * 0.3))
    quads, dlo, dup = [], [], []
    for k in range(4):
        q = heavy[2 * k:2 * k + 4]
        b1, b2, b3 = x[q[1]] - x[q[0]], x[q[2]] - x[q[1]], x[q[3]] - x[q[2]]
        n1, n2 = np.cross(b1, b2), np.cross(b2, b3)
        phi = np.arctan2(np.dot(np.cross(n1, n2), b2) / np.linalg.norm(b2), np.dot(n1, n2)) % (2 * np.pi)
        w = np.radians(40.0)
        c0 = (phi + np.radians(60.0 + 30.0 * k)) % (2 * np.pi)   # a window away from phi
        quads.append(q)
        dlo.append(max(0.0, c0 - w / 2))
        dup.append(min(2 * np.pi - 1e-9, c0 + w / 2))
    nh = len(quads)
    dhk = kt * 1.0 / 2.0
    rd["dihe"] = (np.array(quads, np.int32), np.array(dlo), np.array(dup),
                  np.full(nh, dhk / np.radians(10.0) ** 2), np.full(nh, dhk / np.radians(10.0) ** 2))
    if cap:
        ow = np.flatnonzero(t == T_OW)
        centre = x.mean(0)
        rmax = np.linalg.norm(x - centre, axis=1).max()
        rd["cap"] = dict(center=centre, radius=0.85 * rmax, k=2.0,
                         groups=np.stack([ow, ow + 2], 1).astype(np.int32),
                         atoms=heavy.astype(np.int32), atom_radius=0.85 * rmax - 4.0, atom_k=2.0)
    return dict(top, restraints=rd)


def mcmd_weight(e_min, e_max, ndeg=8, t_lo=280.0, t_hi=700.0, tempce=300.0):
    """McMD .nf weight with d ln n/dE = 1/(R T(E)), T linear from t_lo at e_min to t_hi at
    e_max, fitted by a degree-`ndeg` polynomial in x = (E - celw)/(ceup - celw) and
    expressed in md_run's form: force scale = R*T0*P(x) (verlethe.f90:196-238)."""
    R = 8.31451 / 4.184 * 1e-3
    x = np.linspace(0.0, 1.0, 201)
    T = t_lo + (t_hi - t_lo) * x
    # R*T0*P = T0 / T  =>  P = 1/(R*T)
    P = 1.0 / (R * T)
    coef = np.polynomial.polynomial.polyfit(x, P, ndeg)
    return dict(nwindow=1, ndeg=ndeg, coef=coef.reshape(1, -1), low=np.array([0.0]),
                high=np.array([1.0 + 1e-12]), alphalw=1.0 / (R * t_lo),
                alphaup=1.0 / (R * t_hi), celw=float(e_min), ceup=float(e_max),
                tempce=float(tempce))


# ---- the five configurations ------------------------------------------------------------
def config_c1(seed=1):
    """3,000 waters (9,000 atoms) in a 31.0 A box: as specified, ~3x liquid density."""
    return water_box(3000, 31.0, seed=seed)


def config_c1_prime(seed=1):
    """1,000 waters in the same 31.0 A box (10^3 lattice, 3.1 A spacing): liquid density,
    used for the NVE drift measurement."""
    return water_box(1000, 31.0, seed=seed)


def config_c2(seed=2):
    """159-residue chain + 7,000 waters + neutralising ions, 62 A box (~23k atoms)."""
    return solvated_polymer(159, 7000, box=62.0, seed=seed)


def config_c3(seed=3):
    """33,000 waters + 100 Na+ + 100 Cl- (~99,200 atoms) in a 100 A box."""
    return solvated_polymer(0, 33000, box=100.0, seed=seed, nion_pairs=100)


def _c4_one(args):
    nres, nwat, seed = args
    return solvated_polymer(nres, nwat, seed=seed)


def config_c4(nrep=64, seed=4, small=False, workers=None):
    """64 uneven replicas: 8-30-residue chains in 600-9,000 waters (2k-30k atoms).
    small=True shrinks the water counts tenfold for CPU tests.  workers > 1 builds the
    replicas in a process pool started with `spawn` (safe next to CUDA)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for r in range(nrep):
        nres = int(rng.integers(8, 31))
        nwat = int(rng.integers(600, 9001))
        if small:
            nwat = max(300, nwat // 10)
        jobs.append((nres, nwat, seed * 1000 + r))
    if workers and workers > 1:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            return list(ex.map(_c4_one, jobs))
    return [_c4_one(j) for j in jobs]


def alsd_replica(top, ncluster=4, seed=0, walls=20.0):
    """A copy of a solvated chain set up for ALSD (CLSTMETHOD= LMD, METHOD= GE): the atoms
    of `ncluster` residues drawn from the seed form the lambda-scaled cluster (whole SHAKE
    groups, as residue lists give them), and the weight in lambda is linear on [0.6, 1.0]
    (d lnP/dlambda = 40 - 30 lambda) with restoring walls of slope `walls` outside (lower
    -walls, upper +walls: below celw d lnP/dlambda falls, above ceup it rises, and the force
    on lambda, -dE/dlambda - R T d lnP/dlambda, points back into the range)."""
    rng = np.random.default_rng(seed)
    t = dict(top)
    cl = np.zeros(t["natom"], np.int32)
    for r in rng.choice(len(t["residues"]), size=min(ncluster, len(t["residues"])), replace=False):
        cl[t["residues"][r]] = 1
    for g, na in zip(t["shake_atoms"], t["shake_n"]):
        if cl[g[:na]].any():
            cl[g[:na]] = 1
    t["cluster"] = cl
    t["ge"] = dict(coef=np.array([[40.0, -30.0]]), low=np.array([0.0]), high=np.array([2.0]),
                   alphalw=0.0, alphaup=0.0, celw=0.6, ceup=1.0, tempce=300.0, lower=-float(walls),
                   upper=float(walls))
    return t


def _c5_one(args):
    nwat, seed = args
    return alsd_replica(solvated_polymer(12, nwat, seed=seed), seed=seed)


def config_c5(nrep=32, seed=5, nwat=3000, workers=None):
    """32 replicas of a 12-residue chain in 3,000 waters (~9,200 atoms each), each with an
    ALSD cluster of 4 seeded residues and a weight in lambda on [0.6, 1.0] (alsd_replica).
    workers > 1 builds them in a process pool started with `spawn`."""
    jobs = [(nwat, seed * 1000 + r) for r in range(nrep)]
    if workers and workers > 1:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            return list(ex.map(_c5_one, jobs))
    return [_c5_one(j) for j in jobs]
