"""Shared helpers for the test suite (not part of the product)."""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_golden():
    with open(os.path.join(HERE, "golden", "kat.json")) as f:
        return json.load(f)


def golden_top(sysd):
    """Topology dict (abi.make_system format) from a golden-vector system description."""
    n = sysd["natom"]
    excl = sysd["excl"]
    ptr = np.zeros(n + 1, np.int32)
    for i in range(n):
        ptr[i + 1] = ptr[i] + len(excl[i])
    idx = np.array([j for e in excl for j in sorted(e)], np.int32)
    t = dict(natom=n, box=np.array(sysd["box"], float), cord=np.array(sysd["cord"], float),
             vel=np.zeros((n, 3)), mass=np.array(sysd["mass"], float),
             charge=np.array(sysd["charge"], float), atype=np.array(sysd["atype"], np.int32),
             molecule=np.zeros(n, np.int32), ntype=sysd["ntype"],
             c6=np.array(sysd["c6"], float), c12=np.array(sysd["c12"], float),
             s14_vdw=np.array(sysd["s14_vdw"], float), s14_ele=np.array(sysd["s14_ele"], float),
             excl_ptr=ptr, excl_idx=idx,
             bond=np.array(sysd["bond"], np.int32).reshape(-1, 2),
             bond_k=np.array(sysd["bond_k"], float), bond_r0=np.array(sysd["bond_r0"], float),
             angle=np.array(sysd["angle"], np.int32).reshape(-1, 3),
             angle_k=np.array(sysd["angle_k"], float),
             angle_theta0=np.array(sysd["angle_theta0"], float),
             tors=np.array(sysd["tors"], np.int32).reshape(-1, 4),
             tors_k=np.array(sysd["tors_k"], float), tors_nrot=np.array(sysd["tors_nrot"], float),
             tors_phase=np.array(sysd["tors_phase"], float),
             tors_div=np.array(sysd["tors_div"], np.int32),
             tors_nbf=np.array(sysd["tors_nbf"], np.int32),
             impr=np.zeros((0, 4), np.int32), impr_k=np.zeros(0), impr_nrot=np.zeros(0),
             impr_phase=np.zeros(0), impr_div=np.zeros(0, np.int32),
             shake_n=np.zeros(0, np.int32), shake_atoms=np.zeros((0, 4), np.int32),
             shake_dist=np.zeros((0, 6)))
    return t


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))
