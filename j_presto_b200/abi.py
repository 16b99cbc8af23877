"""ctypes mirror of include/jpgpu.h (the C ABI that replaces md_run's call sites).

`make_system` turns a topology dict (numpy arrays, see `systems.py`) into a `JpSystem`
struct whose pointers stay valid as long as the returned keep-alive list lives.
"""
import ctypes as C

import numpy as np

JP_MAXENE = 15
JP_E_TOTAL, JP_E_VDW14, JP_E_VDW15, JP_E_ELE15, JP_E_HBOND = 0, 5, 7, 8, 9   # eneval slots
JP_E_POSRES, JP_E_DISTRES, JP_E_DIHERES, JP_E_CAP = 10, 11, 12, 13
JP_PREC_FP64, JP_PREC_MIXED = 0, 1
JP_METHOD_CONS, JP_METHOD_MICR, JP_METHOD_CANO, JP_METHOD_GE = 1, 2, 3, 4
JP_SHAKE_NONE, JP_SHAKE_HBON, JP_SHAKE_ALLB = 0, 1, 2
JP_ALSD_NONE, JP_ALSD_LMD, JP_ALSD_LMD2 = 0, 1, 2
JP_GEPS_AND, JP_GEPS_OR, JP_GEPS_XOR = 3, 4, 5
JP_SCALE_BOND, JP_SCALE_ANGLE, JP_SCALE_TORS, JP_SCALE_IMPR = 1, 2, 4, 8
JP_STOP_TRANS, JP_STOP_ROT, JP_STOP_BOTH, JP_STOP_NONE = 1, 2, 3, 4
JP_CAL15M_CMM, JP_CAL15M_ATOM, JP_CAL15M_ZD = 1, 2, 4
JP_BOUND_NONE, JP_BOUND_PBC = 0, 1
# return codes (md_run ier convention: >0 warning, <0 fatal)
JP_OK = 0
JP_W_SHAKE_NOT_CONVERGED = 1
JP_E_SHAKE_SINGULAR = -2
JP_E_SHAKE_ABORT = -9999
JP_E_INVALID = -100
JP_E_LIST_OVERFLOW = -151
JP_E_NONFINITE = -200
JP_E_FIXED_OVERFLOW = -201
JP_E_CELL_OVERFLOW = -128
JP_E_TIMEOUT = -302
JP_E_CUDA = -300
JP_E_NO_DEVICE = -301
JP_E_NOALLOC_LIMIT = -110
JP_E_STOP_MASS = -121
JP_E_STOP_SINGULAR = -122
JP_E_FREE_WINDOW = -130
JP_NOALLOC_MAX_ATOMS = 16384
JP_TUNE_CANDIDATES = 5           # column-edge factors tried by the block-shape tuner
JP_ALSD_MAX_LBINS, JP_ALSD_MAX_EBINS = 64, 256

# energy slot names (md_run main.f90:157-159 cyenam order)
ENERGY_NAMES = ["TOTAL", "BOND", "ANGLE", "TORSION", "IMPROPER", "VDW14", "ELEC14",
                "VDW15", "ELEC15", "HBOND", "VDW15_NC", "ELEC15_NC", "HBOND_NC",
                "POSRES", "DISRES"]

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class JpGe(C.Structure):
    _fields_ = [("nwindow", C.c_int32), ("ndeg", C.c_int32),
                ("coef", _dp), ("low", _dp), ("high", _dp),
                ("alphalw", C.c_double), ("alphaup", C.c_double),
                ("celw", C.c_double), ("ceup", C.c_double),
                ("tempce", C.c_double), ("lower", C.c_double), ("upper", C.c_double)]


class JpExtCmm(C.Structure):
    _fields_ = [("nlev", C.c_int32), ("cell", C.c_double), ("center", C.c_double * 3),
                ("flag", C.POINTER(C.c_uint8)), ("pot", _dp)]


JP_GE_MAX_WINDOWS, JP_GE_MAX_DEG, JP_GE_MAX_BINS = 16, 15, 4096


class JpGeFitParams(C.Structure):
    _fields_ = [("emin", C.c_double), ("emax", C.c_double), ("nbin", C.c_int32), ("nbor", C.c_int32),
                ("next_emin", C.c_double), ("next_emax", C.c_double), ("next_temp", C.c_double),
                ("nwindow", C.c_int32), ("ndeg", C.c_int32), ("ignore_empty", C.c_int32),
                ("neglect_low", C.c_int32), ("neglect_high", C.c_int32)]


class JpRestraints(C.Structure):
    _fields_ = [
        ("npos", C.c_int32), ("pos_atom", _ip), ("pos_k", _dp), ("pos_ref", _dp),
        ("ndist", C.c_int32), ("dist_iptr", _ip), ("dist_iatom", _ip), ("dist_jptr", _ip),
        ("dist_jatom", _ip), ("dist_lo", _dp), ("dist_up", _dp), ("dist_klo", _dp), ("dist_kup", _dp),
        ("ndihe", C.c_int32), ("dihe_atom", _ip), ("dihe_lo", _dp), ("dihe_up", _dp),
        ("dihe_klo", _dp), ("dihe_kup", _dp),
        ("ncap_group", C.c_int32), ("cap_group", _ip), ("ncap_atom", C.c_int32), ("cap_atom", _ip),
        ("cap_center", C.c_double * 3), ("cap_radius", C.c_double), ("cap_k", C.c_double),
        ("cap_atom_radius", C.c_double), ("cap_atom_k", C.c_double),
        ("cap_shape", C.c_int32), ("cap_wall", C.c_double * 6), ("cap_atom_wall", C.c_double * 6),
        ("cap_ellipse", C.c_double * 3), ("cap_atom_ellipse", C.c_double * 3),
        ("cap_function", C.c_int32),
    ]


JP_MIN_STEEP, JP_MIN_CONJ = 1, 2
JP_CAP_SPHERE, JP_CAP_BOX, JP_CAP_ELLIPSOID = 1, 2, 3
JP_CAP_HARMONIC, JP_CAP_BIQUADRATIC = 1, 2
JP_E_MIN_STEP = -140


class JpMinParams(C.Structure):
    _fields_ = [("method", C.c_int32), ("max_loop", C.c_int32), ("update", C.c_int32),
                ("convgr", C.c_double), ("step0", C.c_double), ("up", C.c_double), ("down", C.c_double),
                ("line_conv", C.c_double), ("line_max", C.c_int32)]


def min_params(**kw):
    """jp_min_params with md_run's EXE> MIN defaults (inpmin.f90), overridden by kw."""
    p = JpMinParams(method=JP_MIN_STEEP, max_loop=1000, update=10, convgr=0.1, step0=0.01, up=1.2,
                    down=0.6, line_conv=0.1, line_max=10)
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


class JpSystem(C.Structure):
    _fields_ = [
        ("natom", C.c_int32), ("index_base", C.c_int32), ("box", C.c_double * 3),
        ("cord", _dp), ("vel", _dp), ("mass", _dp), ("charge", _dp),
        ("atype", _ip), ("molecule", _ip),
        ("ntype", C.c_int32), ("c6", _dp), ("c12", _dp), ("s14_vdw", _dp), ("s14_ele", _dp),
        ("excl_ptr", _ip), ("excl_idx", _ip),
        ("nbond", C.c_int32), ("bond", _ip), ("bond_k", _dp), ("bond_r0", _dp),
        ("nangle", C.c_int32), ("angle", _ip), ("angle_k", _dp), ("angle_theta0", _dp),
        ("ntors", C.c_int32), ("tors", _ip), ("tors_k", _dp), ("tors_nrot", _dp),
        ("tors_phase", _dp), ("tors_div", _ip), ("tors_nbf", _ip),
        ("nimpr", C.c_int32), ("impr", _ip), ("impr_k", _dp), ("impr_nrot", _dp),
        ("impr_phase", _dp), ("impr_div", _ip),
        ("nshake", C.c_int32), ("shake_n", _ip), ("shake_atoms", _ip), ("shake_dist", _dp),
        ("ge", C.POINTER(JpGe)), ("cluster", _ip), ("ext_cmm", C.POINTER(JpExtCmm)),
        ("hbond", _ip), ("c10", _dp), ("c12h", _dp), ("restraints", C.POINTER(JpRestraints)),
        ("tors_unscaled", _ip), ("ncelres", C.c_int32), ("celres", _ip),
    ]


class JpParams(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("method", C.c_int32), ("dt", C.c_double),
        ("cutoff", C.c_double), ("dielectric", C.c_double), ("update", C.c_int32),
        ("temp", C.c_double), ("temp_start", C.c_double), ("heat_loop", C.c_int32),
        ("tempco", C.c_int32), ("shake_method", C.c_int32), ("shake_tol", C.c_double),
        ("shake_maxit", C.c_int32), ("icslop", C.c_int32), ("fcstol", C.c_double),
        ("psetmp", C.c_double), ("device", C.c_int32),
        ("alsd", C.c_int32), ("lambda0", C.c_double), ("lambda_mass", C.c_double),
        ("lambda_temp_control", C.c_int32), ("scale_terms", C.c_int32),
        ("taut", C.c_double), ("stop_center", C.c_int32), ("stop_natom", C.c_int32),
        ("cal15m", C.c_int32), ("bounda", C.c_int32), ("cmm_levels", C.c_int32),
        ("cmm_cell", C.c_double), ("cmm_update", C.c_int32), ("tune_blocks", C.c_int32),
    ]


def default_params(**kw):
    """md_run defaults (inpmd.f90:120-160, main.f90:134-174) plus keyword overrides."""
    p = JpParams(precision=JP_PREC_MIXED, method=JP_METHOD_CANO, dt=2.0, cutoff=12.0,
                 dielectric=1.0, update=10, temp=300.0, temp_start=300.0, heat_loop=0,
                 tempco=2, shake_method=JP_SHAKE_HBON, shake_tol=1e-6, shake_maxit=1000,
                 icslop=3, fcstol=1e-3, psetmp=0.0, device=0, alsd=JP_ALSD_NONE, lambda0=1.0,
                 lambda_mass=0.0, lambda_temp_control=0, scale_terms=0, taut=40.0,
                 stop_center=JP_STOP_NONE, stop_natom=0, cal15m=JP_CAL15M_ZD,
                 bounda=JP_BOUND_PBC, cmm_levels=3, cmm_cell=6.0, cmm_update=5, tune_blocks=1)
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def _ptr(a, ctype, keep):
    if a is None:
        return None
    dt = np.float64 if ctype is C.c_double else np.int32
    a = np.ascontiguousarray(a, dtype=dt)
    keep.append(a)
    return a.ctypes.data_as(C.POINTER(ctype))


def make_system(top, keep, cord=None, vel=None):
    """Build a JpSystem from a topology dict; arrays are appended to `keep`."""
    s = JpSystem()
    s.natom = int(top["natom"])
    s.index_base = 0
    for k in range(3):
        s.box[k] = float(top["box"][k])
    s.cord = _ptr(top["cord"] if cord is None else cord, C.c_double, keep)
    v = top.get("vel") if vel is None else vel
    s.vel = _ptr(v, C.c_double, keep)
    s.mass = _ptr(top["mass"], C.c_double, keep)
    s.charge = _ptr(top["charge"], C.c_double, keep)
    s.atype = _ptr(top["atype"], C.c_int32, keep)
    s.molecule = _ptr(top.get("molecule"), C.c_int32, keep)
    s.ntype = int(top["ntype"])
    s.c6 = _ptr(top["c6"], C.c_double, keep)
    s.c12 = _ptr(top["c12"], C.c_double, keep)
    s.s14_vdw = _ptr(top["s14_vdw"], C.c_double, keep)
    s.s14_ele = _ptr(top["s14_ele"], C.c_double, keep)
    s.excl_ptr = _ptr(top["excl_ptr"], C.c_int32, keep)
    s.excl_idx = _ptr(top["excl_idx"] if len(top["excl_idx"]) else np.zeros(1, np.int32),
                      C.c_int32, keep)

    def seg(name, cols, fields):
        arr = top[name]
        n = len(arr) // cols if np.ndim(arr) == 1 else len(arr)
        setattr(s, "n" + name, n)
        setattr(s, name, _ptr(np.asarray(arr).reshape(-1) if n else np.zeros(cols, np.int32),
                              C.c_int32, keep))
        for f, ct in fields:
            val = top[f] if n else np.zeros(1)
            setattr(s, f, _ptr(val, ct, keep))

    seg("bond", 2, [("bond_k", C.c_double), ("bond_r0", C.c_double)])
    seg("angle", 3, [("angle_k", C.c_double), ("angle_theta0", C.c_double)])
    seg("tors", 4, [("tors_k", C.c_double), ("tors_nrot", C.c_double),
                    ("tors_phase", C.c_double), ("tors_div", C.c_int32),
                    ("tors_nbf", C.c_int32)])
    seg("impr", 4, [("impr_k", C.c_double), ("impr_nrot", C.c_double),
                    ("impr_phase", C.c_double), ("impr_div", C.c_int32)])
    sh_n = np.asarray(top["shake_n"], np.int32)
    s.nshake = len(sh_n)
    s.shake_n = _ptr(sh_n if len(sh_n) else np.zeros(1, np.int32), C.c_int32, keep)
    s.shake_atoms = _ptr(np.asarray(top["shake_atoms"]).reshape(-1) if len(sh_n)
                         else np.zeros(4, np.int32), C.c_int32, keep)
    s.shake_dist = _ptr(np.asarray(top["shake_dist"]).reshape(-1) if len(sh_n)
                        else np.zeros(6), C.c_double, keep)
    cl = top.get("cluster")
    s.cluster = None if cl is None else _ptr(np.asarray(cl, np.int32), C.c_int32, keep)
    ex = top.get("ext_cmm")   # dict(nlev, cell, center[3], flag[nv^3] 0/1, pot[nv^3][13])
    if ex is not None:
        flag = np.ascontiguousarray(np.asarray(ex["flag"]).reshape(-1), np.uint8)
        pot = np.ascontiguousarray(np.asarray(ex["pot"], np.float64).reshape(-1))
        keep += [flag, pot]
        e = JpExtCmm(nlev=int(ex["nlev"]), cell=float(ex["cell"]),
                     center=(C.c_double * 3)(*[float(v) for v in ex["center"]]),
                     flag=flag.ctypes.data_as(C.POINTER(C.c_uint8)),
                     pot=pot.ctypes.data_as(_dp))
        keep.append(e)
        s.ext_cmm = C.pointer(e)
    if top.get("hbond") is not None:   # [ntype][ntype] 0/1 flags and the 10-12 tables
        s.hbond = _ptr(np.asarray(top["hbond"], np.int32), C.c_int32, keep)
        s.c10 = _ptr(top["c10"], C.c_double, keep)
        s.c12h = _ptr(top["c12h"], C.c_double, keep)
    if top.get("celres") is not None:   # [n][2] first / last atom of each CELRES residue
        cr = np.asarray(top["celres"], np.int32).reshape(-1, 2)
        s.ncelres = len(cr)
        s.celres = _ptr(cr.reshape(-1), C.c_int32, keep)
    if top.get("tors_unscaled") is not None:
        s.tors_unscaled = _ptr(top["tors_unscaled"], C.c_int32, keep)
    if top.get("restraints") is not None:
        s.restraints = C.pointer(make_restraints(top["restraints"], keep))
    ge = top.get("ge")
    if ge is not None:
        g = make_ge(ge, keep)
        keep.append(g)
        s.ge = C.pointer(g)
    return s


def make_restraints(rd, keep):
    """JpRestraints from a dict: pos=(atoms, k, ref[n][3]); dist=(igroups, jgroups, lo, up,
    klo, kup) with the groups as lists of atom lists; dihe=(atoms[n][4], lo, up, klo, kup);
    cap=dict(center, radius, k, groups[n][2] first/last atom, atoms, atom_radius, atom_k)."""
    r = JpRestraints()
    if rd.get("pos") is not None:
        atoms, k, ref = rd["pos"]
        r.npos = len(atoms)
        r.pos_atom = _ptr(atoms, C.c_int32, keep)
        r.pos_k = _ptr(k, C.c_double, keep)
        r.pos_ref = _ptr(np.asarray(ref, np.float64).reshape(-1), C.c_double, keep)
    if rd.get("dist") is not None:
        ig, jg, lo, up, klo, kup = rd["dist"]
        r.ndist = len(ig)
        r.dist_iptr = _ptr(np.concatenate([[0], np.cumsum([len(g) for g in ig])]), C.c_int32, keep)
        r.dist_iatom = _ptr(np.concatenate([np.asarray(g, np.int32) for g in ig]), C.c_int32, keep)
        r.dist_jptr = _ptr(np.concatenate([[0], np.cumsum([len(g) for g in jg])]), C.c_int32, keep)
        r.dist_jatom = _ptr(np.concatenate([np.asarray(g, np.int32) for g in jg]), C.c_int32, keep)
        r.dist_lo, r.dist_up = _ptr(lo, C.c_double, keep), _ptr(up, C.c_double, keep)
        r.dist_klo, r.dist_kup = _ptr(klo, C.c_double, keep), _ptr(kup, C.c_double, keep)
    if rd.get("dihe") is not None:
        atoms, lo, up, klo, kup = rd["dihe"]
        r.ndihe = len(atoms)
        r.dihe_atom = _ptr(np.asarray(atoms, np.int32).reshape(-1), C.c_int32, keep)
        r.dihe_lo, r.dihe_up = _ptr(lo, C.c_double, keep), _ptr(up, C.c_double, keep)
        r.dihe_klo, r.dihe_kup = _ptr(klo, C.c_double, keep), _ptr(kup, C.c_double, keep)
    cap = rd.get("cap")
    if cap is not None:
        groups = np.asarray(cap.get("groups", np.zeros((0, 2))), np.int32).reshape(-1, 2)
        atoms = np.asarray(cap.get("atoms", []), np.int32)
        r.ncap_group = len(groups)
        r.cap_group = _ptr(groups.reshape(-1), C.c_int32, keep) if len(groups) else None
        r.ncap_atom = len(atoms)
        r.cap_atom = _ptr(atoms, C.c_int32, keep) if len(atoms) else None
        r.cap_center[:] = [float(v) for v in cap["center"]]
        r.cap_radius, r.cap_k = float(cap["radius"]), float(cap["k"])
        r.cap_atom_radius = float(cap.get("atom_radius", 0.0))
        r.cap_atom_k = float(cap.get("atom_k", 0.0))
        r.cap_shape = int(cap.get("shape", JP_CAP_SPHERE))   # box: wall / atom_wall [6];
        r.cap_function = int(cap.get("function", JP_CAP_HARMONIC))
        for key, n in (("wall", 6), ("atom_wall", 6), ("ellipse", 3), ("atom_ellipse", 3)):
            if key in cap:                                   # ellipsoid: ellipse / atom_ellipse [3]
                getattr(r, "cap_" + key)[:] = [float(v) for v in np.ravel(cap[key])][:n]
    keep.append(r)
    return r


def make_systems(tops, keep):
    """Array of JpSystem for several replicas."""
    arr = (JpSystem * len(tops))()
    for i, t in enumerate(tops):
        arr[i] = make_system(t, keep)
    return arr


def make_ge(nf, keep):
    """JpGe from a weight dict {coef [nwin][ndeg+1], low, high, alphalw, alphaup, celw, ceup,
    tempce[, lower, upper]}; arrays appended to `keep`."""
    g = JpGe()
    coef = np.asarray(nf["coef"], np.float64)
    nwin = int(nf.get("nwindow", coef.shape[0] if coef.ndim == 2 else 1))
    coef = np.ascontiguousarray(coef.reshape(nwin, -1))
    g.nwindow, g.ndeg = nwin, coef.shape[1] - 1
    g.coef = _ptr(coef, C.c_double, keep)
    g.low = _ptr(np.ascontiguousarray(nf["low"], np.float64), C.c_double, keep)
    g.high = _ptr(np.ascontiguousarray(nf["high"], np.float64), C.c_double, keep)
    for k in ("alphalw", "alphaup", "celw", "ceup", "tempce"):
        setattr(g, k, float(nf[k]))
    g.lower, g.upper = float(nf.get("lower", 0.0)), float(nf.get("upper", 0.0))
    return g
