"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU FP64 oracle (oracle.cpp).

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.
The product path (j_presto_b200) never imports this package.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from j_presto_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(
                os.path.join(_HERE, "oracle.cpp")):
            build()
        L = C.CDLL(_LIB)
        vp, dp = C.c_void_p, C.POINTER(C.c_double)
        L.or_create.restype = vp
        L.or_create.argtypes = [C.POINTER(abi.JpSystem), C.POINTER(abi.JpParams), C.c_int]
        L.or_destroy.argtypes = [vp]
        L.or_set_state.argtypes = [vp, dp, dp]
        L.or_get_state.argtypes = [vp, dp, dp]
        L.or_rebuild.argtypes = [vp]
        L.or_npairs_listed.argtypes = [vp]
        L.or_npairs_listed.restype = C.c_longlong
        L.or_npairs_cut.argtypes = [vp]
        L.or_npairs_cut.restype = C.c_longlong
        L.or_dself.argtypes = [vp]
        L.or_dself.restype = C.c_double
        L.or_dof.argtypes = [vp]
        L.or_dof.restype = C.c_int
        L.or_energy_grad.argtypes = [vp, dp, dp, dp]
        L.or_energy_grad_cls.argtypes = [vp, dp, dp, dp, dp]
        L.or_shake.argtypes = [vp, dp, dp]
        L.or_temperature.argtypes = [vp, dp]
        L.or_temperature.restype = C.c_double
        L.or_run.argtypes = [vp, C.c_int, dp, dp]
        L.or_first_force.argtypes = [vp, dp, dp, dp]
        L.or_first_force.restype = None
        ipp = C.POINTER(C.c_int)
        L.or_minimize.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                  ipp, dp, dp, ipp]
        L.or_minimize_conj.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                       ipp, dp, dp, ipp]
        L.or_mcmd_scale.argtypes = [vp, C.c_double]
        L.or_mcmd_scale.restype = C.c_double
        L.or_get_lambda.argtypes = [vp, dp, dp]
        L.or_get_lambda.restype = None
        L.or_set_lambda.argtypes = [vp, C.c_double, C.c_double]
        L.or_set_lambda.restype = None
        L.or_remotv.argtypes = [vp, dp, dp]
        L.or_nfrmol.argtypes = [vp, dp]
        L.or_cmm_level.argtypes = [vp, C.c_int, dp, C.POINTER(C.c_int), dp]
        L.or_cmm_nlev.argtypes = [vp]
        L.or_cmm_far.argtypes = [vp, dp]
        L.or_cmm_far.restype = C.c_double
        _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """One replica of the reference algorithm on the host cores."""

    def __init__(self, top, params=None, nthreads=0, **kw):
        self._keep = []
        self.top = top
        self.n = int(top["natom"])
        self.params = params if params is not None else abi.default_params(**kw)
        hb = top.get("hbond")
        if hb is not None and np.any(hb) and self.params.cal15m == abi.JP_CAL15M_CMM:
            raise ValueError("the H-bond 10-12 pairs are restated for CAL15M= ZD and ATOM only")
        self._sys = abi.make_system(top, self._keep)
        self._h = lib().or_create(C.byref(self._sys), C.byref(self.params), int(nthreads))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_destroy(self._h)
            self._h = None

    def set_state(self, cord=None, vel=None):
        c = None if cord is None else np.ascontiguousarray(cord, np.float64)
        v = None if vel is None else np.ascontiguousarray(vel, np.float64)
        lib().or_set_state(self._h, _dp(c), _dp(v))

    def get_state(self):
        c = np.empty((self.n, 3))
        v = np.empty((self.n, 3))
        lib().or_get_state(self._h, _dp(c), _dp(v))
        return c, v

    def rebuild(self):
        lib().or_rebuild(self._h)

    def energy_grad(self, cord=None):
        c = None if cord is None else np.ascontiguousarray(cord, np.float64)
        e = np.zeros(abi.JP_MAXENE)
        g = np.zeros((self.n, 3))
        lib().or_energy_grad(self._h, _dp(c), _dp(e), _dp(g))
        return e, g

    def energy_grad_cls(self, cord=None):
        """dnergy's per-class outputs: (eneval, class totals [nfrg], unscaled gradients
        [nfrg, natom, 3]); nfrg = 1 without clusters, 3 for ALSD, 2 for GEPSME= AND/OR/XOR."""
        c = None if cord is None else np.ascontiguousarray(cord, np.float64)
        e = np.zeros(abi.JP_MAXENE)
        ec = np.zeros(3)
        g = np.zeros((3, self.n, 3))
        nfrg = lib().or_energy_grad_cls(self._h, _dp(c), _dp(e), _dp(ec), _dp(g))
        return e, ec[:nfrg].copy(), g[:nfrg].copy()

    def shake(self, r1, r2):
        r1 = np.ascontiguousarray(r1, np.float64).copy()
        r2 = np.ascontiguousarray(r2, np.float64)
        ier = lib().or_shake(self._h, _dp(r1), _dp(r2))
        return ier, r1

    def temperature(self, vel=None):
        v = None if vel is None else np.ascontiguousarray(vel, np.float64)
        return lib().or_temperature(self._h, _dp(v))

    def run(self, nsteps):
        e = np.zeros((nsteps, abi.JP_MAXENE))
        t = np.zeros(nsteps)
        ier = lib().or_run(self._h, int(nsteps), _dp(e), _dp(t))
        return ier, e, t

    @property
    def npairs_listed(self):
        return lib().or_npairs_listed(self._h)

    @property
    def npairs_cut(self):
        return lib().or_npairs_cut(self._h)

    @property
    def dself(self):
        return lib().or_dself(self._h)

    @property
    def dof(self):
        return lib().or_dof(self._h)

    def mcmd_scale(self, e):
        return lib().or_mcmd_scale(self._h, float(e))

    def get_lambda(self):
        """(lambda, lambda velocity), class energies (AA, AB, BB) of the last force call."""
        l2, ec = np.zeros(2), np.zeros(3)
        lib().or_get_lambda(self._h, _dp(l2), _dp(ec))
        return l2, ec

    def first_force(self):
        """(eneval, lambda_f, grad) as md_run's FDEBUG dumps them at the first step: the
        gradient after verlethe's scaling (pseudo temperature, McMD weight, ALSD classes)."""
        e = np.zeros(abi.JP_MAXENE)
        g = np.zeros((self.n, 3))
        lf = C.c_double()
        lib().or_first_force(self._h, _dp(e), C.byref(lf), _dp(g))
        return e, lf.value, g

    def minimize(self, max_loop=1000, update=10, convgr=0.1, step0=0.01, up=1.2, down=0.6):
        """steep (steep.f90) on this replica: (ier, iters, energies, rms gradient, state)."""
        it, st = C.c_int(), C.c_int()
        e = np.zeros(abi.JP_MAXENE)
        rm = C.c_double()
        ier = lib().or_minimize(self._h, int(max_loop), int(update), float(convgr), float(step0),
                                float(up), float(down), C.byref(it), _dp(e), C.byref(rm), C.byref(st))
        return ier, it.value, e, rm.value, st.value

    def minimize_conj(self, max_loop=1000, update=10, convgr=0.1, step0=0.01, line_conv=0.1,
                      line_max=10):
        """conj (conj.f90) on this replica: (ier, iters, energies, rms gradient, state)."""
        it, st = C.c_int(), C.c_int()
        e = np.zeros(abi.JP_MAXENE)
        rm = C.c_double()
        ier = lib().or_minimize_conj(self._h, int(max_loop), int(update), float(convgr), float(step0),
                                     float(line_conv), int(line_max), C.byref(it), _dp(e), C.byref(rm),
                                     C.byref(st))
        return ier, it.value, e, rm.value, st.value

    def set_lambda(self, lam, lam_v=0.0):
        lib().or_set_lambda(self._h, float(lam), float(lam_v))

    def remotv(self, xp, vel):
        """remotv applied to a copy of `vel` with positions `xp`; (ier, new velocities)."""
        v = np.ascontiguousarray(vel, np.float64).copy()
        ier = lib().or_remotv(self._h, _dp(np.ascontiguousarray(xp, np.float64)), _dp(v))
        return ier, v

    def cmm_levels(self):
        """Per CMM level (1..nlev): (multipoles [nv^3][13], populations [nv^3], centres
        [nv][3]); cells x fastest."""
        out = []
        for l in range(1, lib().or_cmm_nlev(self._h) + 1):
            nv = lib().or_cmm_level(self._h, l, None, None, None)
            pot = np.zeros((nv ** 3, 13))
            pop = np.zeros(nv ** 3, np.int32)
            cen = np.zeros((nv, 3))
            lib().or_cmm_level(self._h, l, _dp(pot), pop.ctypes.data_as(C.POINTER(C.c_int)),
                               _dp(cen))
            out.append((pot, pop, cen))
        return out

    def cmm_far(self):
        """(far-field energy, its gradient [natom][3]) of the last force call (CMM)."""
        g = np.zeros((self.n, 3))
        e = lib().or_cmm_far(self._h, _dp(g))
        return e, g

    def nfrmol(self):
        n = lib().or_nfrmol(self._h, None)
        out = np.zeros(n)
        lib().or_nfrmol(self._h, _dp(out))
        return out
