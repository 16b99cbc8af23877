"""Python host binding of libjpgpu.so (the C ABI in include/jpgpu.h).

`Engine` mirrors the md_run call sites the ABI replaces: celprp -> rebuild(), dnergy ->
energy_grad(), verlet/verlethe loop -> step(), shake_PB -> shake(), restart/monitor state
-> get_state()/set_state().  Errors raise `JpError` carrying md_run's ier convention.
There is no CPU fallback: without the CUDA library or a GPU the constructor raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libjpgpu.so")
_lib = None

# every symbol the header declares
EXPORTS = ["jp_default_params", "jp_create", "jp_rebuild_cells", "jp_energy_grad", "jp_step",
           "jp_shake", "jp_get_state", "jp_set_state", "jp_pair_count", "jp_set_timing",
           "jp_last_timing", "jp_launch_counts", "jp_list_stats", "jp_calibrate_fp32",
           "jp_strerror", "jp_destroy", "jp_nonbond_noalloc", "jp_ge_hist_setup",
           "jp_ge_hist_get", "jp_ge_set", "jp_lstsq_windows", "jp_ge_fit", "jp_ge_dlnn",
           "jp_mlp_nparam", "jp_mlp_init", "jp_mlp_train", "jp_mlp_forward", "jp_ge_set_mlp",
           "jp_get_lambda", "jp_set_lambda", "jp_set_grid_limit", "jp_default_min_params",
           "jp_minimize", "jp_set_wait_limit", "jp_step_io", "jp_tile_shape", "jp_alsd_hist_setup",
           "jp_alsd_hist_get", "jp_alsd_set_mlp", "jp_energy_grad_cls"]


class JpError(RuntimeError):
    def __init__(self, code, where):
        self.code = code
        msg = lib().jp_strerror(code).decode() if _lib is not None else str(code)
        super().__init__(f"{where}: {msg} (code {code})")


def lib():
    """Load libjpgpu.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run `python -m j_presto_b200.build` first")
        L = C.CDLL(LIB_PATH)
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.c_int32
        L.jp_default_params.argtypes = [C.POINTER(abi.JpParams)]
        L.jp_default_params.restype = None
        L.jp_create.argtypes = [C.POINTER(abi.JpSystem), ip, C.POINTER(abi.JpParams), C.POINTER(vp)]
        L.jp_rebuild_cells.argtypes = [vp, ip]
        L.jp_energy_grad.argtypes = [vp, ip, dp, dp, dp]
        L.jp_energy_grad_cls.argtypes = [vp, ip, dp, dp, dp, dp, C.POINTER(C.c_int32)]
        L.jp_step.argtypes = [vp, ip, dp, dp]
        L.jp_step_io.argtypes = [vp, ip, dp, dp, dp, dp, dp, dp]
        L.jp_shake.argtypes = [vp, ip, dp, dp]
        L.jp_get_state.argtypes = [vp, ip, dp, dp]
        L.jp_set_state.argtypes = [vp, ip, dp, dp]
        L.jp_pair_count.argtypes = [vp, ip, C.POINTER(C.c_int64)]
        L.jp_set_timing.argtypes = [vp, C.c_int]
        L.jp_set_grid_limit.argtypes = [vp, C.c_int32]
        L.jp_set_wait_limit.argtypes = [vp, C.c_int64]
        L.jp_tile_shape.argtypes = [vp, ip, dp, C.POINTER(C.c_int64)]
        L.jp_alsd_hist_setup.argtypes = [vp, ip, C.c_double, C.c_double, ip, ip, C.c_double, C.c_double, ip]
        L.jp_alsd_hist_get.argtypes = [vp, ip, dp, dp, dp, dp, ip]
        L.jp_alsd_set_mlp.argtypes = [vp, ip, C.POINTER(C.c_float), C.c_double, C.c_double]
        L.jp_last_timing.argtypes = [vp, dp, dp, C.POINTER(C.c_int32)]
        L.jp_launch_counts.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.jp_list_stats.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int64)]
        L.jp_calibrate_fp32.argtypes = [C.c_int32, C.POINTER(C.c_double)]
        L.jp_strerror.argtypes = [C.c_int]
        L.jp_strerror.restype = C.c_char_p
        L.jp_destroy.argtypes = [vp]
        L.jp_destroy.restype = None
        L.jp_ge_hist_setup.argtypes = [vp, ip, C.c_double, C.c_double, ip, ip]
        L.jp_ge_hist_get.argtypes = [vp, ip, dp, ip]
        L.jp_ge_set.argtypes = [vp, ip, C.POINTER(abi.JpGe)]
        L.jp_lstsq_windows.argtypes = [ip, ip, ip, C.c_double, C.c_double, dp, dp, dp, dp, dp, dp, dp]
        L.jp_ge_fit.argtypes = [dp, C.POINTER(abi.JpGeFitParams), C.POINTER(abi.JpGe), dp, dp, dp,
                                C.POINTER(abi.JpGe), dp]
        fp_ = C.POINTER(C.c_float)
        L.jp_ge_dlnn.argtypes = [dp, C.POINTER(abi.JpGeFitParams), C.POINTER(abi.JpGe), dp, dp, dp,
                                 C.POINTER(C.c_int32)]
        L.jp_mlp_nparam.argtypes = [ip, ip]
        L.jp_mlp_nparam.restype = C.c_int32
        L.jp_mlp_init.argtypes = [ip, ip, ip, fp_, fp_, C.POINTER(C.c_int32), C.c_uint64, fp_]
        L.jp_mlp_train.argtypes = [ip, ip, ip, fp_, fp_, fp_, C.POINTER(C.c_int32), ip, C.c_float, ip,
                                   fp_, fp_, fp_]
        L.jp_mlp_forward.argtypes = [ip, ip, fp_, fp_, ip, ip, fp_]
        L.jp_ge_set_mlp.argtypes = [vp, ip, fp_]
        L.jp_get_lambda.argtypes = [vp, ip, dp, dp]
        L.jp_set_lambda.argtypes = [vp, ip, C.c_double, C.c_double]
        L.jp_default_min_params.argtypes = [C.POINTER(abi.JpMinParams)]
        L.jp_default_min_params.restype = None
        L.jp_minimize.argtypes = [vp, C.POINTER(abi.JpMinParams), C.POINTER(C.c_int32), dp, dp,
                                  C.POINTER(C.c_int32)]
        # all array arguments are device addresses except box (host double[3])
        L.jp_nonbond_noalloc.argtypes = [ip, vp, vp, vp, ip, vp, vp, vp, vp, ip, dp, C.c_double,
                                         C.c_double, vp, vp, vp]
        _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _chk(code, where, warn_ok=False):
    if code < 0 or (code > 0 and not warn_ok):
        raise JpError(code, where)
    return code


def lstsq_windows(x, y, w, nwindow, ndeg, minv=0.0, maxv=1.0):
    """lstsquare_final: windowed weighted polynomial fit; returns (coef, low, high, resid)."""
    x, y, w = (np.ascontiguousarray(a, np.float64) for a in (x, y, w))
    coef = np.zeros((nwindow, ndeg + 1))
    low, high, resid = np.zeros(nwindow), np.zeros(nwindow), np.zeros(2)
    _chk(lib().jp_lstsq_windows(nwindow, len(x), ndeg, minv, maxv, _dp(x), _dp(y), _dp(w),
                                _dp(coef), _dp(low), _dp(high), _dp(resid)), "jp_lstsq_windows")
    return coef, low, high, resid


def ge_fit(hist, old_nf, emin, emax, nbin, nbor, next_emin, next_emax, next_temp, nwindow, ndeg,
           ignore_empty=True, neglect_low=False, neglect_high=False):
    """One McMD weight iteration (distrib_MULT): new weight dict and residual errors."""
    keep = []
    h = np.ascontiguousarray(hist, np.float64)
    fp = abi.JpGeFitParams(emin, emax, nbin, nbor, next_emin, next_emax, next_temp, nwindow, ndeg,
                           int(ignore_empty), int(neglect_low), int(neglect_high))
    old = abi.make_ge(old_nf, keep)
    coef = np.zeros((nwindow, ndeg + 1))
    low, high, resid = np.zeros(nwindow), np.zeros(nwindow), np.zeros(2)
    out = abi.JpGe()
    _chk(lib().jp_ge_fit(_dp(h), C.byref(fp), C.byref(old), _dp(coef), _dp(low), _dp(high),
                         C.byref(out), _dp(resid)), "jp_ge_fit")
    nf = dict(coef=coef, low=low, high=high, alphalw=out.alphalw, alphaup=out.alphaup,
              celw=out.celw, ceup=out.ceup, tempce=out.tempce, lower=out.lower, upper=out.upper)
    return nf, resid


def _fp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def _fit_params(emin, emax, nbin, nbor, next_emin, next_emax, next_temp, nwindow, ndeg,
                ignore_empty=True, neglect_low=False, neglect_high=False):
    return abi.JpGeFitParams(emin, emax, nbin, nbor, next_emin, next_emax, next_temp, nwindow,
                             ndeg, int(ignore_empty), int(neglect_low), int(neglect_high))


def ge_dlnn(hist, old_nf, emin, emax, nbin, nbor, next_emin, next_emax, **kw):
    """The (x, y = d lnN/dE, w) points the McMD weight fit takes (distrib_MULT)."""
    keep = []
    h = np.ascontiguousarray(hist, np.float64)
    fp = _fit_params(emin, emax, nbin, nbor, next_emin, next_emax, 300.0, 1, 1, **kw)
    old = abi.make_ge(old_nf, keep)
    cap = nbin + 2 * nbor
    x, y, w = np.zeros(cap), np.zeros(cap), np.zeros(cap)
    n = C.c_int32()
    _chk(lib().jp_ge_dlnn(_dp(h), C.byref(fp), C.byref(old), _dp(x), _dp(y), _dp(w), C.byref(n)),
         "jp_ge_dlnn")
    return x[:n.value].copy(), y[:n.value].copy(), w[:n.value].copy()


def mlp_nparam(nin=1, nout=1):
    return int(lib().jp_mlp_nparam(nin, nout))


def mlp_train(data, nin=1, nout=1, epochs=3000, lr=1e-3, seed=1, device=0, params=None,
              grad=False):
    """Train one surrogate network per (x[n][nin], y[n][nout], w[n]) dataset, all in one launch.
    Returns (params [nnet][np], loss [nnet], grad [nnet][np] or None)."""
    xs = [np.asarray(d[0], np.float32).reshape(len(d[0]), nin) for d in data]
    ys = [np.asarray(d[1], np.float32).reshape(len(d[1]), nout) for d in data]
    ws = [np.asarray(d[2], np.float32).reshape(-1) for d in data]
    off = np.zeros(len(data) + 1, np.int32)
    off[1:] = np.cumsum([len(w) for w in ws])
    X = np.ascontiguousarray(np.concatenate(xs)); Y = np.ascontiguousarray(np.concatenate(ys))
    W = np.ascontiguousarray(np.concatenate(ws))
    npar = mlp_nparam(nin, nout)
    if params is None:
        params = np.zeros((len(data), npar), np.float32)
        _chk(lib().jp_mlp_init(nin, nout, len(data), _fp(X), _fp(Y),
                               off.ctypes.data_as(C.POINTER(C.c_int32)), seed, _fp(params)),
             "jp_mlp_init")
    params = np.ascontiguousarray(params, np.float32).reshape(len(data), npar).copy()
    loss = np.zeros(len(data), np.float32)
    g = np.zeros_like(params) if grad else None
    _chk(lib().jp_mlp_train(nin, nout, len(data), _fp(X), _fp(Y), _fp(W),
                            off.ctypes.data_as(C.POINTER(C.c_int32)), int(epochs), float(lr), device,
                            _fp(params), _fp(loss), _fp(g)), "jp_mlp_train")
    return params, loss, g


def mlp_forward(params, x, nin=1, nout=1, device=0):
    p = np.ascontiguousarray(params, np.float32).reshape(-1)
    X = np.ascontiguousarray(np.asarray(x, np.float32).reshape(-1, nin))
    y = np.zeros((X.shape[0], nout), np.float32)
    _chk(lib().jp_mlp_forward(nin, nout, _fp(p), _fp(X), X.shape[0], device, _fp(y)), "jp_mlp_forward")
    return y


def calibrate_fp32(device=0):
    """Measured FP32 FMA throughput (TFLOP/s) of the device."""
    v = C.c_double()
    _chk(lib().jp_calibrate_fp32(int(device), C.byref(v)), "jp_calibrate_fp32")
    return v.value


class Engine:
    """A device context over one or more replicas sharing run parameters."""

    def __init__(self, tops, params=None, **kw):
        if isinstance(tops, dict):
            tops = [tops]
        self.tops = tops
        self.nrep = len(tops)
        self.natoms = [int(t["natom"]) for t in tops]
        self.params = params if params is not None else abi.default_params(**kw)
        self._keep = []
        self._hist_n = {}
        self._sys = abi.make_systems(tops, self._keep)
        h = C.c_void_p()
        _chk(lib().jp_create(self._sys, self.nrep, C.byref(self.params), C.byref(h)), "jp_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().jp_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- state ----
    def get_state(self, rep=0, cord=None, vel=None):
        n = self.natoms[rep]
        cord = np.empty((n, 3)) if cord is None else cord
        vel = np.empty((n, 3)) if vel is None else vel
        _chk(lib().jp_get_state(self._h, rep, _dp(cord), _dp(vel)), "jp_get_state")
        return cord, vel

    def set_state(self, rep=0, cord=None, vel=None):
        c = None if cord is None else np.ascontiguousarray(cord, np.float64)
        v = None if vel is None else np.ascontiguousarray(vel, np.float64)
        _chk(lib().jp_set_state(self._h, rep, _dp(c), _dp(v)), "jp_set_state")

    def rebuild(self, rep=-1):
        _chk(lib().jp_rebuild_cells(self._h, rep), "jp_rebuild_cells")

    # ---- dnergy ----
    def energy_grad(self, rep=0, cord=None):
        n = self.natoms[rep]
        c = None if cord is None else np.ascontiguousarray(cord, np.float64)
        e = np.zeros(abi.JP_MAXENE)
        g = np.zeros((n, 3))
        _chk(lib().jp_energy_grad(self._h, rep, _dp(c), _dp(e), _dp(g)), "jp_energy_grad")
        return e, g

    def energy_grad_cls(self, rep=0, cord=None):
        """dnergy's outputs by class: (eneval, class totals [nfrg], unscaled class gradients
        [nfrg, natom, 3]); nfrg = 1 without cluster atoms, 3 for ALSD (AA, AB, BB), 2 for
        GEPSME= AND / OR / XOR (classes 1, 2)."""
        n = self.natoms[rep]
        c = None if cord is None else np.ascontiguousarray(cord, np.float64)
        e = np.zeros(abi.JP_MAXENE)
        ec = np.zeros(3)
        g = np.zeros((3, n, 3))
        nf = C.c_int32(0)
        _chk(lib().jp_energy_grad_cls(self._h, rep, _dp(c), _dp(e), _dp(ec), _dp(g), C.byref(nf)),
             "jp_energy_grad_cls")
        return e, ec[:nf.value].copy(), g[:nf.value].copy()

    # ---- McMD iteration ----
    def ge_hist_setup(self, emin, emax, nbin, nbor, rep=-1):
        _chk(lib().jp_ge_hist_setup(self._h, rep, emin, emax, nbin, nbor), "jp_ge_hist_setup")
        for r in (range(self.nrep) if rep < 0 else [rep]):
            self._hist_n[r] = nbin + 2 * nbor if nbin > 0 else 0

    def ge_hist_get(self, rep=0, clear=False):
        n = int(self._hist_n.get(rep, abi.JP_GE_MAX_BINS))
        h = np.zeros(abi.JP_GE_MAX_BINS)
        _chk(lib().jp_ge_hist_get(self._h, rep, _dp(h), int(clear)), "jp_ge_hist_get")
        return h[:n]

    def ge_set(self, nf, rep=0):
        keep = []
        g = abi.make_ge(nf, keep)
        _chk(lib().jp_ge_set(self._h, rep, C.byref(g)), "jp_ge_set")

    # ---- ALSD ----
    def get_lambda(self, rep=0):
        """(lambda, lambda velocity), class energies (AA, AB, BB) of the last force call."""
        l2, ec = np.zeros(2), np.zeros(3)
        _chk(lib().jp_get_lambda(self._h, rep, _dp(l2), _dp(ec)), "jp_get_lambda")
        return l2, ec

    def set_lambda(self, lam, lam_v=0.0, rep=0):
        _chk(lib().jp_set_lambda(self._h, rep, float(lam), float(lam_v)), "jp_set_lambda")

    # ---- ALSD weight iteration ----
    def alsd_hist_setup(self, lmin, lmax, nbin, nbor, emin=0.0, emax=1.0, ne=0, rep=0):
        _chk(lib().jp_alsd_hist_setup(self._h, rep, lmin, lmax, nbin, nbor, emin, emax, ne),
             "jp_alsd_hist_setup")
        self._alsd_n = getattr(self, "_alsd_n", {})
        self._alsd_n[rep] = (nbin + 2 * nbor if nbin > 0 else 0, ne if nbin > 0 else 0)

    def alsd_hist_get(self, rep=0, clear=False):
        """(counts [nl], sums of dE/dlambda [nl], counts [ne][nl], sums [ne][nl])."""
        nl, ne = self._alsd_n.get(rep, (0, 0))
        c, f = np.zeros(nl), np.zeros(nl)
        c2, f2 = np.zeros((ne, nl)), np.zeros((ne, nl))
        _chk(lib().jp_alsd_hist_get(self._h, rep, _dp(c), _dp(f), _dp(c2), _dp(f2), int(clear)),
             "jp_alsd_hist_get")
        return c, f, c2, f2

    def alsd_set_mlp(self, params, emin=0.0, emax=1.0, rep=0):
        p = None if params is None else np.ascontiguousarray(params, np.float32).reshape(-1)
        _chk(lib().jp_alsd_set_mlp(self._h, rep, _fp(p), float(emin), float(emax)), "jp_alsd_set_mlp")

    def ge_set_mlp(self, params, rep=0):
        p = None if params is None else np.ascontiguousarray(params, np.float32).reshape(-1)
        _chk(lib().jp_ge_set_mlp(self._h, rep, _fp(p)), "jp_ge_set_mlp")

    def pair_count(self, rep=0):
        v = C.c_int64()
        _chk(lib().jp_pair_count(self._h, rep, C.byref(v)), "jp_pair_count")
        return v.value

    # ---- runmd ----
    def step(self, nsteps=1, energies=True, temps=True, warn_ok=False):
        e = np.zeros((nsteps, self.nrep, abi.JP_MAXENE)) if energies else None
        t = np.zeros((nsteps, self.nrep)) if temps else None
        code = _chk(lib().jp_step(self._h, int(nsteps), _dp(e), _dp(t)), "jp_step", warn_ok)
        self.last_code = code
        return e, t

    def step_io(self, x_in, v_in, x_out, v_out, ene=None, temp=None, nsteps=1, warn_ok=False):
        """jp_step_io: all replicas' state in from host arrays [natom_total][3] (None = keep),
        nsteps steps, state out (None = not wanted), one synchronisation.  ene [nsteps][nrep][15]
        and temp [nsteps][nrep] are filled when given."""
        code = lib().jp_step_io(self._h, int(nsteps), _dp(x_in), _dp(v_in), _dp(x_out), _dp(v_out),
                                _dp(ene), _dp(temp))
        self.last_code = _chk(code, "jp_step_io", warn_ok)
        return code

    def minimize(self, warn_ok=False, **kw):
        """Steepest descent of every replica (jp_minimize); kw override the md_run defaults
        (max_loop, update, convgr, step0, up, down).  Returns per replica (iters, energies,
        rms gradient, state); JpError for JP_E_MIN_STEP or a SHAKE failure."""
        mp = abi.min_params(**kw)
        it = np.zeros(self.nrep, np.int32)
        st = np.zeros(self.nrep, np.int32)
        e = np.zeros((self.nrep, abi.JP_MAXENE))
        rm = np.zeros(self.nrep)
        code = lib().jp_minimize(self._h, C.byref(mp), it.ctypes.data_as(C.POINTER(C.c_int32)), _dp(e),
                                 _dp(rm), st.ctypes.data_as(C.POINTER(C.c_int32)))
        self.last_code = _chk(code, "jp_minimize", warn_ok)
        return it, e, rm, st

    def shake(self, r1, r2, rep=0):
        r1 = np.ascontiguousarray(r1, np.float64).copy()
        r2 = np.ascontiguousarray(r2, np.float64)
        code = lib().jp_shake(self._h, rep, _dp(r1), _dp(r2))
        return code, r1

    # ---- timing ----
    def set_timing(self, on):
        _chk(lib().jp_set_timing(self._h, 1 if on else 0), "jp_set_timing")

    def set_grid_limit(self, blocks):
        """Cap the integration grid (0 = co-resident maximum); a smaller grid than the
        system's lanes selects the grid-stride form of the integrator."""
        _chk(lib().jp_set_grid_limit(self._h, int(blocks)), "jp_set_grid_limit")

    def tile_shape(self, rep=0):
        """(column-edge factor chosen for the replica, pair records per candidate)."""
        f = C.c_double()
        t = (C.c_int64 * abi.JP_TUNE_CANDIDATES)()
        _chk(lib().jp_tile_shape(self._h, rep, C.byref(f), t), "jp_tile_shape")
        return f.value, list(t)

    def set_wait_limit(self, cycles):
        """Bound of the integration kernel's grid-barrier waits in SM cycles (0 = default)."""
        _chk(lib().jp_set_wait_limit(self._h, int(cycles)), "jp_set_wait_limit")

    def last_timing(self):
        tot = C.c_double()
        ph = (C.c_double * 4)()
        ln = (C.c_int32 * 4)()
        _chk(lib().jp_last_timing(self._h, C.byref(tot), ph, ln), "jp_last_timing")
        return tot.value, list(ph), list(ln)

    def list_stats(self):
        t, p, s = C.c_int64(), C.c_int64(), C.c_int64()
        _chk(lib().jp_list_stats(self._h, C.byref(t), C.byref(p), C.byref(s)), "jp_list_stats")
        return t.value, p.value, s.value

    def launch_counts(self):
        a, b = C.c_int32(), C.c_int32()
        _chk(lib().jp_launch_counts(self._h, C.byref(a), C.byref(b)), "jp_launch_counts")
        return a.value, b.value
