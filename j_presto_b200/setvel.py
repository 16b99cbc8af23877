"""Initial velocities as md_run draws them (md.f90:1009-1040 calling setvel.f90), for the
Python host: the same generator and seed give the same velocities.

  ranun (ranun.f90)  uniform numbers from a 30-bit multiplicative-congruential sequence
                     kept in two 15-bit halves (a = 32771, c = 123456781, m = 2^30), each
                     number the state converted to single precision over 2^30
  ranno (ranno.f90)  Box-Muller pairs from consecutive uniforms, in single precision; an
                     odd count takes one extra pair of uniforms for its last number
  setvel             v = N(0, 1) * sqrt(T R 1e-7 / m) per component, atom by atom
  md.f90:1018-1040   then the centre-of-mass translation and rotation are removed and the
                     velocities scaled to the temperature T exactly

The single-precision log, cos and sin come from numpy here and from the Fortran runtime in
md_run; they may differ in the last bit, so velocities agree to single precision.
"""
import numpy as np

GAS = 8.31451      # gascst, J / (mol K)


def ranun(n, seed):
    """n uniform numbers in (0, 1) as float32 and the next seed (ranun.f90:35-58)."""
    ia, ib, d, e = 32771, 123456781, 2 ** 15, 2 ** 15
    iu, il = divmod(int(seed), d)
    out = np.empty(n, np.float32)
    for i in range(n):
        ild = il * ia + ib
        ils, il = divmod(ild, d)
        iu = (ia * iu + ils) % e
        seed = d * iu + il
        out[i] = np.float32(seed) * np.float32(2.0 ** -30)
    return out, seed


def ranno(n, seed, mean=0.0, sd=1.0):
    """n normal numbers (float32) by Box-Muller and the next seed (ranno.f90:36-70)."""
    x, seed = ranun(n, seed)
    if n % 2:
        extra, seed = ranun(2, seed)
    f32 = np.float32
    phi2 = f32(2.0) * f32(3.141593)
    mean, sd = f32(mean), f32(sd)
    out = x.copy()
    last = n - 1 if n % 2 else n
    for i in range(0, last, 2):
        r = sd * np.sqrt(f32(-2.0) * np.log(x[i]))
        a = phi2 * x[i + 1]
        out[i] = r * np.cos(a) + mean
        out[i + 1] = r * np.sin(a) + mean
    if n % 2:
        out[n - 1] = sd * np.sqrt(f32(-2.0) * np.log(x[n - 1])) * np.cos(phi2 * extra[0]) + mean
    return out, seed


def initial_velocities(mass, cord, temp, seed, dof):
    """md_run's starting velocities (A/fs) at `temp` K for `dof` degrees of freedom, and the
    next seed: setvel, then no centre-of-mass motion, then scaled to `temp` exactly."""
    m = np.asarray(mass, np.float64)
    x = np.asarray(cord, np.float64).reshape(-1, 3)
    n = len(m)
    r, seed = ranno(3 * n, seed)
    v = r.reshape(n, 3).astype(np.float64) * np.sqrt(temp * GAS * 1.0e-7) / np.sqrt(m)[:, None]
    # remotv mode 3: translation of the centre and rotation about it
    mt = m.sum()
    c = (m[:, None] * x).sum(0) / mt
    v -= (m[:, None] * v).sum(0) / mt
    d = x - c
    inertia = np.einsum("i,ij->", m, d * d) * np.eye(3) - np.einsum("i,ij,ik->jk", m, d, d)
    w = np.linalg.solve(inertia, (m[:, None] * np.cross(d, v)).sum(0))
    v -= np.cross(w, d)
    # caltmp: T = sum m v^2 / (dof R) in md_run units (amu A^2 fs^-2 -> J/mol: 1e7)
    t_now = (m[:, None] * v * v).sum() * 1.0e7 / (dof * GAS)
    return v * np.sqrt(temp / t_now), seed
