"""TEST INFRASTRUCTURE ONLY: md_run's FDEBUG force file, 1stp_force.bin.

md_run with `FDEBUG= MAKE` stops after the first force evaluation of verlethe and writes
three Fortran unformatted sequential records (verlethe.f90:382-387): eneval(1:15), the
lambda force, grad(1:3, 1:natom) -- after verlethe's scaling of the gradient.  With
`FDEBUG= CHECK` it reads such a file and prints the largest force and energy differences
against a threshold of 1e-9 (verlethe.f90:325-380).

`write` produces the file from the oracle (`Oracle.first_force`), so that a reference run
with FDEBUG= CHECK on the same system pins the oracle; `read` and `compare` do the reverse
for a file made by the reference.  Records use gfortran's default framing: a 4-byte
little-endian byte count before and after each record.
"""
import struct

import numpy as np

MAXENE = 15
THRESHOLD = 1.0e-9   # erth, verlethe.f90:73


def _record(f, payload):
    n = struct.pack("<i", len(payload))
    f.write(n + payload + n)


def _read_record(f):
    head = f.read(4)
    if len(head) != 4:
        raise ValueError("truncated record marker")
    (n,) = struct.unpack("<i", head)
    payload = f.read(n)
    tail = f.read(4)
    if len(payload) != n or tail != head:
        raise ValueError("record length markers do not match")
    return payload


def write(path, epot, lambda_f, grad):
    """1stp_force.bin from eneval (15), lambda_f and grad (natom x 3, dE/dx)."""
    epot = np.ascontiguousarray(epot, np.float64).reshape(MAXENE)
    grad = np.ascontiguousarray(grad, np.float64).reshape(-1, 3)
    with open(path, "wb") as f:
        _record(f, epot.tobytes())
        _record(f, struct.pack("<d", float(lambda_f)))
        _record(f, grad.tobytes())   # grad(1:3, i) fastest: the same order as C [natom][3]


def read(path):
    """(eneval, lambda_f, grad[natom][3]) from a 1stp_force.bin."""
    with open(path, "rb") as f:
        e = np.frombuffer(_read_record(f), np.float64)
        (lf,) = struct.unpack("<d", _read_record(f))
        g = np.frombuffer(_read_record(f), np.float64)
    if e.size != MAXENE or g.size % 3:
        raise ValueError("not a 1stp_force.bin record layout")
    return e.copy(), lf, g.reshape(-1, 3).copy()


def compare(ref, epot, lambda_f, grad, threshold=THRESHOLD):
    """FDEBUG= CHECK: the largest absolute gradient-component and lambda-force
    differences, the largest energy difference over slots 2..15 (eneval(2:)) and its slot,
    the atoms whose difference vector is at least the threshold, and whether both the
    force and the energy differences stay within it."""
    e0, lf0, g0 = ref
    dg = np.abs(np.asarray(grad, np.float64).reshape(-1, 3) - g0)
    de = np.abs(np.asarray(epot, np.float64) - e0)
    worst = int(np.argmax(de[1:])) + 1
    big = np.flatnonzero(np.linalg.norm(dg, axis=1) >= threshold)
    fmax = float(dg.max()) if dg.size else 0.0
    return dict(max_force_error=fmax, lambda_force_error=abs(float(lambda_f) - lf0),
                max_energy_error=float(de[worst]), energy_slot=worst, atoms_over=big,
                passed=fmax <= threshold and float(de[1:].max()) <= threshold)
