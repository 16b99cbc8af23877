"""md_run's trajectory, velocity and energy output (monmd.f90 outtco / outtve / outten) for
the Python host, as Fortran unformatted sequential records (4-byte little-endian byte
counts around each record, gfortran's default).

NAMECO / NAMEVE / NAMETO files: per output step two records.  REAL4 files (iflag 1) hold
single-precision reals, REAL8 files (iflag 2) double precision; integers are 4 bytes in
both.  The Fortran driver keeps its own writers; these produce the same records from
`Engine.get_state` / `Engine.step` output so that md_run's analysis tools read them.

  trajectory (outtco, monmd.f90:235-285)
    idloop, time, cpu, E_total, E_kin, T, E_pot, lambda, n15v, n15h, rmsd, E_pot by class(3)
    coordinates (3, natom_out)
  velocities (outtve, :291-335)
    idloop, time, cpu, E_total, E_kin, T, E_pot, rmsf, n15v, n15h, rmsd
    velocities (3, natom_out)
  energies (outten, :341-375)
    idloop, time, cpu
    E_total, E_kin, T, eneval(1:15), rmsf, n15v, n15h, rmsd

Under periodic boundaries outtco first moves every chain by whole box lengths so that its
geometric centre lies in the cell (PBcord.f90); `wrap_chains` does that.

Restart files (outrst.f90 / inprst.f90:37-56), always double precision:
    title (80 characters) / natom, nvar / step, time, E_total, E_kin, E_pot /
    coordinates (3, natom) / velocities (3, nvar) / lambda, lambda velocity
"""
import struct

import numpy as np

REAL4, REAL8 = 1, 2


def _rec(f, payload):
    n = struct.pack("<i", len(payload))
    f.write(n + payload + n)


def read_records(path):
    """Every record of a Fortran unformatted sequential file, as bytes."""
    out = []
    with open(path, "rb") as f:
        while True:
            head = f.read(4)
            if not head:
                return out
            (n,) = struct.unpack("<i", head)
            body = f.read(n)
            if len(body) != n or f.read(4) != head:
                raise ValueError(f"{path}: damaged record {len(out)}")
            out.append(body)


def wrap_chains(cord, chains, box, wall_lo):
    """PBcord (PBcord.f90): each chain (first, last atom, inclusive) shifted by whole box
    lengths so that its geometric centre lies in [wall_lo, wall_lo + box)."""
    x = np.array(cord, np.float64, copy=True)
    box = np.asarray(box, np.float64)
    wall_lo = np.asarray(wall_lo, np.float64)
    for f, l in chains:
        c = x[f:l + 1].sum(0) / (l - f + 1)
        x[f:l + 1] -= box * np.floor((c - wall_lo) / box)
    return x


class _Writer:
    def __init__(self, path, precision=REAL4, atoms=None):
        if precision not in (REAL4, REAL8):
            raise ValueError("precision is REAL4 (1) or REAL8 (2)")
        self.f = open(path, "wb")
        self.real = "f" if precision == REAL4 else "d"
        self.np_real = np.float32 if precision == REAL4 else np.float64
        self.atoms = None if atoms is None else np.asarray(atoms)   # OUTATM selection

    def _pack(self, fields):
        """fields: sequence of ('i' | 'r', value)."""
        fmt = "<" + "".join("i" if k == "i" else self.real for k, _ in fields)
        return struct.pack(fmt, *[int(v) if k == "i" else float(v) for k, v in fields])

    def _array(self, a):
        a = np.asarray(a, np.float64).reshape(-1, 3)
        if self.atoms is not None:
            a = a[self.atoms]
        return np.ascontiguousarray(a, self.np_real).tobytes()   # (3, natom) column order

    def close(self):
        self.f.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class TrajectoryWriter(_Writer):
    """NAMECO (outtco)."""

    def write(self, cord, step, time=0.0, cpu=0.0, etot=0.0, ekin=0.0, temp=0.0, epot=0.0,
              lam=0.0, n15v=0, n15h=0, rmsd=0.0, epot_cls=(0.0, 0.0, 0.0)):
        c3 = list(epot_cls) + [0.0] * (3 - len(epot_cls))
        head = [("i", step), ("r", time), ("r", cpu), ("r", etot), ("r", ekin), ("r", temp),
                ("r", epot), ("r", lam), ("i", n15v), ("i", n15h), ("r", rmsd)]
        _rec(self.f, self._pack(head + [("r", v) for v in c3[:3]]))
        _rec(self.f, self._array(cord))


class VelocityWriter(_Writer):
    """NAMEVE (outtve)."""

    def write(self, vel, step, time=0.0, cpu=0.0, etot=0.0, ekin=0.0, temp=0.0, epot=0.0,
              rmsf=0.0, n15v=0, n15h=0, rmsd=0.0):
        head = [("i", step), ("r", time), ("r", cpu), ("r", etot), ("r", ekin), ("r", temp),
                ("r", epot), ("r", rmsf), ("i", n15v), ("i", n15h), ("r", rmsd)]
        _rec(self.f, self._pack(head))
        _rec(self.f, self._array(vel))


class EnergyWriter(_Writer):
    """NAMETO (outten): eneval has md_run's 15 slots (the engine's JP_E_* order)."""

    def write(self, eneval, step, time=0.0, cpu=0.0, etot=0.0, ekin=0.0, temp=0.0, rmsf=0.0,
              n15v=0, n15h=0, rmsd=0.0):
        e = np.asarray(eneval, np.float64).reshape(-1)
        if e.size != 15:
            raise ValueError("eneval has 15 slots")
        _rec(self.f, self._pack([("i", step), ("r", time), ("r", cpu)]))
        _rec(self.f, self._pack([("r", etot), ("r", ekin), ("r", temp)] + [("r", v) for v in e]
                                + [("r", rmsf), ("i", n15v), ("i", n15h), ("r", rmsd)]))


def write_restart(path, cord, vel, step=0, time=0.0, etot=0.0, ekin=0.0, epot=0.0, lam=0.0,
                  lam_v=0.0, title="     VERLET"):
    """A restart file as outrst.f90 writes it (all atoms variable: nvar = natom)."""
    x = np.ascontiguousarray(cord, np.float64).reshape(-1, 3)
    v = np.ascontiguousarray(vel, np.float64).reshape(-1, 3)
    with open(path, "wb") as f:
        _rec(f, title.encode("ascii", "replace")[:80].ljust(80))
        _rec(f, struct.pack("<ii", len(x), len(v)))
        _rec(f, struct.pack("<i4d", int(step), float(time), float(etot), float(ekin), float(epot)))
        _rec(f, x.tobytes())
        _rec(f, v.tobytes())
        _rec(f, struct.pack("<2d", float(lam), float(lam_v)))


def read_restart(path):
    """The records inprst.f90 reads: dict(title, step, time, etot, ekin, epot, cord, vel,
    lam, lam_v); a file without the last record has lam = lam_v = 0."""
    recs = read_records(path)
    natom, nvar = struct.unpack("<ii", recs[1])
    step, time, etot, ekin, epot = struct.unpack("<i4d", recs[2])
    out = dict(title=recs[0].decode("ascii", "replace").rstrip(), step=step, time=time, etot=etot,
               ekin=ekin, epot=epot,
               cord=np.frombuffer(recs[3], np.float64).reshape(natom, 3).copy(),
               vel=np.frombuffer(recs[4], np.float64).reshape(nvar, 3).copy(), lam=0.0, lam_v=0.0)
    if len(recs) > 5:
        out["lam"], out["lam_v"] = struct.unpack("<2d", recs[5])
    return out


def read_trajectory(path, precision=REAL4):
    """(headers, frames[nframe][natom_out][3]) of a NAMECO file written as above."""
    r = "f" if precision == REAL4 else "d"
    fmt = "<i" + r * 7 + "ii" + r * 4
    recs = read_records(path)
    heads, frames = [], []
    for h, body in zip(recs[0::2], recs[1::2]):
        heads.append(struct.unpack(fmt, h))
        frames.append(np.frombuffer(body, np.float32 if precision == REAL4 else np.float64).reshape(-1, 3))
    return heads, np.array(frames)
