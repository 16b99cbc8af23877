"""md.inp keywords of the EXE> MD and EXE> MIN blocks mapped to the engine's parameters, for
the Python host (md_run's inpmd.f90 / inpmin.f90 read the same blocks for the Fortran
driver).

A block starts at a line `EXE> MD` (or `EXE> MIN`) and ends at `QUIT`; inside, `KEY= value`
pairs, several per line allowed; `;` starts a comment.  Keywords are six letters and
case-insensitive; choice values are compared on their first four letters, as inpmd.f90's
tables are.  Unknown keywords are kept in `other` untouched.
"""
import re

from j_presto_b200 import abi

_PAIR = re.compile(r"([A-Za-z_][A-Za-z0-9_]*)\s*=\s*([^\s;]+)")

# choice keywords (inpmd.f90:62-82) -> engine values
_CHOICES = {
    "METHOD": {"CONS": abi.JP_METHOD_CONS, "MICR": abi.JP_METHOD_MICR, "CANO": abi.JP_METHOD_CANO,
               "GE": abi.JP_METHOD_GE, "MULT": abi.JP_METHOD_GE},
    "STOPCE": {"TRAN": abi.JP_STOP_TRANS, "ROTA": abi.JP_STOP_ROT, "BOTH": abi.JP_STOP_BOTH,
               "NO": abi.JP_STOP_NONE},
    "CAL15M": {"CMM": abi.JP_CAL15M_CMM, "ATOM": abi.JP_CAL15M_ATOM, "ZD": abi.JP_CAL15M_ZD},
    "SHAKEM": {"HBON": abi.JP_SHAKE_HBON, "ALLB": abi.JP_SHAKE_ALLB},
    "BOUNDA": {"NO": abi.JP_BOUND_NONE, "PBC": abi.JP_BOUND_PBC},
    "TEMPCO": {"NO": 1, "YES": 2},
}
# keyword -> jp_params field (numbers)
_MD_FIELDS = {
    "TIMEST": "dt", "CUTLEN": "cutoff", "DIEVAL": "dielectric", "UPDATE": "update",
    "SETTEM": "temp", "STARTT": "temp_start", "HEATLO": "heat_loop", "COVSHK": "shake_tol",
    "LIMSHK": "shake_maxit", "PSETMP": "psetmp", "RELAXA": "taut", "CMMUPD": "cmm_update",
    "LAMBDA": "lambda0",
}
_MD_CHOICE_FIELDS = {"METHOD": "method", "STOPCE": "stop_center", "CAL15M": "cal15m",
                     "SHAKEM": "shake_method", "BOUNDA": "bounda", "TEMPCO": "tempco"}
_MIN_FIELDS = {"LOOPLI": "max_loop", "UPDATE": "update", "CONVGR": "convgr", "ISTEPL": "step0"}


def blocks(text):
    """{block name: {KEY: value string}} of every EXE> block (a later block of the same
    name replaces an earlier one)."""
    out, cur = {}, None
    for raw in text.splitlines():
        line = raw.split(";", 1)[0].strip()
        if not line:
            continue
        up = line.upper()
        if up.startswith("EXE>"):
            cur = up[4:].strip()
            out[cur] = {}
            continue
        if up.startswith("QUIT"):
            cur = None
            continue
        if cur is not None:
            for k, v in _PAIR.findall(line):
                out[cur][k.upper()] = v
    return out


def _choice(key, value):
    table = _CHOICES[key]
    v = value.upper()
    for name, code in table.items():
        if v[:4] == name[:4]:
            return code
    raise ValueError(f"{key}= {value}: not one of {', '.join(table)}")


def md_params(text):
    """(jp_params keyword arguments, steps, seed, other keywords) of the EXE> MD block."""
    kv = blocks(text).get("MD", {})
    params, other = {}, {}
    for k, v in kv.items():
        if k in _MD_CHOICE_FIELDS:
            params[_MD_CHOICE_FIELDS[k]] = _choice(k, v)
        elif k in _MD_FIELDS:
            f = _MD_FIELDS[k]
            params[f] = int(v) if f in ("update", "heat_loop", "shake_maxit", "cmm_update") else float(v)
        elif k not in ("LOOPLI", "RANDOM"):
            other[k] = v
    steps = int(kv.get("LOOPLI", 0))
    seed = int(kv.get("RANDOM", 584287))   # inpmd.f90 default seed
    return params, steps, seed, other


def min_params(text):
    """jp_min_params keyword arguments of the EXE> MIN block (METHOD= STEE / CONJ)."""
    kv = blocks(text).get("MIN", {})
    out = {}
    for k, v in kv.items():
        if k == "METHOD":
            m = v.upper()[:4]
            if m not in ("STEE", "CONJ"):
                raise ValueError(f"METHOD= {v}: STEE or CONJ")
            out["method"] = abi.JP_MIN_STEEP if m == "STEE" else abi.JP_MIN_CONJ
        elif k in _MIN_FIELDS:
            f = _MIN_FIELDS[k]
            out[f] = int(v) if f in ("max_loop", "update") else float(v)
    return out
