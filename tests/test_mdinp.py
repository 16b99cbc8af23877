"""md.inp EXE> MD / EXE> MIN keywords mapped to the engine's parameters (no GPU)."""
import pytest

from j_presto_b200 import abi, mdinp

TEXT = """
; a comment line
EXE> INPUT
  TOPOLO= sys.tpl     ; not an MD keyword
QUIT
EXE> MD
  METHOD= CANO  LOOPLI= 5000   ; two pairs on a line
  settem= 310.0                ; lower case
  STARTT= 100.0  HEATLO= 2000
  STOPCE= BOTH   CAL15M= ATOM   CUTLEN= 10.5
  BOUNDA= PBC    SHAKEM= HBONd  TIMEST= 2.0  UPDATE= 20
  RANDOM= 12345  OUTLOG= 100
QUIT
EXE> MIN
  METHOD= CONJugate  LOOPLI= 300  CONVGR= 0.5  ISTEPL= 0.002
QUIT
"""


def test_md_block():
    params, steps, seed, other = mdinp.md_params(TEXT)
    assert steps == 5000 and seed == 12345 and other == {"OUTLOG": "100"}
    assert params == dict(method=abi.JP_METHOD_CANO, temp=310.0, temp_start=100.0, heat_loop=2000,
                          stop_center=abi.JP_STOP_BOTH, cal15m=abi.JP_CAL15M_ATOM, cutoff=10.5,
                          bounda=abi.JP_BOUND_PBC, shake_method=abi.JP_SHAKE_HBON, dt=2.0, update=20)
    p = abi.default_params(**params)   # the engine takes them as they are
    assert p.update == 20 and p.cal15m == abi.JP_CAL15M_ATOM


def test_min_block_and_errors():
    mp = mdinp.min_params(TEXT)
    assert mp == dict(method=abi.JP_MIN_CONJ, max_loop=300, convgr=0.5, step0=0.002)
    assert abi.min_params(**mp).line_max == 10
    with pytest.raises(ValueError):
        mdinp.md_params("EXE> MD\n METHOD= FAST\nQUIT\n")
    assert mdinp.md_params("EXE> MD\nQUIT\n")[1:3] == (0, 584287)
