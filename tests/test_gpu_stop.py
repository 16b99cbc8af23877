"""Centre-of-mass stop (STOPCE, remotv) and METHOD= CONS (Berendsen, scalet) on the GPU
against the oracle, in both forms of the CANO/GE integrator: one cooperative launch with the
unit state on chip (the default at these sizes) and one launch per phase (the form of
systems with more lanes than the cooperative grid holds, forced by a small grid limit).

Tolerances as the other parity tests: 15-step FP64 trajectories within 1e-8 A of the
oracle; the mixed path's stopped momentum and angular momentum within 1e-9 of the
molecule's own scale (the sums are FP64 on the device).
"""
import numpy as np
import pytest

import oracle
from j_presto_b200 import abi, systems

pytestmark = pytest.mark.gpu

FP64, MIXED = abi.JP_PREC_FP64, abi.JP_PREC_MIXED
M, C_, CANO, GE = abi.JP_METHOD_MICR, abi.JP_METHOD_CONS, abi.JP_METHOD_CANO, abi.JP_METHOD_GE
TR, ROT, BOTH, NONE = abi.JP_STOP_TRANS, abi.JP_STOP_ROT, abi.JP_STOP_BOTH, abi.JP_STOP_NONE


@pytest.fixture(scope="module")
def eng_mod(engine_lib):
    from j_presto_b200 import engine
    return engine


@pytest.fixture(scope="module")
def poly():
    top = dict(systems.solvated_polymer(20, 1500, seed=7))
    e0 = oracle.Oracle(top, method=M).energy_grad()[0][0]
    top["ge"] = dict(coef=np.array([[1.2, -0.3]]), low=np.array([0.0]), high=np.array([1.0 + 1e-12]),
                     alphalw=1.2, alphaup=0.9, celw=e0 - 2000.0, ceup=e0 + 2000.0, tempce=300.0)
    return top


def _parity(eng_mod, top, grid=0, nstep=15, **kw):
    o = oracle.Oracle(top, **kw)
    ier, _, _ = o.run(nstep)
    assert ier == 0
    xo, vo = o.get_state()
    with eng_mod.Engine(top, precision=FP64, **kw) as e:
        if grid:
            e.set_grid_limit(grid)
        e.step(nstep)
        x, v = e.get_state()
    assert np.abs(x - xo).max() < 1e-8
    assert np.abs(v - vo).max() < 1e-8


@pytest.mark.parametrize("method,stop,tempco", [
    (M, BOTH, 1), (C_, NONE, 1), (C_, TR, 2), (CANO, BOTH, 2), (CANO, ROT, 1), (GE, TR, 2),
])
def test_trajectory_vs_oracle(eng_mod, poly, method, stop, tempco):
    _parity(eng_mod, poly, method=method, stop_center=stop, tempco=tempco)


def test_without_shake_vs_oracle(eng_mod, poly):
    _parity(eng_mod, poly, method=CANO, stop_center=BOTH, shake_method=abi.JP_SHAKE_NONE)


def test_stop_natom_vs_oracle(eng_mod, poly):
    _parity(eng_mod, poly, method=CANO, stop_center=BOTH, stop_natom=40)


@pytest.mark.parametrize("method,stop,tempco", [(CANO, NONE, 2), (CANO, BOTH, 2), (GE, TR, 1), (GE, NONE, 2)])
def test_per_phase_form_vs_oracle(eng_mod, poly, method, stop, tempco):
    """A two-block cooperative grid for a few thousand lanes: the step runs as one launch per
    phase with the unit state in the atom arrays between them, 4-atom groups included (GE:
    the McMD force scale evaluated per replica before the phases)."""
    _parity(eng_mod, poly, grid=2, method=method, stop_center=stop, tempco=tempco)


def test_per_phase_form_without_shake_vs_oracle(eng_mod, poly):
    _parity(eng_mod, poly, grid=2, method=CANO, stop_center=BOTH, shake_method=abi.JP_SHAKE_NONE)


def test_mixed_path_stops_the_molecule(eng_mod, poly):
    mol = np.asarray(poly["molecule"])
    n0 = int(np.argmax(mol != mol[0]))
    m = np.asarray(poly["mass"])[:n0, None]
    with eng_mod.Engine(poly, precision=MIXED, method=CANO, stop_center=BOTH) as e:
        e.step(20)
        x, v = e.get_state()
    x, v = x[:n0], v[:n0]
    c = (m * x).sum(0) / m.sum()
    p = np.abs((m * v).sum(0)).max()
    L = np.abs((m * np.cross(x - c, v)).sum(0)).max()
    scale_p = (m * np.abs(v)).sum()
    scale_l = (m[:, 0] * np.linalg.norm(x - c, axis=1) * np.linalg.norm(v, axis=1)).sum()
    assert p < 1e-9 * scale_p and L < 1e-9 * scale_l


def test_invalid_parameters_are_rejected(eng_mod, poly):
    for kw in (dict(method=C_, taut=0.0), dict(stop_center=7), dict(stop_natom=10 ** 7),
               dict(method=C_, alsd=abi.JP_ALSD_LMD)):
        with pytest.raises(eng_mod.JpError) as ex:
            eng_mod.Engine(poly, precision=MIXED, **kw)
        assert ex.value.code == abi.JP_E_INVALID
