"""jp_nonbond_noalloc (the entry point whose scratch is a static device array) against the
existing entry point jp_energy_grad.

The system is the 1,000-water box with its bond and angle force constants set to zero, so
that jp_energy_grad's gradient is the non-bonded gradient alone (the water exclusions are
exactly its 1-2 and 1-3 pairs, the pairs md_run applies the ZD excess to).  Tolerances are
those of the FP64 path: gradient RMS relative 1e-12, energies 1e-8 relative.
"""
import ctypes as C

import numpy as np
import pytest

from j_presto_b200 import abi, systems
from tests._util import rms_rel

VDW15, ELE15 = 7, 8    # energy slots of jp_energy_grad (include/jpgpu.h JP_E_VDW15/ELE15)


def _water():
    top = dict(systems.config_c1_prime())
    top["bond_k"] = np.zeros_like(top["bond_k"])
    top["angle_k"] = np.zeros_like(top["angle_k"])
    return top


def test_noalloc_rejects_sizes_beyond_the_limit(engine_lib):
    box = (C.c_double * 3)(100.0, 100.0, 100.0)
    rc = engine_lib.jp_nonbond_noalloc(abi.JP_NOALLOC_MAX_ATOMS + 1, None, None, None, 1, None,
                                       None, None, None, 0, box, 12.0, 1.0, None, None, None)
    assert rc == abi.JP_E_NOALLOC_LIMIT
    assert b"JP_NOALLOC_MAX_ATOMS" in engine_lib.jp_strerror(rc)


@pytest.mark.gpu
def test_noalloc_matches_energy_grad(engine_lib):
    import torch
    from j_presto_b200 import engine

    top = _water()
    n = int(top["natom"])
    assert n <= abi.JP_NOALLOC_MAX_ATOMS
    with engine.Engine(top, precision=abi.JP_PREC_FP64, method=abi.JP_METHOD_MICR) as e:
        ene_ref, grad_ref = e.energy_grad()
        rc_cut = e.params.cutoff
        eps = e.params.dielectric

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)

    def d(a, dt):
        return torch.as_tensor(np.ascontiguousarray(a), dtype=dt).to(dev)

    cord = d(top["cord"], torch.float64)
    chg = d(top["charge"], torch.float64)
    typ = d(top["atype"], torch.int32)
    c6 = d(top["c6"], torch.float64)
    c12 = d(top["c12"], torch.float64)
    eptr = d(top["excl_ptr"], torch.int32)
    eidx = d(top["excl_idx"], torch.int32)
    grad = torch.empty((n, 3), dtype=torch.float64, device=dev)
    ene = torch.empty(2, dtype=torch.float64, device=dev)
    box = (C.c_double * 3)(*[float(b) for b in top["box"]])
    stream = torch.cuda.current_stream(dev).cuda_stream

    def call(atype, excl_idx, base, excl_ptr=None):
        grad.fill_(np.nan)
        ene.fill_(np.nan)
        ep = eptr if excl_ptr is None else excl_ptr
        return engine_lib.jp_nonbond_noalloc(n, cord.data_ptr(), chg.data_ptr(), atype.data_ptr(),
                                             int(top["ntype"]), c6.data_ptr(), c12.data_ptr(),
                                             ep.data_ptr(), excl_idx.data_ptr(), base, box,
                                             rc_cut, eps, grad.data_ptr(), ene.data_ptr(), stream)

    def check():
        g = grad.cpu().numpy()
        en = ene.cpu().numpy()
        assert rms_rel(g, grad_ref) < 1e-12
        np.testing.assert_allclose(en[0], ene_ref[ELE15], rtol=1e-8, atol=1e-7)
        np.testing.assert_allclose(en[1], ene_ref[VDW15], rtol=1e-8, atol=1e-7)

    # two calls in a row share (and re-clear) the static scratch
    for _ in range(2):
        assert call(typ, eidx, 0) == abi.JP_OK
        check()
    # Fortran numbering of the same system
    assert call(typ + 1, eidx + 1, 1) == abi.JP_OK
    check()
    # an out-of-range type index is caught by the kernel's own check
    bad = typ.clone()
    bad[5] = int(top["ntype"])
    assert call(bad, eidx, 0) == abi.JP_E_INVALID
    # so is a decreasing exclusion offset (every offset stays inside the partner list, so the
    # check, not an out-of-range read, decides)
    badp = eptr.clone()
    assert int(badp[5]) >= 1
    badp[6] = badp[5] - 1
    assert call(typ, eidx, 0, badp) == abi.JP_E_INVALID
    # and the next call is unaffected
    assert call(typ, eidx, 0) == abi.JP_OK
    check()
