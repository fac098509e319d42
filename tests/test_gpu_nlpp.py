"""Non-local pseudopotential ratios (qmc_nlpp_evaluate) against the FP64
oracle's restatement of the reference loop (miniqmc.cpp:472-495,
NonLocalPP.hpp:115-134): same points counted, same ratios."""
import numpy as np
import pytest

from miniqmc_b200 import api, capi
from tests import gpu_helpers as H
from tests.test_gpu_parity import elem_rel, rel_err

pytestmark = pytest.mark.gpu


def _pair(precision, tiling=(1, 1, 1), walkers=2, delay=4):
    gw, ow = H.make_pair(precision=precision, walkers=walkers, delay=delay, tiling=tiling,
                         grid=tuple(12 * t for t in tiling), jastrow='synthetic')
    gw.evaluate_log()
    ow.evaluate_log()
    return gw, ow


@pytest.mark.parametrize('form', [capi.NLPP_SPHERE, capi.NLPP_DRIVER])
def test_nlpp_fp64_matches_oracle(form):
    gw, ow = _pair(capi.PREC_FP64)
    for call in range(2):  # the second call uses the stream's second rotation
        ng, wg, rg = gw.nlpp(1.7, form, max_ratios=4096)
        no, wo, ro = ow.nlpp(1.7, form, max_ratios=4096)
        assert np.array_equal(ng, no) and ng[0] > 0, (ng, no)
        assert elem_rel(wg, wo).max() < 1e-10
        m = int(ng[0])
        assert rel_err(rg[:m], ro[:m]) < 1e-10
        # a step between the calls: NLPP sees the swept walkers
        ur, de = H.host_streams(H.oracle_primes(2), gw.N, 1, 1)
        gw.sweep(1, 1, 0.5, ur=ur, delta=de)
        ow.sweep(1, 1, 0.5, ur=ur, delta=de)


def test_nlpp_larger_cell_fp64():
    gw, ow = _pair(capi.PREC_FP64, tiling=(2, 2, 1), walkers=1, delay=8)
    ng, wg, rg = gw.nlpp(1.7, capi.NLPP_SPHERE, max_ratios=1 << 15)
    no, wo, ro = ow.nlpp(1.7, capi.NLPP_SPHERE, max_ratios=1 << 15)
    assert np.array_equal(ng, no)
    m = int(ng[0])
    assert rel_err(rg[:m], ro[:m]) < 1e-9 and elem_rel(wg, wo).max() < 1e-9


def test_nlpp_mixed_precision():
    """FP32 orbitals, inverse rows and Jastrows: ratio errors at FP32
    rounding amplified by the ratio dots' cancellation."""
    gw, ow = _pair(capi.PREC_MIXED)
    ng, wg, rg = gw.nlpp(1.7, capi.NLPP_SPHERE, max_ratios=4096)
    no, wo, ro = ow.nlpp(1.7, capi.NLPP_SPHERE, max_ratios=4096)
    assert np.array_equal(ng, no)
    m = int(ng[0])
    e = elem_rel(rg[:m], ro[:m])
    assert np.median(e) < 1e-5 and np.percentile(e, 99) < 1e-2, (np.median(e), np.percentile(e, 99))


def test_nlpp_needs_complete_updates():
    gw, _ = _pair(capi.PREC_FP64, delay=4)
    lib = H.product()
    iat = 3
    lib.call('pset_set_active', gw.h, iat)
    d = np.full((gw.W, 3), 0.05)
    lib.call('pset_make_move', gw.h, iat, d.ctypes.data_as(capi.PD))
    r = np.zeros(gw.W)
    g = np.zeros((gw.W, 3))
    lib.call('wf_ratio_grad', gw.h, iat, r.ctypes.data_as(capi.PD), g.ctypes.data_as(capi.PD))
    acc = np.ones(gw.W, dtype=np.int32)
    lib.call('wf_accept_restore', gw.h, iat, acc.ctypes.data_as(capi.PI))
    lib.call('pset_accept_reject', gw.h, iat, acc.ctypes.data_as(capi.PI))
    with pytest.raises(api.QMCError) as ei:
        gw.nlpp(1.7)
    assert capi.STATUS[ei.value.status] == 'QMC_ERR_STATE'
    lib.call('wf_complete_updates', gw.h)
    n, _, _ = gw.nlpp(1.7)
    assert n[0] > 0
