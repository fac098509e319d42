"""The bounded waits of the tensor-core Woodbury flush run out and return.

Every wait of the flush on its MMAs (mbarrier try_wait on a tcgen05.commit)
gives up after the batch's limit (qmc_walkers_set_wait_limit).  With a limit
of 0 the first wait gives up at once: no fault, no hang, only a short wait
that returns.  The launch then unwinds, the CTA drains its own MMAs before it
frees its tensor memory, and the status read reports QMC_ERR_TIMEOUT.  The
reference has no device waits (it aborts the process on errors,
Configuration.h:35-39), so the checks are: the sweep returns, the status is
the timeout, the batch rebuilds from its positions and then sweeps to the
FP64 oracle, the handle can be destroyed, and a fresh batch sweeps to the
oracle on the same GPU context."""
import numpy as np
import pytest

from miniqmc_b200 import api, capi
from tests import gpu_helpers as H
from tests.test_gpu_parity import elem_rel

pytestmark = pytest.mark.gpu

# NiO 4x4x2 of the 4-atom cell (768 orbitals per spin: 192 threads per
# walker, so the FP32 flush runs on the tensor cores), on a coarse grid
KW = dict(tiling=(4, 4, 2), grid=(24, 24, 12), jastrow='synthetic')
DELAY = 32


def _tc_pair(walkers, seeds):
    gw, ow = H.make_pair(precision=capi.PREC_MIXED, walkers=walkers, delay=DELAY, seeds=seeds, **KW)
    H.product().call('walkers_set_tensor_cores', gw.h, 1)
    return gw, ow


def _sweep_pair(a, b, seeds, step):
    ur, de = H.host_streams(seeds, a.N, step + 1, 1)
    ur, de = ur[step:step + 1], de[step:step + 1]
    return (a.sweep(1, 1, 0.5, ur=ur, delta=de, trace=True), b.sweep(1, 1, 0.5, ur=ur, delta=de, trace=True))


def test_wait_limit_timeout_unwinds_and_recovers():
    seeds = H.oracle_primes(2)
    gw, ow = _tc_pair(2, seeds)
    gw.evaluate_log()
    ow.evaluate_log()
    H.product().call('walkers_set_wait_limit', gw.h, 0)
    ur, de = H.host_streams(seeds, gw.N, 1, 1)
    with pytest.raises(api.QMCError) as ex:
        gw.sweep(1, 1, 0.5, ur=ur, delta=de)
    assert ex.value.status == 6  # QMC_ERR_TIMEOUT
    # the status was read and cleared: the batch answers again.  Rebuilt
    # from its positions it must sweep exactly like a batch that never
    # timed out, placed at the same positions, and keep the oracle's accept
    # sequence.
    H.product().call('walkers_set_wait_limit', gw.h, 2000000000)
    R = gw.positions()
    g_new, _ = _tc_pair(2, seeds)
    for w in (ow, g_new):
        w.set_positions(R)
    lg, ln, lo = gw.evaluate_log(), g_new.evaluate_log(), ow.evaluate_log()
    assert np.array_equal(lg, ln)
    assert elem_rel(lg, lo).max() < 1e-7
    rg, rn = _sweep_pair(gw, g_new, seeds, 1)
    assert np.array_equal(rg['trace'], rn['trace'])
    assert np.array_equal(rg['logpsi'], rn['logpsi'])
    _, ro = _sweep_pair(gw, ow, seeds, 1)  # the oracle's step 1 (gw's output unused)
    assert np.array_equal(rg['trace'][..., 7], ro['trace'][..., 7])
    gw.close()
    g_new.close()
    # a fresh batch on the same context keeps the oracle's accept sequence
    g2, o2 = _tc_pair(2, seeds)
    g2.evaluate_log()
    o2.evaluate_log()
    r2, r2o = _sweep_pair(g2, o2, seeds, 0)
    assert np.array_equal(r2['trace'][..., 7], r2o['trace'][..., 7])
    assert np.array_equal(r2['accepted'], r2o['accepted'])
    g2.close()


def test_wait_limit_rejects_negative():
    gw, _ = _tc_pair(1, H.oracle_primes(1))
    with pytest.raises(api.QMCError):
        H.product().call('walkers_set_wait_limit', gw.h, -1)
    gw.close()
