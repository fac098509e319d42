"""Local kinetic energy from the evaluateGL arrays, and checkpoint /
restore of a batch's walker state."""
import numpy as np
import pytest

from miniqmc_b200 import api, capi
from tests import gpu_helpers as H
from tests.test_gpu_parity import elem_rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('precision', [capi.PREC_FP64, capi.PREC_MIXED])
def test_local_kinetic(precision):
    gw, ow = H.make_pair(precision=precision, walkers=3, delay=4)
    gw.evaluate_log()
    ow.evaluate_log()
    ur, de = H.host_streams(H.oracle_primes(3), gw.N, 1, 1)
    gw.sweep(1, 1, 0.5, ur=ur, delta=de)
    ow.sweep(1, 1, 0.5, ur=ur, delta=de)
    G, L, _ = gw.evaluate_gl()
    ke = gw.local_kinetic()
    ref = -0.5 * (L.sum(axis=1) + (G ** 2).sum(axis=(1, 2)))
    assert elem_rel(ke, ref).max() < 1e-12
    Go, Lo, _ = ow.evaluate_gl()
    ke_o = -0.5 * (Lo.sum(axis=1) + (Go ** 2).sum(axis=(1, 2)))
    assert elem_rel(ke, ke_o).max() < (1e-9 if precision == capi.PREC_FP64 else 1e-3)


@pytest.mark.parametrize('precision', [capi.PREC_FP64, capi.PREC_MIXED])
def test_checkpoint_restore_continues_exactly(precision):
    lib = H.product()
    spec = api.SystemSpec(lib, cell=capi.NIO_PRIM4, tiling=(2, 1, 1), grid=(24, 12, 12), jastrow='synthetic')
    system = api.System(lib, spec, precision)
    seeds = np.arange(5, dtype=np.uint32) * 7919 + 3
    a = api.Walkers(system, 5, 8)
    a.init_random(seeds)
    a.evaluate_log()
    a.sweep(3, 1, 0.5, recompute_every=4)
    snap = a.checkpoint()
    ra = a.sweep(3, 1, 0.5, recompute_every=4)
    b = api.Walkers(system, 5, 8)
    b.restore(snap)
    rb = b.sweep(3, 1, 0.5, recompute_every=4)
    assert np.array_equal(ra['accepted'], rb['accepted'])
    assert np.array_equal(ra['logpsi'], rb['logpsi'])
    assert np.array_equal(a.positions(), b.positions())
    # a batch of another shape refuses the checkpoint
    c = api.Walkers(system, 4, 8)
    with pytest.raises(api.QMCError):
        c.restore(snap)
