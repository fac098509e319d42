"""The fused sweep's work-queue schedule (qmc_walkers_set_schedule) against
the static one.  The same walkers are swept by fewer CTAs than walkers in
units of a few moves, so that nearly every unit boundary hands a walker to
another CTA (and another SM); the results must be the static form's bit for
bit: the per-move trace (ratio, gradient, accept flag of every move), the
accepted counts, the log values after each step, the positions and the G, L
of a fresh evaluateGL.  Covered: FP64 and mixed precision, the CUDA-core and
the tensor-core Woodbury flush, the three-body Jastrow, moves evaluated in
epochs, host and device random streams, several substeps, units of one move
and units longer than a spin.  A tensor-core wait that runs out in the queue
form stops every CTA and reports QMC_ERR_TIMEOUT, after which the batch
rebuilds and sweeps like a static one."""
import numpy as np
import pytest

from miniqmc_b200 import api, capi
from tests import gpu_helpers as H

pytestmark = pytest.mark.gpu

SMALL = dict(tiling=(1, 1, 2), grid=(12, 12, 12))
# NiO 4x4x2 of the 4-atom cell: 768 orbitals per spin, the tensor-core flush
NIO128 = dict(tiling=(4, 4, 2), grid=(24, 24, 12), jastrow='synthetic')


def _batch(spec, precision, W, delay, seeds, mode, unit=0, ctas=0, moves=1, tc=None, threads=0):
    lib = H.product()
    w = api.Walkers(api.System(lib, spec, precision), W, delay)
    w.init_random(seeds)
    if threads:
        lib.call('walkers_set_threads', w.h, threads)
    w.set_schedule(mode, unit, ctas)
    if moves > 1:
        lib.call('walkers_set_move_batching', w.h, moves)
    if tc is not None:
        lib.call('walkers_set_tensor_cores', w.h, tc)
    return w


def _compare(kw, precision, W, delay, unit, ctas, steps=2, substeps=1, host_rng=False, moves=1, tc=None,
             components=capi.WF_ALL, threads=0):
    sp, _ = H.spec_pair(components=components, **kw)
    seeds = H.oracle_primes(W)
    a = _batch(sp, precision, W, delay, seeds, capi.SCHED_STATIC, moves=moves, tc=tc, threads=threads)
    b = _batch(sp, precision, W, delay, seeds, capi.SCHED_QUEUE, unit, ctas, moves=moves, tc=tc, threads=threads)
    assert np.array_equal(a.evaluate_log(), b.evaluate_log())
    ur = de = None
    if host_rng:
        ur, de = H.host_streams(seeds, a.N, steps, substeps)
    acc = 0
    for s in range(steps):
        args = dict(ur=ur[s:s + 1], delta=de[s:s + 1]) if host_rng else {}
        ra = a.sweep(1, substeps, 0.5, trace=True, **args)
        rb = b.sweep(1, substeps, 0.5, trace=True, **args)
        assert np.array_equal(ra['trace'], rb['trace'], equal_nan=True), s
        assert np.array_equal(ra['accepted'], rb['accepted']), s
        assert np.array_equal(ra['logpsi'], rb['logpsi']), s
        acc += int(rb['trace'][..., 7].sum())
    assert acc > 0
    assert np.array_equal(a.positions(), b.positions())
    ga, gb = a.evaluate_gl(), b.evaluate_gl()
    for x, y in zip(ga, gb):
        assert np.array_equal(x, y)
    a.close()
    b.close()


@pytest.mark.parametrize('precision', [capi.PREC_FP64, capi.PREC_MIXED])
@pytest.mark.parametrize('threads', [0, 256])
def test_queue_equals_static_small(precision, threads):
    # 5 walkers on 2 CTAs, units of 3 moves, 2 substeps, device streams;
    # the default block and a 256-thread one (the queue kernel's two
    # register budgets)
    _compare(SMALL, precision, 5, 4, unit=3, ctas=2, substeps=2, threads=threads)


def test_queue_units_of_one_move_host_streams():
    _compare(SMALL, capi.PREC_MIXED, 6, 8, unit=1, ctas=4, host_rng=True)


def test_queue_units_longer_than_a_spin():
    # one unit per spin and substep, one CTA per walker
    _compare(SMALL, capi.PREC_MIXED, 4, 4, unit=100000, ctas=4)


def test_queue_three_body_jastrow():
    _compare(SMALL, capi.PREC_FP64, 4, 4, unit=5, ctas=3, components=capi.WF_ALL | capi.WF_J3)


def test_queue_jastrow_only():
    # no determinant: no Binv to carry between units, no flushes
    _compare(SMALL, capi.PREC_MIXED, 5, 4, unit=7, ctas=2, components=capi.WF_J1 | capi.WF_J2)


def test_queue_epochs():
    _compare(SMALL, capi.PREC_MIXED, 4, 8, unit=7, ctas=2, moves=4)


@pytest.mark.parametrize('tc', [0, 1])
def test_queue_nio128_flushes(tc):
    # delay 32 at 768 orbitals: the units cross the flushes of both engines
    _compare(NIO128, capi.PREC_MIXED, 3, 32, unit=16, ctas=2, steps=1, tc=tc)


def test_queue_rejects_bad_settings():
    sp, _ = H.spec_pair(**SMALL)
    w = _batch(sp, capi.PREC_FP64, 2, 4, H.oracle_primes(2), capi.SCHED_AUTO)
    for bad in ((3, 0, 0), (-1, 0, 0), (capi.SCHED_QUEUE, -1, 0), (capi.SCHED_QUEUE, 0, -2)):
        with pytest.raises(api.QMCError) as e:
            H.product().call('walkers_set_schedule', w.h, *bad)
        assert e.value.status == 1  # QMC_ERR_ARG
    w.close()


def test_queue_timeout_stops_and_recovers():
    """Wait limit 0: the first tensor-core wait of some unit gives up; its CTA
    raises the stop flag, the others stop taking units (or leave their wait
    for a walker's previous unit), and the status read reports the timeout.
    Rebuilt from its positions, the batch then sweeps like a static batch
    placed at the same positions."""
    sp, _ = H.spec_pair(**NIO128)
    seeds = H.oracle_primes(3)
    lib = H.product()
    b = _batch(sp, capi.PREC_MIXED, 3, 32, seeds, capi.SCHED_QUEUE, 16, 2, tc=1)
    b.evaluate_log()
    lib.call('walkers_set_wait_limit', b.h, 0)
    with pytest.raises(api.QMCError) as ex:
        b.sweep(1, 1, 0.5)
    assert ex.value.status == 6  # QMC_ERR_TIMEOUT
    lib.call('walkers_set_wait_limit', b.h, 2000000000)
    a = _batch(sp, capi.PREC_MIXED, 3, 32, seeds, capi.SCHED_STATIC, tc=1)
    R = b.positions()
    a.set_positions(R)
    b.set_positions(R)
    assert np.array_equal(a.evaluate_log(), b.evaluate_log())
    ur, de = H.host_streams(seeds, a.N, 1, 1)
    ra = a.sweep(1, 1, 0.5, ur=ur, delta=de, trace=True)
    rb = b.sweep(1, 1, 0.5, ur=ur, delta=de, trace=True)
    assert np.array_equal(ra['trace'], rb['trace'])
    assert np.array_equal(ra['logpsi'], rb['logpsi'])
    a.close()
    b.close()
