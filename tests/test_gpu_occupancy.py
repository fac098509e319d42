"""Walkers per SM of the fused sweep (qmc_walkers_occupancy) at the NiO-128
size.  In the static schedule the headline configuration (512 walkers,
delay 32, the tensor-core flush, 192 threads per walker) needs four walkers
per SM to run in one wave on 148 SMs: the kernel sits at its 80-register cap
and 4 x 57 KB of shared memory, so a few hundred bytes more of static shared
memory drop it to three and the step to 1.5x the time (seen once: 170 -> 256
ms).  The work-queue schedule (the default at 512 walkers) runs three CTAs
per SM at up to 112 registers instead and time-slices the walkers over them.
This pins both."""
import pytest

from miniqmc_b200 import api, capi
from tests import gpu_helpers as H

pytestmark = pytest.mark.gpu


def _occupancy(delay, tensor_cores, precision=capi.PREC_MIXED, schedule=capi.SCHED_STATIC):
    lib = H.product()
    spec = api.SystemSpec(lib, cell=capi.NIO_PRIM4, tiling=(4, 4, 2), grid=(24, 24, 12), fill=capi.FILL_UNIFORM,
                          spo_seed=11, jastrow='synthetic')
    system = api.System(lib, spec, precision)
    w = api.Walkers(system, 1, delay)
    lib.call('walkers_set_schedule', w.h, schedule, 0, 0)
    if precision == capi.PREC_MIXED:
        lib.call('walkers_set_tensor_cores', w.h, 1 if tensor_cores else 0)
    import ctypes as C
    n = C.c_int()
    lib.call('walkers_occupancy', w.h, C.byref(n))
    threads, k, tc = C.c_int(), C.c_int(), C.c_int()
    lib.call('walkers_get_config', w.h, C.byref(threads), C.byref(k), C.byref(tc))
    w.close()
    system.close()
    return n.value, threads.value


def test_headline_configuration_holds_four_walkers_per_sm():
    n, threads = _occupancy(32, True)
    assert threads == 192
    assert n >= 4, n


def test_queue_form_runs_three_ctas_per_sm():
    n, threads = _occupancy(32, True, schedule=capi.SCHED_QUEUE)
    assert threads == 192
    assert n == 3, n


def test_occupancy_of_the_delay_ranks():
    """Delay 16 keeps four walkers per SM; delay 64 takes more shared
    memory (its Binv cache 32 KB, the tensor-core tiles 96 KB), so fewer."""
    got = {}
    for delay in (16, 32, 64):
        for tc in (True, False):
            got[delay, tc] = _occupancy(delay, tc)[0]
            print('delay %d, %s flush: %d walkers per SM' % (delay, 'tensor-core' if tc else 'CUDA-core',
                                                            got[delay, tc]))
    assert got[16, True] >= 4
    assert got[64, True] == 2
    assert 2 <= got[64, False] < 4
