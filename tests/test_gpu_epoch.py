"""The fused sweep's epochs (qmc_walkers_set_move_batching) against one move
at a time.

The reference's accept rule compares a uniform with a fixed threshold
(miniqmc.cpp:445), so the run of moves from one accepted move to the next
sees one walker state; the sweep evaluates up to four such moves together.
Per move the arithmetic is that of one-at-a-time evaluation, so every ratio,
gradient, accept flag, log value and the final positions must be the same
bit for bit, in both arithmetic forms and with either Woodbury flush, for
host and device random streams and for wavefunctions with and without the
determinant."""
import ctypes as C

import numpy as np
import pytest

from miniqmc_b200 import api, capi
from tests import gpu_helpers as H

pytestmark = pytest.mark.gpu


def _batch(precision, tiling, grid, delay, walkers, components=capi.WF_ALL, tc=None):
    spec = api.SystemSpec(H.product(), tiling=tiling, grid=grid, jastrow='synthetic', components=components)
    system = api.System(H.product(), spec, precision)
    out = []
    for moves in (1, 2, 4):
        w = api.Walkers(system, walkers, delay)
        if tc is not None:
            H.product().call('walkers_set_tensor_cores', w.h, 1 if tc else 0)
        H.product().call('walkers_set_move_batching', w.h, moves)
        w.init_random((np.arange(walkers, dtype=np.uint32) * 7919 + 1009).astype(np.uint32))
        w.evaluate_log()
        out.append(w)
    return spec, system, out


def _same(runs, ws):
    for r in runs[1:]:
        assert np.array_equal(r['trace'], runs[0]['trace'])
        assert np.array_equal(r['logpsi'], runs[0]['logpsi'])
        assert np.array_equal(r['accepted'], runs[0]['accepted'])
    for w in ws[1:]:
        assert np.array_equal(w.positions(), ws[0].positions())
        assert np.array_equal(w.components(), ws[0].components())


@pytest.mark.parametrize('precision,tc', [(capi.PREC_FP64, None), (capi.PREC_MIXED, True), (capi.PREC_MIXED, False)])
def test_epochs_equal_single_moves_nio128(precision, tc):
    spec, system, ws = _batch(precision, (4, 4, 2), (24, 24, 12), 32, 2, tc=tc)
    rs = np.random.default_rng(7)
    ur = rs.uniform(size=(2, 2, 1, spec.n_elec))
    de = rs.normal(size=(2, 2, 1, spec.n_elec, 3))
    runs = [w.sweep(2, 1, 0.5, ur=ur, delta=de, trace=True) for w in ws]
    _same(runs, ws)
    # the runs contain epochs of every length up to 4
    acc = runs[0]['trace'][..., 7].ravel()
    assert 0.4 < acc.mean() < 0.6


@pytest.mark.parametrize('precision', [capi.PREC_FP64, capi.PREC_MIXED])
def test_epochs_equal_single_moves_small_device_rng(precision):
    """48 electrons, delay 4, two substeps, device random streams and an
    acceptance threshold of 0.3 (longer runs of rejected moves)."""
    spec, system, ws = _batch(precision, (1, 1, 1), (12, 12, 12), 4, 3)
    runs = []
    for w in ws:
        acc = np.zeros(3, dtype=np.int64)
        lp = np.zeros(3)
        o = capi.SweepOpts()
        o.n_steps, o.n_substeps, o.accept, o.rng_mode = 2, 2, 0.3, capi.RNG_DEVICE
        tr = np.zeros((2, 3, 2, spec.n_elec, 8))
        o.trace = tr.ctypes.data_as(capi.PD)
        o.n_accepted = acc.ctypes.data_as(C.POINTER(C.c_int64))
        o.logpsi = lp.ctypes.data_as(capi.PD)
        H.product().call('sweep', w.h, C.byref(o))
        runs.append({'trace': tr, 'logpsi': lp, 'accepted': acc})
    _same(runs, ws)


def test_epochs_equal_single_moves_jastrow_only():
    spec, system, ws = _batch(capi.PREC_MIXED, (2, 1, 1), (12, 12, 12), 4, 2, components=capi.WF_J1 | capi.WF_J2)
    rs = np.random.default_rng(9)
    ur = rs.uniform(size=(1, 2, 1, spec.n_elec))
    de = rs.normal(size=(1, 2, 1, spec.n_elec, 3))
    _same([w.sweep(1, 1, 0.5, ur=ur, delta=de, trace=True) for w in ws], ws)


def test_move_batching_rejects_bad_values():
    spec, system, ws = _batch(capi.PREC_FP64, (1, 1, 1), (12, 12, 12), 2, 1)
    for bad in (0, 5, -1):
        with pytest.raises(api.QMCError):
            H.product().call('walkers_set_move_batching', ws[0].h, bad)
