"""Shared check of a batch against the reference's determinant golden dump
(tests/golden/reference_det_dump.json, printed by oracle/ref_det_harness.cpp
from the reference's own DiracDeterminant<DelayedUpdate<double,double>> and
DiracMatrix over OpenBLAS): the reference's NiO cell at -g "1 1 1" (384
electrons, 192 orbitals per spin), a 16x16x16 table with the uniform fill,
determinants only, electrons and one substep of moves from the stream of the
first prime, delay ranks 1 and 32.

Tolerances: log|det| 1e-12 relative; every move's ratio 1e-11 relative at
the median and 5e-9 at the worst (the near-node moves of the threshold rule,
|ratio| down to 2e-3, amplify round-off); gradients 1e-8 of their largest
magnitude; the inverse's rows after completeUpdates 1e-10 of their largest
entry; the accept sequence exact."""
import json
import os

import numpy as np

from miniqmc_b200 import api, capi
from tests import gpu_helpers as H
from tests import oracle_lib

DUMP = json.load(open(os.path.join(oracle_lib.GOLDEN, 'reference_det_dump.json')))


def check(lib, delay):
    x = DUMP['det_k%d' % delay]
    spec = api.SystemSpec(lib, cell=capi.NIO_REF32, tiling=(1, 1, 1),
                          quirks=capi.NIO_QUIRK_UNIT_IONS | capi.NIO_QUIRK_ONE_GROUP, grid=tuple(x['grid']),
                          fill=capi.FILL_UNIFORM, spo_seed=11, jastrow='reference', components=capi.WF_DET)
    system = api.System(lib, spec, capi.PREC_FP64)
    w = api.Walkers(system, 1, delay)
    seeds = H.oracle_primes(1)
    w.init_random(seeds)
    w.evaluate_log()
    c = w.components()[0]
    np.testing.assert_allclose(c[:2], x['log_init'], rtol=1e-12)
    np.testing.assert_allclose(c[2:4], x['phase_init'], atol=1e-12)
    ur, de = H.host_streams(seeds, spec.n_elec, 1, 1)
    t = w.sweep(1, 1, 0.5, ur=ur, delta=de, trace=True)['trace'].reshape(-1, 8)
    assert np.array_equal(t[:, 7], np.array(x['accept'], dtype=float))
    ref = np.array(x['ratio'])
    rel = np.abs(t[:, 0] - ref) / np.abs(ref)
    assert np.median(rel) < 1e-11 and rel.max() < 5e-9, (np.median(rel), rel.max())
    for col, key in ((slice(1, 4), 'grad_new'), (slice(4, 7), 'grad_now')):
        g = np.array(x[key]).reshape(-1, 3)
        assert np.abs(t[:, col] - g).max() < 1e-8 * np.abs(g).max(), key
    c = w.components()[0]
    np.testing.assert_allclose(c[:2], x['log_after'], rtol=1e-12)
    for s, name in ((0, 'up'), (1, 'dn')):
        inv = w.inverse(0, s)
        for row in (0, 96, 191):
            r = np.array(x['psiM_%s_row%d' % (name, row)])
            assert np.abs(inv[row] - r).max() < 1e-10 * np.abs(r).max(), (name, row)
    w.evaluate_log()
    np.testing.assert_allclose(w.components()[0][:2], x['log_fresh'], rtol=1e-12)
    w.close()
    system.close()
