"""The reference's own drivers, unmodified, on the device through the adapter
classes (miniqmc_b200/adapter/): Drivers/miniqmc.cpp (one walker per mover,
the per-walker WaveFunction verbs, NLPP through WaveFunction::ratio) and
Drivers/miniqmc_sync_move.cpp (flex_ verbs over a batch of movers, NLPP
through WaveFunction::evaluateRatios); and the reference's SPO set against
the SPOSet adapter (check_spo_gpu).  Each walker's counters and last log
value (QMCGPU_ADAPTER_REPORT) are compared with the oracle driven through
the C ABI over the same system, random streams and NLPP spheres.

The binaries are linked from the reference's sources where they lie
(adapter.mk); where they were not built the tests are skipped."""
import json
import os
import subprocess

import numpy as np
import pytest

from miniqmc_b200 import api, capi
from tests import oracle_lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, 'miniqmc_b200', 'bin')
MINIQMC = os.path.join(BIN, 'ref_miniqmc')
SYNC = os.path.join(BIN, 'ref_miniqmc_sync_move')
CHECK_SPO = os.path.join(BIN, 'check_spo_gpu')
PRIMES = [3, 5, 7, 11]  # PrimeNumberSet<uint32_t> from 3
QUIRKS = 3  # the reference's 32-atom cell at -g "1 1 1": ions in lattice units, one species group

needs_binaries = pytest.mark.skipif(not all(os.path.exists(b) for b in (MINIQMC, SYNC, CHECK_SPO)),
                                    reason='reference drivers on the device not built (no reference tree)')


def run(exe, args, report, threads, extra_env=None):
    env = dict(os.environ, QMCGPU_SPO_FILL='uniform', QMCGPU_ADAPTER_REPORT=report, OMP_NUM_THREADS=str(threads))
    env.update(extra_env or {})
    if os.path.exists(report):
        os.remove(report)
    r = subprocess.run([exe, *args], capture_output=True, text=True, timeout=900, env=env, cwd=os.path.dirname(report))
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    with open(report) as f:
        return [json.loads(line) for line in f], r


def oracle_system(grid, j3=False):
    lib = oracle_lib.library()
    spec = api.SystemSpec(lib, cell=capi.NIO_REF32, tiling=(1, 1, 1), quirks=QUIRKS, grid=grid, fill=capi.FILL_UNIFORM,
                          spo_seed=11, jastrow='reference', components=capi.WF_ALL | (capi.WF_J3 if j3 else 0))
    return lib, spec, api.System(lib, spec, capi.PREC_FP64)


def match(reports, walkers_r0):
    """The report line of each oracle walker, by the first electron's
    initial position (the drivers build their movers in any order)."""
    out = []
    for r0 in walkers_r0:
        hits = [r for r in reports if np.allclose(r['r0'], r0, rtol=0, atol=1e-12)]
        assert len(hits) == 1, (r0, [r['r0'] for r in reports])
        out.append(hits[0])
    return out


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


# Over the oracle (the CPU shim) the adapter's run is the oracle's own loop:
# equal but for the order of a few sums.  On the device the FP64 kernels
# differ from the oracle in summation order, and the threshold rule accepts
# moves close to a node, where the ratios amplify that round-off: measured
# log psi 3.4e-12, sum of log ratios 4.0e-8, NLPP ratio sum 7.4e-9 at
# worst over the six walkers; the bounds are 7-30 times that.
EXACT = dict(log=1e-12, sum_log_ratio=1e-12, sum_virtual=1e-12)
DEVICE = dict(log=1e-10, sum_log_ratio=1e-6, sum_virtual=5e-8)


def compare(got, i, acc, slr, lp, n_virtual, wsum, steps, N, batch, tol):
    g = got[i]
    errs = dict(log=rel(g['log'], lp[i]), sum_log_ratio=rel(g['sum_log_ratio'], slr[i]),
                sum_virtual=rel(g['sum_virtual'] / 12.0, wsum[i]))
    print('walker %d: accepted %d, NLPP points %d, relative errors %s' % (i, acc[i], n_virtual[i], errs))
    assert g['status'] == 0 and g['batch'] == batch
    assert g['ratio_grad'] == steps * N and g['accepted'] == acc[i]
    assert g['virtual'] == n_virtual[i] and n_virtual[i] > 0
    for key, e in errs.items():
        assert e < tol[key], (key, e)


def check_miniqmc_driver(tmp_path, j3, tol, extra_env=None):
    """Drivers/miniqmc.cpp, 2 movers on 2 threads (seeds by thread: 3, 5),
    2 steps, delay 8, NLPP within the default rmax 1.7."""
    steps, k = 2, 8
    reports, out = run(MINIQMC, ['-g', '1 1 1', '-m', '0.5', '-w', '2', '-n', str(steps), '-k', str(k),
                                 *(['-j'] if j3 else [])], str(tmp_path / 'report.jsonl'), 2, extra_env)
    assert 'Diffusion throughput' in out.stdout
    lib, spec, system = oracle_system((18, 18, 18), j3)
    N = spec.n_elec
    w = api.Walkers(system, 2, k)
    seeds = np.array(PRIMES[:2], dtype=np.uint32)
    w.init_random(seeds)
    got = match(reports, w.positions()[:, 0])
    w.evaluate_log()
    from tests import gpu_helpers as H
    ur, de = H.host_streams(seeds, N, steps, 1)
    acc = np.zeros(2, dtype=np.int64)
    slr = np.zeros(2)
    n_virtual = np.zeros(2, dtype=np.int64)
    wsum = np.zeros(2)
    for st in range(steps):
        for iel in range(N):
            w.eval_grad(iel)
            w.make_move(iel, de[st, :, 0, iel])
            r, _ = w.ratio_grad(iel)
            slr += np.log(np.abs(r))
            a = (ur[st, :, 0, iel] < 0.5).astype(np.int32)
            acc += a
            w.accept_restore(iel, a)
            w.accept_reject(iel, a)
        w.complete_updates()
        _, _, lp = w.evaluate_gl()
        npt, ws, _ = w.nlpp(1.7, capi.NLPP_DRIVER)
        n_virtual += npt
        wsum += ws
    for i in range(2):
        compare(got, i, acc, slr, lp, n_virtual, wsum, steps, N, 1, tol)


@needs_binaries
@pytest.mark.gpu
@pytest.mark.parametrize('j3', [False, True])
def test_reference_miniqmc_driver(tmp_path, j3):
    check_miniqmc_driver(tmp_path, j3, DEVICE)


def check_sync_move_driver(tmp_path, tol, extra_env=None, j3=False):
    """Drivers/miniqmc_sync_move.cpp, 4 movers in 2 batches of 2 (one device
    batch each, one launch per verb), 2 steps, delay 8, NLPP through
    NonLocalPP::evaluate's virtual particle sets; with -j the three-body
    Jastrow in every verb and virtual ratio."""
    steps, k, nw = 2, 8, 2
    reports, out = run(SYNC, ['-g', '1 1 1', '-m', '0.5', '-w', '4', '-c', str(nw), '-n', str(steps), '-k', str(k),
                              *(['-j'] if j3 else [])], str(tmp_path / 'report.jsonl'), 1, extra_env)
    assert 'Diffusion throughput' in out.stdout
    lib, spec, system = oracle_system((18, 18, 18), j3)
    N = spec.n_elec
    per = nw + 2 * ((3 * nw + 1) // 2)
    for first in (0, 2):
        w = api.Walkers(system, nw, k)
        w.init_random(np.array(PRIMES[first:first + nw], dtype=np.uint32))
        got = match(reports, w.positions()[:, 0])
        w.evaluate_log()
        u = np.zeros(3 * N + steps * N * per)
        lib.fn['rng_uniform'](PRIMES[first], len(u), oracle_lib.pd(u))
        acc = np.zeros(nw, dtype=np.int64)
        slr = np.zeros(nw)
        n_virtual = np.zeros(nw, dtype=np.int64)
        wsum = np.zeros(nw)
        for st in range(steps):
            for iel in range(N):
                off = 3 * N + (st * N + iel) * per
                ur = u[off:off + nw]
                d = np.zeros(3 * nw)
                lib.fn['rng_normal'](PRIMES[first], off + nw, 3 * nw, oracle_lib.pd(d))
                w.eval_grad(iel)
                w.make_move(iel, d.reshape(nw, 3))
                r, _ = w.ratio_grad(iel)
                slr += np.log(np.abs(r))
                a = (ur < 0.5).astype(np.int32)
                acc += a
                w.accept_restore(iel, a)
                w.accept_reject(iel, a)
            w.complete_updates()
            _, _, lp = w.evaluate_gl()
            npt, ws, _ = w.nlpp(1.7, capi.NLPP_SPHERE)
            n_virtual += npt
            wsum += ws
        for i in range(nw):
            compare(got, i, acc, slr, lp, n_virtual, wsum, steps, N, nw, tol)


@needs_binaries
@pytest.mark.gpu
@pytest.mark.parametrize('j3', [False, True])
def test_reference_sync_move_driver(tmp_path, j3):
    check_sync_move_driver(tmp_path, DEVICE, j3=j3)


def check_reference_table(tmp_path, extra_env=None):
    """Without QMCGPU_SPO_FILL the device gets the SPO set's own table (the
    reference's fill, rank one per tile): the library reports the singular
    Slater matrices once and the driver finishes, as the reference's own
    run does."""
    report = str(tmp_path / 'report.jsonl')
    env = dict(os.environ, QMCGPU_ADAPTER_REPORT=report, OMP_NUM_THREADS='1', **(extra_env or {}))
    env.pop('QMCGPU_SPO_FILL', None)
    r = subprocess.run([MINIQMC, '-g', '1 1 1', '-m', '0.5', '-w', '1', '-n', '1', '-x', '0'], capture_output=True,
                       text=True, timeout=600, env=env, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    assert 'QMC_ERR_SINGULAR' in r.stderr and 'Diffusion throughput' in r.stdout
    with open(report) as f:
        rep = [json.loads(line) for line in f]
    assert len(rep) == 1 and rep[0]['status'] == 4 and rep[0]['ratio_grad'] == 384


@needs_binaries
@pytest.mark.gpu
def test_reference_table_is_singular_and_the_run_goes_on(tmp_path):
    check_reference_table(tmp_path)


def check_sposet(tmp_path, args, extra_env=None):
    """The reference's own SPO set (its builder, fill and tiles) against the
    SPOSet adapter on the device copy of its table (check_spo_gpu)."""
    env = dict(os.environ, OMP_NUM_THREADS='1', **(extra_env or {}))
    env.pop('QMCGPU_SPO_FILL', None)
    r = subprocess.run([CHECK_SPO, *args], capture_output=True, text=True, timeout=600, env=env, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert 'All checks passed for spo on the device' in r.stdout
    return r.stdout


@needs_binaries
@pytest.mark.gpu
@pytest.mark.parametrize('args,precision', [(['-g', '1 1 1', '-m', '0.5', '-a', '48'], 'fp64'),
                                            (['-g', '1 1 1', '-m', '0.5'], 'fp64'),
                                            (['-g', '2 1 1', '-m', '0.5', '-a', '96'], 'mixed')])
def test_reference_sposet_on_the_device(tmp_path, args, precision):
    print(check_sposet(tmp_path, args + ['-n', '24'], {'QMCGPU_PRECISION': precision}))
