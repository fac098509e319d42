"""Batch groups (several systems in one fused launch, optionally replayed
from a CUDA graph), the autotuner and the request loop.  None of these has a
reference counterpart: the checks are that each batch or job gives the same
result as it does alone, and that admission follows the memory budget."""
import ctypes as C

import numpy as np
import pytest

from miniqmc_b200 import api, capi
from tests import gpu_helpers as H

pytestmark = pytest.mark.gpu


def _system(tiling, precision=capi.PREC_MIXED):
    lib = H.product()
    spec = api.SystemSpec(lib, cell=capi.NIO_PRIM4, tiling=tiling, grid=tuple(12 * t for t in tiling),
                          fill=capi.FILL_UNIFORM, spo_seed=11, jastrow='synthetic')
    return api.System(lib, spec, precision)


def _batch(system, W, delay, seed0):
    w = api.Walkers(system, W, delay)
    w.init_random((np.arange(W, dtype=np.uint32) * 7919 + seed0).astype(np.uint32))
    w.evaluate_log()
    return w


def _results(w):
    acc = np.zeros(w.W, dtype=np.int64)
    lp = np.zeros(w.W)
    w.lib.call('sweep_results', w.h, acc.ctypes.data_as(C.POINTER(C.c_int64)), lp.ctypes.data_as(capi.PD))
    return acc, lp, w.positions()


@pytest.mark.parametrize('precision', [capi.PREC_MIXED, capi.PREC_FP64])
def test_group_equals_batches_alone(precision):
    """Two systems (48 and 96 electrons) in one launch per step, with the
    periodic FP64 refresh, give bit-identical walkers to each batch alone."""
    sa, sb = _system((1, 1, 1), precision), _system((2, 1, 1), precision)
    alone = []
    for sys_, W, k, seed in ((sa, 6, 4, 11), (sb, 5, 8, 101)):
        w = _batch(sys_, W, k, seed)
        w.lib.call('sweep_async', w.h, 3, 1, 0.5, 2)
        alone.append(_results(w))
    wa, wb = _batch(sa, 6, 4, 11), _batch(sb, 5, 8, 101)
    g = api.Group(H.product(), [wa, wb])
    g.sweep(3, 1, 0.5, recompute_every=2)
    g.sync()
    for w, ref in zip((wa, wb), alone):
        got = _results(w)
        assert np.array_equal(got[0], ref[0])
        assert np.array_equal(got[1], ref[1])
        assert np.array_equal(got[2], ref[2])
    assert g.stats()['launches'] == 3


def test_group_graph_replay_equals_eager():
    sa, sb = _system((1, 1, 1)), _system((2, 1, 1))
    out = []
    for graph in (False, True):
        ws = [_batch(sa, 4, 4, 7), _batch(sb, 3, 8, 9)]
        g = api.Group(H.product(), ws)
        g.use_graph(graph)
        g.sweep(4, 1, 0.5)
        g.sync()
        out.append([_results(w) for w in ws])
        st = g.stats()
        assert st['graph_launches'] == (3 if graph else 0)  # the first step runs eagerly
        g.close()
    for a, b in zip(out[0], out[1]):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


@pytest.mark.parametrize('graph', [False, True])
def test_group_queue_equals_static(graph):
    """Three systems (48, 96 and 192 electrons) in one launch per step, with
    the periodic FP64 refresh: the work-queue form on 3 CTAs in units of 5
    moves (walkers of every system handed between the CTAs, each CTA loading
    the system of the walker it takes) gives the static form's walkers bit
    for bit, eagerly and replayed from a graph."""
    systems = [_system(t) for t in ((1, 1, 1), (2, 1, 1), (2, 2, 1))]
    out = []
    for mode, unit, ctas in ((capi.SCHED_STATIC, 0, 0), (capi.SCHED_QUEUE, 5, 3)):
        ws = [_batch(s, W, k, seed) for s, W, k, seed in zip(systems, (4, 3, 2), (4, 8, 8), (5, 17, 29))]
        g = api.Group(H.product(), ws)
        g.set_schedule(mode, unit, ctas)
        g.use_graph(graph)
        g.sweep(3, 1, 0.5, recompute_every=2)
        g.sync()
        out.append([_results(w) for w in ws])
        g.close()
    for a, b in zip(out[0], out[1]):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    assert any(r[0].sum() > 0 for r in out[1])


def test_group_schedule_rejects_bad_settings():
    ws = [_batch(_system((1, 1, 1)), 2, 4, 3)]
    g = api.Group(H.product(), ws)
    for bad in ((3, 0, 0), (-1, 0, 0), (capi.SCHED_QUEUE, -1, 0), (capi.SCHED_QUEUE, 0, -1)):
        with pytest.raises(api.QMCError) as e:
            g.set_schedule(*bad)
        assert e.value.status == 1  # QMC_ERR_ARG
    g.set_schedule(capi.SCHED_STATIC)
    g.sweep(1, 1, 0.5)
    g.sync()
    g.close()


def test_autotune_returns_a_measured_candidate():
    s = _system((2, 1, 1))
    best, allr = api.autotune(H.product(), s, 16, delays=(4, 8), n_steps=1)
    assert len(allr) >= 2 and best in allr
    assert best['ms_per_step'] == min(r['ms_per_step'] for r in allr)
    assert best['delay'] in (4, 8) and best['threads'] % 32 == 0


def _run_server(server, jobs):
    ids = [server.submit(*j) for j in jobs]
    max_waiting = 0
    for _ in range(10000):
        running, waiting = server.tick()
        max_waiting = max(max_waiting, waiting)
        if running == 0 and waiting == 0:
            break
    infos = [server.job(i) for i in ids]
    assert all(i['state'] == capi.JOB_DONE for i in infos), infos
    return infos, max_waiting


def test_server_results_alone_equal_in_the_mix():
    lib = H.product()
    sa, sb = _system((1, 1, 1)), _system((2, 1, 1))
    jobs = [(sa, 8, 5, 4, 3), (sb, 4, 3, 8, 5), (sa, 3, 7, 4, 9)]
    srv = api.Server(lib, 8 << 30, threads=128, recompute_every=4)
    mix, _ = _run_server(srv, jobs)
    for job, m in zip(jobs, mix):
        alone, _ = _run_server(api.Server(lib, 8 << 30, threads=128, recompute_every=4), [job])
        assert alone[0]['n_accepted'] == m['n_accepted']
        assert alone[0]['logpsi_mean'] == m['logpsi_mean']
        assert m['steps_done'] == job[2]
        assert m['t_done'] >= m['t_start'] >= m['t_submit']


def test_server_admission_follows_the_budget():
    lib = H.product()
    s = _system((2, 1, 1))
    w = _batch(s, 8, 8, 1)
    size = C.c_size_t()
    lib.call('walkers_bytes', w.h, C.byref(size))
    w.close()
    srv = api.Server(lib, int(size.value * 1.5), threads=128)
    infos, max_waiting = _run_server(srv, [(s, 8, 2, 8, 1), (s, 8, 2, 8, 2), (s, 8, 2, 8, 3)])
    assert max_waiting >= 1  # one job's state at a time fits
    starts = sorted(i['t_start'] for i in infos)
    dones = sorted(i['t_done'] for i in infos)
    assert starts[1] >= dones[0] and starts[2] >= dones[1]
    with pytest.raises(api.QMCError) as ei:
        srv.submit(s, 64, 2, 8, 4)
    assert capi.STATUS[ei.value.status] == 'QMC_ERR_ADMISSION'


def test_handles_are_reentrant_across_host_threads():
    """One host thread per batch (each on its own stream): two batches of
    different systems swept concurrently give the walkers each gives alone
    (the thread-local error state and the per-handle streams keep the calls
    independent; ctypes releases the GIL around them)."""
    import threading
    seeds = [H.oracle_primes(3), H.oracle_primes(5)[2:]]
    kw = [dict(tiling=(1, 1, 1)), dict(tiling=(1, 1, 2))]

    def run(i, out):
        gw, _ = H.make_pair(walkers=3, delay=4, seeds=seeds[i], **kw[i])
        gw.evaluate_log()
        ur, de = H.host_streams(seeds[i], gw.N, 2, 1)
        r = gw.sweep(2, 1, 0.5, ur=ur, delta=de)
        out[i] = (r['logpsi'].copy(), r['accepted'].copy(), gw.positions().copy())

    alone = {}
    for i in range(2):
        run(i, alone)
    together = {}
    threads = [threading.Thread(target=run, args=(i, together)) for i in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for i in range(2):
        for a, b in zip(alone[i], together[i]):
            assert np.array_equal(a, b)


def test_server_failed_job_leaves_the_others_unchanged():
    """A job whose Slater matrices are singular (the reference's own rank-1
    orbital fill, einspline_spo.hpp:145-155, on an FP64 table) fails inside
    the request loop: its evaluateLog raises the zero-pivot bit in the job's
    own status word, the job keeps its slot in the shared launches until it
    retires, and it is reported QMC_JOB_FAILED with QMC_ERR_SINGULAR.  The
    jobs admitted before and after it finish with exactly the results they
    give alone (the reference has no counterpart: it aborts the process,
    Configuration.h:35-39)."""
    lib = H.product()
    sa, sb = _system((1, 1, 1), capi.PREC_FP64), _system((2, 1, 1), capi.PREC_FP64)
    bad_spec = api.SystemSpec(lib, cell=capi.NIO_PRIM4, tiling=(1, 1, 1), grid=(12, 12, 12),
                              fill=capi.FILL_REFERENCE, spo_seed=11, jastrow='synthetic')
    bad = api.System(lib, bad_spec, capi.PREC_FP64)
    jobs = [(sa, 8, 5, 4, 3), (bad, 4, 4, 4, 7), (sb, 4, 3, 8, 5)]
    srv = api.Server(lib, 8 << 30, threads=128, recompute_every=2)
    ids = [srv.submit(*j) for j in jobs]
    for _ in range(10000):
        running, waiting = srv.tick()
        if running == 0 and waiting == 0:
            break
    infos = [srv.job(i) for i in ids]
    assert infos[1]['state'] == capi.JOB_FAILED
    assert capi.STATUS[infos[1]['status']] == 'QMC_ERR_SINGULAR'
    for k in (0, 2):
        assert infos[k]['state'] == capi.JOB_DONE, infos[k]
        alone, _ = _run_server(api.Server(lib, 8 << 30, threads=128, recompute_every=2), [jobs[k]])
        assert alone[0]['n_accepted'] == infos[k]['n_accepted']
        assert alone[0]['logpsi_mean'] == infos[k]['logpsi_mean']
