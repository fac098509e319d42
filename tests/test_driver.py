"""The command-line drivers (miniqmc_b200/drivers/): miniqmc, the batched
per-verb miniqmc_sync_move, check_wfc and check_spo.  Their options and exit
codes follow the reference's drivers (src/Drivers/*.cpp); on the GPU,
miniqmc gives the same walkers as the Python API, miniqmc_sync_move the same
accepted count and log values as the oracle driven through the same verbs
and random streams, and the checkers pass."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from miniqmc_b200 import api, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, 'miniqmc_b200', 'bin')
EXE = os.path.join(BIN, 'miniqmc')
DRIVERS = ['miniqmc', 'miniqmc_sync_move', 'check_wfc', 'check_spo']


@pytest.fixture(scope='module')
def exe():
    from miniqmc_b200 import build
    build.build()
    return EXE


@pytest.mark.parametrize('name', DRIVERS)
def test_every_driver_prints_help(exe, name):
    r = run(os.path.join(BIN, name), '-h')
    assert r.returncode == 1 and 'usage:' in r.stdout


def test_check_wfc_rejects_unknown_component(exe):
    r = run(os.path.join(BIN, 'check_wfc'), '-f', 'J5')
    assert r.returncode == 1 and 'Uknown wave funciton component' in r.stderr


def run(exe, *args):
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=600)


def test_help_and_version_exit_1(exe):
    r = run(exe, '-h')
    assert r.returncode == 1 and 'usage:' in r.stdout and '-k  matrix delayed update rank' in r.stdout
    assert run(exe, '-V').returncode == 1


@pytest.mark.parametrize('opt', ['-b'])
def test_unavailable_options_stop_with_a_message(exe, opt):
    r = run(exe, opt)
    assert r.returncode == 1 and r.stderr.strip()


def test_bad_arguments(exe):
    assert run(exe, '-t', 'medium').returncode == 1
    assert run(exe, 'stray').returncode == 1
    assert run(exe, '-g', '1 1').returncode == 1


@pytest.mark.gpu
@pytest.mark.parametrize('j3', [False, True])
def test_driver_matches_the_api(exe, j3):
    r = run(exe, '-g', '1 1 1', '-m', '0.5', '-w', '6', '-n', '2', '-k', '8', '-v', *(['-j'] if j3 else []))
    assert r.returncode == 0, r.stdout + r.stderr
    assert 'Diffusion throughput' in r.stdout and 'Number of electrons = 384' in r.stdout
    accepted = int(re.search(r'Accepted moves = (\d+)', r.stdout).group(1))
    # the same run through the Python mirror of the C ABI
    lib = api.Library()
    lib.call('init', 0)
    spec = api.SystemSpec(lib, cell=capi.NIO_REF32, tiling=(1, 1, 1), grid=(18, 18, 18), fill=capi.FILL_UNIFORM,
                          spo_seed=11, jastrow='reference',
                          components=capi.WF_ALL | (capi.WF_J3 if j3 else 0))
    system = api.System(lib, spec, capi.PREC_MIXED)
    w = api.Walkers(system, 6, 8)
    primes = [3, 5, 7, 11, 13, 17]  # PrimeNumberSet<uint32_t> from 3
    w.init_random(np.array(primes, dtype=np.uint32))
    w.evaluate_log()
    out = w.sweep(2, 1, 0.5, recompute_every=8)
    assert int(np.sum(out['accepted'])) == accepted
    lp = float(re.search(r'mean log\|psi\| = (\S+)', r.stdout).group(1))
    assert abs(lp - float(np.mean(out['logpsi']))) <= 1e-12 * abs(lp)


@pytest.mark.gpu
@pytest.mark.parametrize('comp', ['J1', 'J2', 'J3', 'Det'])
def test_check_wfc_passes(exe, comp):
    """Each component in the mixed form against the FP64 form on the device."""
    r = run(os.path.join(BIN, 'check_wfc'), '-f', comp)
    assert r.returncode == 0, r.stdout + r.stderr
    assert 'All checks passed for %s' % comp in r.stdout, r.stdout


@pytest.mark.gpu
def test_check_wfc_fp64_is_exact(exe):
    r = run(os.path.join(BIN, 'check_wfc'), '-f', 'J2', '-p', 'fp64')
    assert r.returncode == 0 and 'All checks passed for J2' in r.stdout, r.stdout
    assert 'evaluateLog::V Error = 0' in r.stdout


@pytest.mark.gpu
def test_check_spo_passes(exe):
    r = run(os.path.join(BIN, 'check_spo'), '-m', '0.5', '-n', '2')
    assert r.returncode == 0, r.stdout + r.stderr
    assert 'All checks passed for spo' in r.stdout, r.stdout


@pytest.mark.gpu
def test_sync_move_driver_matches_oracle(exe):
    """miniqmc_sync_move (FP64, 2 batches of 2 movers, no NLPP) against the
    oracle driven through the same verbs with the batches' random streams
    (the first mover's mt19937 after its 3N build_els draws: per electron
    nw uniforms, then 3 nw BoxMuller2 normals)."""
    from tests import oracle_lib
    r = run(os.path.join(BIN, 'miniqmc_sync_move'), '-g', '1 1 1', '-m', '0.25', '-w', '4', '-c', '2', '-n', '1',
            '-p', 'fp64', '-k', '4', '-P', '-v')
    assert r.returncode == 0, r.stdout + r.stderr
    accepted = int(re.search(r'Accepted moves = (\d+)', r.stdout).group(1))
    lp = float(re.search(r'mean log\|psi\| = (\S+)', r.stdout).group(1))
    lib = oracle_lib.library()
    spec = api.SystemSpec(lib, cell=capi.NIO_REF32, tiling=(1, 1, 1), grid=(9, 9, 9), fill=capi.FILL_UNIFORM,
                          spo_seed=11, jastrow='reference')
    system = api.System(lib, spec, capi.PREC_FP64)
    N = spec.n_elec
    primes = [3, 5, 7, 11]
    acc_total, lp_sum = 0, 0.0
    for first in (0, 2):
        nw = 2
        w = api.Walkers(system, nw, 4)
        w.init_random(np.array(primes[first:first + nw], dtype=np.uint32))
        w.evaluate_log()
        per = nw + 2 * ((3 * nw + 1) // 2)
        u = np.zeros(3 * N + N * per)
        lib.fn['rng_uniform'](primes[first], len(u), oracle_lib.pd(u))
        for iel in range(N):
            off = 3 * N + iel * per
            ur = u[off:off + nw]
            de = np.zeros(3 * nw)
            lib.fn['rng_normal'](primes[first], off + nw, 3 * nw, oracle_lib.pd(de))
            w.eval_grad(iel)
            w.make_move(iel, de.reshape(nw, 3))
            w.ratio_grad(iel)
            acc = (ur < 0.5).astype(np.int32)
            acc_total += int(acc.sum())
            w.accept_restore(iel, acc)
            w.accept_reject(iel, acc)
        w.complete_updates()
        _, _, lps = w.evaluate_gl()
        lp_sum += float(np.sum(lps))
    assert accepted == acc_total
    assert abs(lp - lp_sum / 4) <= 1e-9 * abs(lp)
