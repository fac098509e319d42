"""The miniqmc command-line driver (miniqmc_b200/drivers/miniqmc.cpp): the
reference driver's options and exit codes (src/Drivers/miniqmc.cpp:149-290),
and on the GPU the same walkers as the Python API for the same system,
seeds (PrimeNumberSet) and settings."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from miniqmc_b200 import api, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, 'miniqmc_b200', 'bin', 'miniqmc')


@pytest.fixture(scope='module')
def exe():
    from miniqmc_b200 import build
    build.build()
    return EXE


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
