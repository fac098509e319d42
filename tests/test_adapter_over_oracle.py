"""The adapter classes (miniqmc_b200/adapter/) on a machine without a GPU:
the reference's drivers linked with the adapter run over the CPU oracle (a
libqmcgpu.so stand-in that forwards the adapter's qmc_* calls to the
oracle's, tests/adapter_oracle_shim.cpp), and each walker's counters and log
value must equal the oracle's own run of the same driver loop bit for bit
in everything but the order of summation.  This checks the adapter's
translation of every WaveFunction verb -- per-walker and flex_, the exact
move displacements, the batches, the NLPP ratios -- with the same checks as
the GPU tests (tests/test_gpu_reference_drivers.py)."""
import os
import subprocess

import pytest

from tests import oracle_lib
from tests import test_gpu_reference_drivers as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope='module')
def shim_env(tmp_path_factory):
    d = tmp_path_factory.mktemp('shim')
    oracle_lib.library()  # builds oracle/liboracle.so
    oracle_dir = os.path.join(ROOT, 'oracle')
    subprocess.check_call(['g++', '-O1', '-shared', '-fPIC', '-I' + os.path.join(ROOT, 'include'), '-o',
                           str(d / 'libqmcgpu.so'), os.path.join(ROOT, 'tests', 'adapter_oracle_shim.cpp'),
                           '-L' + oracle_dir, '-loracle', '-Wl,-rpath,' + oracle_dir])
    return {'LD_LIBRARY_PATH': str(d) + os.pathsep + os.environ.get('LD_LIBRARY_PATH', '')}


@R.needs_binaries
@pytest.mark.parametrize('j3', [False, True])
def test_miniqmc_driver_over_oracle(tmp_path, shim_env, j3):
    R.check_miniqmc_driver(tmp_path, j3, R.EXACT, shim_env)


@R.needs_binaries
@pytest.mark.parametrize('j3', [False, True])
def test_sync_move_driver_over_oracle(tmp_path, shim_env, j3):
    R.check_sync_move_driver(tmp_path, R.EXACT, shim_env, j3=j3)


@R.needs_binaries
def test_reference_table_over_oracle(tmp_path, shim_env):
    R.check_reference_table(tmp_path, shim_env)


@R.needs_binaries
def test_driver_without_a_device_stops(tmp_path):
    """With the real library and no GPU the first device call fails loudly
    (exit code 1, QMC_ERR_NODEVICE); nothing falls back to the host."""
    from miniqmc_b200 import api
    try:
        lib = api.Library()
        has_gpu = lib.fn['init'](0) == 0
    except OSError:
        pytest.skip('the product library is not built')
    if has_gpu:
        pytest.skip('a GPU is present')
    r = subprocess.run([R.MINIQMC, '-g', '1 1 1', '-m', '0.5', '-w', '1', '-n', '1'], capture_output=True, text=True,
                       timeout=300, cwd=str(tmp_path), env=dict(os.environ, OMP_NUM_THREADS='1'))
    assert r.returncode == 1 and 'QMC_ERR_NODEVICE' in r.stderr


@R.needs_binaries
def test_reference_sposet_over_oracle(tmp_path, shim_env):
    R.check_sposet(tmp_path, ['-g', '1 1 1', '-m', '0.5', '-a', '48', '-n', '8'], shim_env)
