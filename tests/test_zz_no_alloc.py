"""qmc_invert_transpose_noalloc (no reference counterpart): the FP64 inverse
on caller-owned device buffers with the library's static scratch, checked
bit for bit against qmc_detengine_invert_transpose, the entry point it is a
variant of.  The file name sorts last so the test also runs after every other
GPU test has used the library on the same device."""
import ctypes as C

import numpy as np
import pytest

from miniqmc_b200 import api, capi
from tests.gpu_helpers import product

pytestmark = pytest.mark.gpu


def _noalloc(lib, a):
    import torch
    n = a.shape[0]
    a_dev = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    psim_dev = torch.full_like(a_dev, float('nan'))
    lg, ph = C.c_double(), C.c_double()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib.call('invert_transpose_noalloc', n, C.c_void_p(a_dev.data_ptr()), C.c_void_p(psim_dev.data_ptr()),
             C.byref(lg), C.byref(ph), stream)
    return psim_dev.cpu().numpy(), lg.value, ph.value


def _engine(lib, a):
    e = api.DetEngine(lib, a.shape[0], 1)
    try:
        lg, ph = e.invert_transpose(a)
        return e.ainv(), lg, ph
    finally:
        e.close()


def _matrix(rng, n):
    return rng.standard_normal((n, n)) + 0.5 * np.eye(n)


def test_noalloc_inverse_equals_engine_on_consecutive_calls():
    lib = product()
    rng = np.random.default_rng(20261203)
    # two calls in a row on the same scratch: a ragged size, then the maximum
    for n in (100, capi.NOALLOC_MAX_N):
        a = _matrix(rng, n)
        psim, lg, ph = _noalloc(lib, a)
        ref_psim, ref_lg, ref_ph = _engine(lib, a)
        assert np.array_equal(psim, ref_psim), n
        assert lg == ref_lg and ph == ref_ph, n
        # and it is the inverse transpose
        assert np.abs(psim.T @ a - np.eye(n)).max() < 1e-9
        sign, la = np.linalg.slogdet(a)
        assert abs(lg - la) < 1e-9 * n and ph == (0.0 if sign > 0 else np.pi)


def test_noalloc_rejects_sizes_beyond_the_scratch():
    lib = product()
    for n in (0, capi.NOALLOC_MAX_N + 1):
        with pytest.raises(api.QMCError) as ei:
            lib.call('invert_transpose_noalloc', n, C.c_void_p(0), C.c_void_p(0), None, None, None)
        assert capi.STATUS[ei.value.status] == 'QMC_ERR_ARG'


def test_noalloc_singular_then_regular():
    """The error bits in the scratch are cleared by every call: a singular
    matrix reports QMC_ERR_SINGULAR, the next regular one succeeds."""
    lib = product()
    rng = np.random.default_rng(7)
    a = _matrix(rng, 64)
    s = a.copy()
    s[5] = 0.0  # stays exactly zero through the elimination: a zero pivot
    with pytest.raises(api.QMCError) as ei:
        _noalloc(lib, s)
    assert capi.STATUS[ei.value.status] == 'QMC_ERR_SINGULAR'
    psim, lg, ph = _noalloc(lib, a)
    ref_psim, ref_lg, ref_ph = _engine(lib, a)
    assert np.array_equal(psim, ref_psim) and lg == ref_lg and ph == ref_ph


@pytest.mark.parametrize('n', [64, 900])
def test_nan_entries_are_singular_then_regular(n):
    """A NaN in the matrix competes as 0 in every pivot search, so the
    pivots stay rows of the matrix and the inverse reports a zero pivot:
    QMC_ERR_SINGULAR from the engine (and from the allocation-free entry
    point within its size), after which a regular matrix inverts as before.
    n = 900 takes the column-at-a-time kernel (the blocked one's panel no
    longer fits in shared memory)."""
    lib = product()
    rng = np.random.default_rng(11)
    a = _matrix(rng, n)
    for bad in ('entry', 'column'):
        s = a.copy()
        if bad == 'entry':
            s[3, 7] = np.nan
        else:
            s[:, 5] = np.nan
        calls = [_engine] + ([_noalloc] if n <= capi.NOALLOC_MAX_N else [])
        for f in calls:
            with pytest.raises(api.QMCError) as ei:
                f(lib, s)
            assert capi.STATUS[ei.value.status] == 'QMC_ERR_SINGULAR', (bad, f.__name__)
    psim, lg, _ = _engine(lib, a)
    assert np.abs(psim.T @ a - np.eye(n)).max() < 1e-8
    assert abs(lg - np.linalg.slogdet(a)[1]) < 1e-9 * n
