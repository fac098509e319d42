"""CPU checks of the oracle's restatement of the reference's mixed-precision
arithmetic (qmc_oracle.hpp ARITH_*), the yardstick the mixed form's error is
compared with.  No GPU.

- arithmetic flags 0 are the FP64 oracle bit for bit;
- DelayedUpdate in FP32 (DelayedUpdate<float, double>, DelayedUpdate.h:28-231)
  keeps the sequence of delayed rank-1 updates of the reference's unit test
  (test_dirac_det.cpp) within FP32 rounding of the FP64 result;
- each FP32 piece (orbitals, determinant, log accumulation) perturbs a
  48-electron sweep at its own rounding level, with the accept sequence
  unchanged (it depends on the uniforms only)."""
import numpy as np
import pytest

from miniqmc_b200 import api, capi, precision
from tests import oracle_lib


@pytest.fixture(scope='module')
def lib():
    return oracle_lib.library()


def _system(lib, arith):
    spec = api.SystemSpec(lib, cell=capi.NIO_PRIM4, tiling=(1, 1, 1), grid=(12, 12, 12),
                          fill=capi.FILL_UNIFORM_F32, jastrow='synthetic')
    s = api.System(lib, spec, capi.PREC_FP64)
    lib.call('system_set_arith', s.h, arith)
    return spec, s


def _streams(W, N, S=1):
    rs = np.random.default_rng(5)
    return rs.uniform(size=(S, W, 1, N)), rs.normal(size=(S, W, 1, N, 3))


def test_arith_zero_is_fp64(lib):
    spec, s0 = _system(lib, 0)
    _, s1 = _system(lib, 0)
    seeds = np.array([3, 5], dtype=np.uint32)
    ur, de = _streams(2, spec.n_elec)
    out = []
    for s in (s0, s1):
        w = api.Walkers(s, 2, 4)
        w.init_random(seeds)
        w.evaluate_log()
        out.append(w.sweep(1, 1, 0.5, ur=ur, delta=de, trace=True))
    assert np.array_equal(out[0]['trace'], out[1]['trace'])


def test_arith_flags_rejected_out_of_range(lib):
    _, s = _system(lib, 0)
    with pytest.raises(api.QMCError):
        lib.call('system_set_arith', s.h, 8)


@pytest.mark.parametrize('arith,tol', [(oracle_lib.ARITH_SPO32, 1e-4), (oracle_lib.ARITH_DET32, 1e-3),
                                       (oracle_lib.ARITH_REFERENCE_MIXED, 1e-3)])
def test_fp32_pieces_perturb_at_rounding_level(lib, arith, tol):
    """48 electrons, 24 orbitals: small, well-conditioned Slater matrices, so
    each FP32 piece stays near its rounding (measured medians 1e-7 to 1e-6)
    while a wrong restatement gives O(1) differences."""
    spec, st = _system(lib, arith)
    _, sr = _system(lib, 0)
    seeds = np.array([3, 5], dtype=np.uint32)
    ur, de = _streams(2, spec.n_elec, 2)
    wt, wr = api.Walkers(st, 2, 4), api.Walkers(sr, 2, 4)
    for w in (wt, wr):
        w.init_random(seeds)
    res = precision.sweep_errors(wt, wr, ur, de, checkpoints=(1, 2))
    assert res['accept_sequence_identical']
    assert res['log_ratio_abs']['median'] < tol, res['log_ratio_abs']
    assert res['log_ratio_abs']['median'] > 0.0  # the FP32 piece is really in use
    assert res['logdet_drift_rel']['2']['ref_rel_max'] < 1e-10
