"""qmc_wf_evaluate_ratios (WaveFunction::evaluateRatios over a
VirtualParticleSet, NonLocalPP.hpp:115-134): one walker's ratios of one
electron at absolute positions, against the oracle on the same walkers and
against the product's own move verbs (makeMove, ratio, rejectMove) at the
same positions; the batch's state is untouched, and pending delayed rows are
refused."""
import numpy as np
import pytest

from miniqmc_b200 import api, capi
from tests import gpu_helpers as H
from tests.test_gpu_parity import elem_rel

pytestmark = pytest.mark.gpu


def _walkers(precision, components):
    seeds = H.oracle_primes(3)
    gw, ow = H.make_pair(precision=precision, walkers=3, delay=4, seeds=seeds, tiling=(1, 1, 2), grid=(12, 12, 12),
                         components=components)
    gw.evaluate_log()
    ow.evaluate_log()
    ur, de = H.host_streams(seeds, gw.N, 1, 1)
    gw.sweep(1, 1, 0.5, ur=ur, delta=de)
    ow.sweep(1, 1, 0.5, ur=ur, delta=de)
    return gw, ow


def _points(R, iat, n, seed):
    """n positions around electron iat: a 12-point sphere of radius 0.9
    about a point near it, then random offsets (ragged last group)."""
    rs = np.random.default_rng(seed)
    c = R[iat] + rs.normal(scale=0.3, size=3)
    v = rs.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    p = c + 0.9 * v
    p[12:] = R[iat] + rs.normal(scale=0.7, size=(n - 12, 3))
    return p


@pytest.mark.parametrize('precision', [capi.PREC_FP64, capi.PREC_MIXED])
@pytest.mark.parametrize('j3', [False, True])
def test_evaluate_ratios_matches_oracle_and_verbs(precision, j3):
    comp = capi.WF_ALL | (capi.WF_J3 if j3 else 0)
    gw, ow = _walkers(precision, comp)
    R = gw.positions()
    lp0 = gw.evaluate_gl()[2].copy()
    for walker, iat in ((1, 5), (2, gw.N - 1), (0, gw.N // 2)):
        pts = _points(R[walker], iat, 29, 100 * walker + iat)
        rg = gw.evaluate_ratios(walker, iat, pts)
        ro = ow.evaluate_ratios(walker, iat, pts)
        e = elem_rel(rg, ro)
        tol = 1e-10 if precision == capi.PREC_FP64 else 2e-3
        assert e.max() < tol, (walker, iat, e.max())
        # the same ratios through the move verbs (every walker moves; this
        # walker's displacement puts its electron on the point)
        if precision == capi.PREC_FP64:
            for k in (0, 13, 28):
                d = np.zeros((gw.W, 3))
                d[walker] = pts[k] - R[walker, iat]
                gw.make_move(iat, d)
                q = gw.ratio(iat)[walker]
                gw.accept_reject(iat, np.zeros(gw.W, dtype=np.int32))
                assert abs(q - rg[k]) <= 1e-12 * abs(q) + 1e-300, (k, q, rg[k])
    # the batch state is unchanged: positions, and the log values of a
    # fresh evaluateGL
    assert np.array_equal(gw.positions(), R)
    np.testing.assert_allclose(gw.evaluate_gl()[2], lp0, rtol=1e-12)


def test_evaluate_ratios_refuses_pending_rows():
    seeds = H.oracle_primes(2)
    gw, _ = H.make_pair(walkers=2, delay=4, seeds=seeds, tiling=(1, 1, 1), grid=(12, 12, 12))
    gw.evaluate_log()
    R = gw.positions()
    iat = 3
    gw.eval_grad(iat)
    gw.make_move(iat, np.full((2, 3), 0.1))
    gw.ratio_grad(iat)
    gw.accept_restore(iat, np.ones(2, dtype=np.int32))
    gw.accept_reject(iat, np.ones(2, dtype=np.int32))
    with pytest.raises(api.QMCError) as e:
        gw.evaluate_ratios(0, 7, R[0, 7][None, :] + 0.2)
    assert e.value.status == 7  # QMC_ERR_STATE
    gw.complete_updates()
    assert np.all(np.isfinite(gw.evaluate_ratios(0, 7, R[0, 7][None, :] + 0.2)))
    with pytest.raises(api.QMCError):
        gw.evaluate_ratios(2, 7, R[0, 7][None, :])
