"""GPU parity: the CUDA path (libqmcgpu.so) against the CPU FP64 oracle and
the reference's golden values, through the C ABI.

Tolerances: FP64 plain form 1e-10 relative (the bound the plain form
promises against the reference); mixed form per quantity, stated in each
test.  Integer bookkeeping (accept flags and counts) is compared exactly.
"""
import json
import os

import numpy as np
import pytest

from miniqmc_b200 import api, capi
from tests import gpu_helpers as H
from tests import oracle_lib

pytestmark = pytest.mark.gpu
RTOL64 = 1e-10
GOLD = json.load(open(os.path.join(oracle_lib.GOLDEN, 'reference_dump.json')))
KA = json.load(open(os.path.join(oracle_lib.GOLDEN, 'known_answers.json')))


def rel_err(a, b):
    """Norm-wise relative error max|a-b| / max|b| (vectors, matrices)."""
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def elem_rel(a, b):
    """Element-wise relative errors (scalars per walker or per move)."""
    a = np.asarray(a, dtype=float).ravel()
    b = np.asarray(b, dtype=float).ravel()
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def check_ratios(rg, ro, tol):
    """Per-move ratios: 99% of moves within tol, every move within 100 tol.
    A move near a node of the determinant has a ratio much smaller than the
    terms of its dot product, so its rounding error is amplified by that
    cancellation in any arithmetic (the reference's included)."""
    e = elem_rel(rg, ro)
    assert np.percentile(e, 99) < tol, np.percentile(e, 99)
    assert e.max() < 100 * tol, e.max()


# ------------------------------------------------------------ det engine --
def test_det_engine_known_answers():
    """test_dirac_matrix.cpp / test_dirac_det.cpp known answers on the device."""
    lib = H.product()
    eps = 100 * np.finfo(np.float32).eps
    e = api.DetEngine(lib, 3, 1)
    lg, _ = e.invert_transpose(np.array(KA['dm_a']).T)
    np.testing.assert_allclose(lg, KA['dm_logdet'], rtol=eps)
    np.testing.assert_allclose(e.ainv(), KA['dm_a_inv'], rtol=eps, atol=1e-9)
    ratio = np.array(KA['dm_update_v']) @ e.get_inv_row(0)
    np.testing.assert_allclose(ratio, KA['dm_update_ratio'], rtol=eps)
    e.accept_row(0, np.array(KA['dm_update_v']))
    np.testing.assert_allclose(e.ainv(), KA['dm_update_inv'], rtol=eps, atol=1e-9)


@pytest.mark.parametrize('delay', [1, 2, 3])
def test_det_engine_matches_oracle(delay):
    """Sequential row replacements with delay k (rank-1 SM and Woodbury)."""
    rng = np.random.default_rng(5)
    n = 37
    a = rng.standard_normal((n, n)) + 3 * np.eye(n)
    g = api.DetEngine(H.product(), n, delay)
    o = api.DetEngine(H.oracle(), n, delay)
    lg, pg = g.invert_transpose(a)
    lo, po = o.invert_transpose(a)
    assert abs(lg - lo) < 1e-11 * max(1, abs(lo)) and pg == po
    for row in (3, 17, 0, 36, 5, 9, 22):
        v = rng.standard_normal(n)
        v[row] += 3.0  # keep the updated matrix as well conditioned as the original
        rg, ro = g.get_inv_row(row), o.get_inv_row(row)
        assert rel_err(rg, ro) < RTOL64
        g.accept_row(row, v)
        o.accept_row(row, v)
    g.update_inv_mat()
    o.update_inv_mat()
    assert rel_err(g.ainv(), o.ainv()) < RTOL64


# ------------------------------------------------------------------- SPO --
@pytest.mark.parametrize('prec', [capi.PREC_FP64, capi.PREC_MIXED])
@pytest.mark.parametrize('fill', [capi.FILL_REFERENCE, capi.FILL_UNIFORM])
def test_spo_vgh(prec, fill):
    sp, so = H.spec_pair(grid=(13, 11, 9), fill=fill, components=capi.WF_J1, n_orb=40)
    g = api.System(H.product(), sp, prec)
    o = api.System(H.oracle(), so, prec)
    rng = np.random.default_rng(2)
    pos = rng.uniform(-10, 20, (33, 3))
    pos[0] = [0.0, 0.0, 0.0]
    pos[1] = [-1e-18, 3.0, 2.0]
    vg, gg, hg = g.spo_vgh(pos)
    vo, go, ho = o.spo_vgh(pos)
    # FP32 evaluation of the FP32-rounded table vs its FP64 evaluation
    tol = RTOL64 if prec == capi.PREC_FP64 else 1e-5
    assert rel_err(vg, vo) < tol
    assert rel_err(gg, go) < tol
    assert rel_err(hg, ho) < tol
    assert rel_err(g.spo_v(pos), vo) < tol


def test_spo_reference_golden():
    """check_spo: the reference's own einspline values at fixed points."""
    nx, ny, nz = GOLD['spo_grid']
    sp = api.SystemSpec(H.product(), cell=capi.NIO_REF32, quirks=3, grid=(nx, ny, nz), fill=capi.FILL_REFERENCE,
                        components=capi.WF_J1, n_orb=GOLD['spo_norb'])
    s = api.System(H.product(), sp, capi.PREC_FP64)
    v, g, h = s.spo_vgh(np.array(GOLD['spo_pos']).reshape(-1, 3))
    assert rel_err(v.ravel(), GOLD['spo_v']) < RTOL64
    assert rel_err(g.ravel(), GOLD['spo_g']) < RTOL64
    assert rel_err(h.ravel(), GOLD['spo_h']) < RTOL64


# -------------------------------------------------------------- Jastrows --
@pytest.mark.parametrize('comp,key', [(capi.WF_J1, 'j1'), (capi.WF_J2, 'j2')])
def test_jastrow_check_wfc_values(comp, key):
    """check_wfc -f J1 / J2: the reference's log, G and L on the device."""
    sp = api.SystemSpec(H.product(), cell=capi.NIO_REF32, quirks=3, grid=(8, 8, 8), fill=capi.FILL_REFERENCE,
                        components=comp)
    w = api.Walkers(api.System(H.product(), sp, capi.PREC_FP64), 1, 1)
    w.init_random([3])
    assert np.array_equal(w.positions()[0].ravel(), GOLD['els_111_p0'])  # bit-exact build_els
    lp = w.evaluate_log()
    assert abs(lp[0] - GOLD[key + '_log']) < RTOL64 * abs(GOLD[key + '_log'])
    G, L, _ = w.evaluate_gl()
    assert rel_err(G[0].ravel(), GOLD[key + '_G']) < 1e-9
    assert rel_err(L[0], GOLD[key + '_L']) < 1e-9


def test_jastrow_sweep_golden():
    """One substep of the reference move protocol with J1*J2 (threshold accept)."""
    sp = api.SystemSpec(H.product(), cell=capi.NIO_REF32, quirks=3, grid=(8, 8, 8), fill=capi.FILL_REFERENCE,
                        components=capi.WF_J1 | capi.WF_J2)
    w = api.Walkers(api.System(H.product(), sp, capi.PREC_FP64), 1, 1)
    w.init_random([3])
    w.evaluate_log()
    out = w.sweep(1, 1, 0.5, trace=True)
    t = out['trace'][0, 0, 0]
    assert list(t[:, 7].astype(int)) == GOLD['jsweep_accept']
    assert rel_err(t[:, 0], GOLD['jsweep_ratio']) < 1e-9
    assert rel_err(t[:, 1:4].ravel(), GOLD['jsweep_grad_new']) < 1e-8
    assert np.max(np.abs(w.positions()[0].ravel() - GOLD['jsweep_R'])) < 1e-12


# ------------------------------------------------------ full wavefunction --
def test_reference_fill_is_singular():
    """The reference's SPO fill makes every orbital the same field times
    cos(2 pi n / N), so its Slater matrices have rank 1; the reference
    prints -inf / NaN and passes.  Here the zero pivot is reported."""
    gw, _ = H.make_pair(walkers=1, fill=capi.FILL_REFERENCE, grid=(14, 14, 14))
    with pytest.raises(api.QMCError) as ei:
        gw.evaluate_log()
    assert ei.value.status == 4  # QMC_ERR_SINGULAR


def test_evaluate_log():
    gw, ow = H.make_pair(walkers=3, fill=capi.FILL_UNIFORM, grid=(14, 14, 14))
    lg = gw.evaluate_log()
    lo = ow.evaluate_log()
    assert elem_rel(lg, lo).max() < RTOL64
    assert rel_err(gw.components(), ow.components()) < RTOL64
    Gg, Lg, _ = gw.evaluate_gl()
    Go, Lo, _ = ow.evaluate_gl()
    assert rel_err(Gg, Go) < 1e-9
    assert rel_err(Lg, Lo) < 1e-9
    for s in (0, 1):
        assert rel_err(gw.inverse(1, s), ow.inverse(1, s)) < RTOL64


@pytest.mark.parametrize('delay', [1, 3])
def test_verbs(delay):
    """The drop-in per-call API: evalGrad, makeMove, ratioGrad, ratio,
    acceptMove/restore, accept/rejectMove, completeUpdates, evaluateGL."""
    gw, ow = H.make_pair(walkers=2, delay=delay)
    gw.evaluate_log()
    ow.evaluate_log()
    rng = np.random.default_rng(9)
    N = gw.N
    for it, iel in enumerate([0, 1, 5, 23, 24, 30, 47, 2, 3, 4]):
        assert rel_err(gw.eval_grad(iel), ow.eval_grad(iel)) < 1e-9
        d = rng.normal(size=(2, 3)) * 0.4
        gw.make_move(iel, d)
        ow.make_move(iel, d)
        if it % 3 == 2:
            rg, ro = gw.ratio(iel), ow.ratio(iel)
            check_ratios(rg, ro, RTOL64)
        else:
            rg, gg = gw.ratio_grad(iel)
            ro, go = ow.ratio_grad(iel)
            check_ratios(rg, ro, RTOL64)
            assert rel_err(gg, go) < 1e-9
        acc = np.array([(it + w) % 2 for w in range(2)], dtype=np.int32)
        gw.accept_restore(iel, acc)
        ow.accept_restore(iel, acc)
        gw.accept_reject(iel, acc)
        ow.accept_reject(iel, acc)
    gw.complete_updates()
    ow.complete_updates()
    assert np.array_equal(gw.positions(), ow.positions())
    Gg, Lg, lg = gw.evaluate_gl()
    Go, Lo, lo = ow.evaluate_gl()
    assert rel_err(lg, lo) < RTOL64
    assert rel_err(Gg, Go) < 1e-8
    assert rel_err(gw.components(), ow.components()) < RTOL64


def test_spo_evaluate_batch_device_buffers():
    """qmc_spo_evaluate_batch: the batch's SPO at activeR(iat) into device
    buffers, against the oracle's SPO at the same points (FP64): the proposed
    positions after makeMove, then the current ones once the move is
    rejected (values only)."""
    import torch
    W, iat = 3, 7
    gw, ow = H.make_pair(walkers=W, delay=2)
    gw.evaluate_log()
    d = np.random.default_rng(4).normal(size=(W, 3)) * 0.5
    gw.make_move(iat, d)
    pos = gw.positions()[:, iat] + d
    n = gw.sys.spec.n_orb
    v = torch.zeros((W, n), dtype=torch.float64, device='cuda')
    g = torch.zeros((W, 3, n), dtype=torch.float64, device='cuda')
    h = torch.zeros((W, 6, n), dtype=torch.float64, device='cuda')
    lib = H.product()
    lib.call('spo_evaluate_batch', gw.h, iat, v.data_ptr(), g.data_ptr(), h.data_ptr())
    lib.call('walkers_sync', gw.h)
    vo, go, ho = ow.sys.spo_vgh(pos)
    assert rel_err(v.cpu().numpy(), vo) < RTOL64
    assert rel_err(g.cpu().numpy(), go) < RTOL64
    assert rel_err(h.cpu().numpy(), ho) < RTOL64
    gw.accept_reject(iat, np.zeros(W, dtype=np.int32))
    v.zero_()
    lib.call('spo_evaluate_batch', gw.h, iat, v.data_ptr(), None, None)
    lib.call('walkers_sync', gw.h)
    assert rel_err(v.cpu().numpy(), ow.sys.spo_v(gw.positions()[:, iat])) < RTOL64


@pytest.mark.parametrize('prec,tol', [(capi.PREC_FP64, 1e-10), (capi.PREC_MIXED, 1e-4)])
def test_step_entry_point_matches_sweep(prec, tol):
    """qmc_step, one fused single-electron move of the batch per call, over
    every electron of a substep followed by completeUpdates and evaluateGL
    gives the fused sweep's walkers on the same streams: the same accept
    flags, log values within the form's bound (the sweep flushes the up
    determinant at the spin boundary, the steps at completeUpdates)."""
    W = 2
    seeds = H.oracle_primes(W)
    g1, _ = H.make_pair(precision=prec, walkers=W, delay=4, seeds=seeds)
    g2, _ = H.make_pair(precision=prec, walkers=W, delay=4, seeds=seeds)
    if prec == capi.PREC_MIXED:
        H.product().call('walkers_set_tensor_cores', g1.h, 0)
    g1.evaluate_log()
    g2.evaluate_log()
    ur, de = H.host_streams(seeds, g1.N, 1, 1)
    r1 = g1.sweep(1, 1, 0.5, ur=ur, delta=de, trace=True)
    flags = np.zeros((W, g2.N), dtype=np.int32)
    for iel in range(g2.N):
        flags[:, iel] = g2.step(iel, 0.5, ur[0, :, 0, iel], de[0, :, 0, iel])
    g2.complete_updates()
    _, _, lp2 = g2.evaluate_gl()
    assert np.array_equal(flags, r1['trace'][0, :, 0, :, 7].astype(np.int32))
    assert elem_rel(lp2, r1['logpsi']).max() < tol
    assert np.max(np.abs(g1.positions() - g2.positions())) == 0.0


@pytest.mark.parametrize('last', ['ratio', 'ratio_grad'])
def test_evaluate_gl_after_ratio_only_move(last):
    """DiracDeterminant::evaluateGL re-evaluates the orbital derivative rows
    of a determinant whose last move was ratio-only (the accept of such a
    move leaves its dpsiM / d2psiM row stale); after a ratioGrad move it
    does not, and the stale row stays.  Both outcomes match the oracle."""
    gw, ow = H.make_pair(walkers=1, delay=2)
    gw.evaluate_log()
    ow.evaluate_log()
    acc = np.ones(1, dtype=np.int32)
    d = np.array([[0.3, -0.2, 0.4]])
    for iel, kind in ((3, 'ratio'), (7, last)):
        gw.make_move(iel, d)
        ow.make_move(iel, d)
        if kind == 'ratio':
            check_ratios(gw.ratio(iel), ow.ratio(iel), RTOL64)
        else:
            gw.ratio_grad(iel)
            ow.ratio_grad(iel)
        gw.accept_restore(iel, acc)
        ow.accept_restore(iel, acc)
        gw.accept_reject(iel, acc)
        ow.accept_reject(iel, acc)
    gw.complete_updates()
    ow.complete_updates()
    Gg, Lg, _ = gw.evaluate_gl()
    Go, Lo, _ = ow.evaluate_gl()
    assert rel_err(Gg, Go) < 1e-9 and rel_err(Lg, Lo) < 1e-9


@pytest.mark.parametrize('delay', [1, 4])
def test_sweep_host_rng_fp64(delay):
    """Fused sweep vs oracle on identical random streams: bit-exact accept
    sequence and counts, 1e-10 ratios and log values."""
    W, steps, nsub = 2, 2, 2
    seeds = H.oracle_primes(W)
    gw, ow = H.make_pair(walkers=W, delay=delay, seeds=seeds)
    gw.evaluate_log()
    ow.evaluate_log()
    ur, de = H.host_streams(seeds, gw.N, steps, nsub)
    rg = gw.sweep(steps, nsub, 0.5, ur=ur, delta=de, trace=True)
    ro = ow.sweep(steps, nsub, 0.5, ur=ur, delta=de, trace=True)
    assert np.array_equal(rg['trace'][..., 7], ro['trace'][..., 7])
    assert np.array_equal(rg['accepted'], ro['accepted'])
    # the threshold rule also accepts moves near a node (small |ratio|); each
    # such Sherman-Morrison/Woodbury update amplifies the rounding already in
    # the inverse by ~1/|ratio|, in the oracle as on the GPU, so per-move
    # ratios after several delayed updates agree to ~1e-10 (p99 1e-9)
    check_ratios(rg['trace'][..., 0], ro['trace'][..., 0], 1e-9 if delay > 1 else RTOL64)
    assert rel_err(rg['trace'][..., 1:7], ro['trace'][..., 1:7]) < (1e-7 if delay > 1 else 1e-8)
    assert elem_rel(rg['logpsi'], ro['logpsi']).max() < RTOL64
    assert rel_err(gw.components(), ow.components()) < RTOL64
    assert np.max(np.abs(gw.positions() - ow.positions())) < 1e-12


def test_sweep_device_rng():
    """Device mt19937 streams: the same uniforms as libstdc++ (accept flags
    bit-exact); normals from CUDA's log/cos/sin may differ by ULPs."""
    W = 3
    gw, ow = H.make_pair(walkers=W, delay=2)
    gw.evaluate_log()
    ow.evaluate_log()
    rg = gw.sweep(2, 1, 0.5, trace=True)
    ro = ow.sweep(2, 1, 0.5, trace=True)
    assert np.array_equal(rg['trace'][..., 7], ro['trace'][..., 7])
    assert np.array_equal(rg['accepted'], ro['accepted'])
    assert rel_err(rg['logpsi'], ro['logpsi']) < 1e-9
    assert np.max(np.abs(gw.positions() - ow.positions())) < 1e-10


def test_sweep_mixed_precision():
    """Mixed form (FP32 tables, inverse, Jastrows; FP64 log-det and Binv)
    against the FP64 oracle on the same FP32-rounded spline table and the
    same streams.  Accept flags exact.  Measured on this case: log-ratio
    median 3.5e-6, p99 5.7e-4 (the tail is near-node moves the threshold
    rule accepts, whose updates amplify the FP32 rounding of the stored
    inverse by ~1/|ratio|), log|psi| 1.2e-6 relative; the bounds are about
    twice those."""
    W = 2
    seeds = H.oracle_primes(W)
    gw, ow = H.make_pair(precision=capi.PREC_MIXED, walkers=W, delay=4, seeds=seeds)
    gw.evaluate_log()
    ow.evaluate_log()
    ur, de = H.host_streams(seeds, gw.N, 1, 2)
    rg = gw.sweep(1, 2, 0.5, ur=ur, delta=de, trace=True)
    ro = ow.sweep(1, 2, 0.5, ur=ur, delta=de, trace=True)
    assert np.array_equal(rg['trace'][..., 7], ro['trace'][..., 7])
    lr = np.abs(np.log(np.abs(rg['trace'][..., 0])) - np.log(np.abs(ro['trace'][..., 0]))).ravel()
    print('mixed 48e: log-ratio median %.3e p99 %.3e logpsi %.3e' % (
        np.median(lr), np.percentile(lr, 99), elem_rel(rg['logpsi'], ro['logpsi']).max()))
    assert np.median(lr) < 7e-6, np.median(lr)
    assert np.percentile(lr, 99) < 1.2e-3, np.percentile(lr, 99)
    assert elem_rel(rg['logpsi'], ro['logpsi']).max() < 2.5e-6


def test_recompute_matches_fresh_evaluation():
    gw, ow = H.make_pair(walkers=2, delay=3)
    gw.evaluate_log()
    gw.sweep(2, 1, 0.5, recompute_every=1)
    c1 = gw.components()
    gw.evaluate_log()
    c2 = gw.components()
    # the FP64 refresh after the last step equals a fresh evaluateLog
    assert rel_err(c1[:, :4], c2[:, :4]) < 1e-11
