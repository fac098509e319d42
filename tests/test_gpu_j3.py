"""GPU parity of the three-body (electron-electron-ion) Jastrow: the CUDA
path against the reference's printed values (check_wfc-style J3 alone) and
against the FP64 oracle (full wavefunction, verbs, mixed precision), through
the C ABI.

Tolerances as in test_gpu_parity.py: FP64 1e-10 relative for log values and
ratios, 1e-9 for gradients and Laplacians; accept flags exact.  The
reference's values are dumped on its 32-atom cell with every ion in species
0 ("q", as its NiO input builds them) and with O and Ni apart ("g")."""
import json
import os

import numpy as np
import pytest

from miniqmc_b200 import api, capi
from tests import gpu_helpers as H
from tests import oracle_lib
from tests.test_gpu_parity import RTOL64, check_ratios, elem_rel, rel_err

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(oracle_lib.GOLDEN, 'reference_dump.json')))
VARIANTS = [('q', capi.NIO_QUIRK_UNIT_IONS | capi.NIO_QUIRK_ONE_GROUP), ('g', capi.NIO_QUIRK_UNIT_IONS)]
ALL_J3 = capi.WF_ALL | capi.WF_J3
# the reference's 32-atom NiO cell with its ions at their Cartesian positions
# (384 electrons, J3 cutoff 4.83 bohr: logJ3 ~ -20 per walker); the 4-atom
# cells' Wigner-Seitz radius leaves J3 nearly empty
REF = dict(cell=capi.NIO_REF32, quirks=0)


def ref_walker(quirks, precision=capi.PREC_FP64):
    sp = api.SystemSpec(H.product(), cell=capi.NIO_REF32, quirks=quirks, grid=(8, 8, 8), fill=capi.FILL_REFERENCE,
                        components=capi.WF_J3)
    w = api.Walkers(api.System(H.product(), sp, precision), 1, 1)
    w.init_random([GOLD['primes'][1]])
    return w


@pytest.mark.parametrize('tag,quirks', VARIANTS)
def test_j3_evaluate_log_golden(tag, quirks):
    """ThreeBodyJastrow::evaluateLog, G and L on the device vs the reference."""
    w = ref_walker(quirks)
    assert np.array_equal(w.positions()[0].ravel(), GOLD['j3%s_R0' % tag])
    lp = w.evaluate_log()
    assert abs(lp[0] - GOLD['j3%s_log' % tag]) < RTOL64 * abs(GOLD['j3%s_log' % tag])
    G, L, _ = w.evaluate_gl()
    assert rel_err(G[0].ravel(), GOLD['j3%s_G' % tag]) < 1e-9
    assert rel_err(L[0], GOLD['j3%s_L' % tag]) < 1e-9


@pytest.mark.parametrize('tag,quirks', VARIANTS)
def test_j3_sweep_golden(tag, quirks):
    """One substep of the move protocol with J3 alone in the fused sweep:
    ratios, gradients, the exact accept sequence, logJ3, G and L after."""
    w = ref_walker(quirks)
    w.evaluate_log()
    out = w.sweep(1, 1, 0.5, trace=True)
    t = out['trace'][0, 0, 0]
    assert list(t[:, 7].astype(int)) == GOLD['j3%s_sweep_accept' % tag]
    assert rel_err(t[:, 0], GOLD['j3%s_sweep_ratio' % tag]) < 1e-9
    assert rel_err(t[:, 1:4].ravel(), GOLD['j3%s_sweep_grad_new' % tag]) < 1e-8
    assert rel_err(t[:, 4:7].ravel(), GOLD['j3%s_sweep_grad_now' % tag]) < 1e-8
    lj3 = w.components()[0][6]
    assert abs(lj3 - GOLD['j3%s_sweep_log' % tag]) < 1e-9 * abs(GOLD['j3%s_sweep_log' % tag])
    G, L, _ = w.evaluate_gl()
    assert rel_err(G[0].ravel(), GOLD['j3%s_sweep_G' % tag]) < 1e-8
    assert rel_err(L[0], GOLD['j3%s_sweep_L' % tag]) < 1e-8


def test_j3_jastrow_sweep_exact():
    """J1 * J2 * J3 fused sweep vs the oracle (FP64): the three-body terms
    are sums of a few hundred products, so ratios, gradients and logJ3 agree
    to a few ULPs (measured p99 4e-15)."""
    W, steps = 2, 2
    seeds = H.oracle_primes(W)
    comp = capi.WF_J1 | capi.WF_J2 | capi.WF_J3
    gw, ow = H.make_pair(walkers=W, delay=1, seeds=seeds, components=comp, **REF)
    gw.evaluate_log()
    ow.evaluate_log()
    ur, de = H.host_streams(seeds, gw.N, steps, 1)
    rg = gw.sweep(steps, 1, 0.5, ur=ur, delta=de, trace=True)
    ro = ow.sweep(steps, 1, 0.5, ur=ur, delta=de, trace=True)
    assert np.array_equal(rg['trace'][..., 7], ro['trace'][..., 7])
    assert elem_rel(rg['trace'][..., 0], ro['trace'][..., 0]).max() < 1e-13
    assert rel_err(rg['trace'][..., 1:7], ro['trace'][..., 1:7]) < 1e-12
    assert elem_rel(gw.components()[:, 6], ow.components()[:, 6]).max() < 1e-12


@pytest.mark.parametrize('delay', [1, 4])
def test_j3_full_wavefunction_sweep(delay):
    """Det * J1 * J2 * J3 fused sweep vs the oracle on the same streams (FP64):
    accept flags exact; ratios within the determinant's bound on this cell
    (192 orbitals per spin: near-node moves amplify the inverse's rounding,
    measured p99 1.2e-9 with or without J3, so 2e-9); log values 1e-10; and
    the accumulated J3 state equals a fresh evaluation."""
    W, steps, nsub = 2, 2, 1
    seeds = H.oracle_primes(W)
    gw, ow = H.make_pair(walkers=W, delay=delay, seeds=seeds, components=ALL_J3, **REF)
    gw.evaluate_log()
    ow.evaluate_log()
    ur, de = H.host_streams(seeds, gw.N, steps, nsub)
    rg = gw.sweep(steps, nsub, 0.5, ur=ur, delta=de, trace=True)
    ro = ow.sweep(steps, nsub, 0.5, ur=ur, delta=de, trace=True)
    assert np.array_equal(rg['trace'][..., 7], ro['trace'][..., 7])
    assert np.array_equal(rg['accepted'], ro['accepted'])
    check_ratios(rg['trace'][..., 0], ro['trace'][..., 0], 2e-9)
    assert rel_err(rg['trace'][..., 1:7], ro['trace'][..., 1:7]) < 1e-7
    assert elem_rel(rg['logpsi'], ro['logpsi']).max() < RTOL64
    cg, co = gw.components(), ow.components()
    assert elem_rel(cg[:, 6], co[:, 6]).max() < RTOL64
    # list bookkeeping and Uat updates: a fresh evaluateLog rebuilds the
    # electron lists from the positions and gives the same logJ3
    Gg, Lg, _ = gw.evaluate_gl()
    gw.evaluate_log()
    assert elem_rel(gw.components()[:, 6], cg[:, 6]).max() < 1e-11
    G2, L2, _ = gw.evaluate_gl()
    assert rel_err(Gg, G2) < 1e-9 and rel_err(Lg, L2) < 1e-9


def test_j3_verbs():
    """The drop-in per-call API with J3: evalGrad, ratioGrad, ratio,
    acceptMove/restore (with and without a preceding ratioGrad)."""
    gw, ow = H.make_pair(walkers=2, delay=2, components=ALL_J3, **REF)
    gw.evaluate_log()
    ow.evaluate_log()
    rng = np.random.default_rng(21)
    for it, iel in enumerate([0, 1, 5, 191, 192, 300, 383, 2, 3, 4, 11, 40]):
        assert rel_err(gw.eval_grad(iel), ow.eval_grad(iel)) < 1e-9
        d = rng.normal(size=(2, 3)) * 0.6
        gw.make_move(iel, d)
        ow.make_move(iel, d)
        if it % 3 == 2:
            check_ratios(gw.ratio(iel), ow.ratio(iel), 2e-9)
        else:
            rg, gg = gw.ratio_grad(iel)
            ro, go = ow.ratio_grad(iel)
            check_ratios(rg, ro, 2e-9)
            assert rel_err(gg, go) < 1e-8
        acc = np.array([(it + w) % 2 for w in range(2)], dtype=np.int32)
        gw.accept_restore(iel, acc)
        ow.accept_restore(iel, acc)
        gw.accept_reject(iel, acc)
        ow.accept_reject(iel, acc)
    gw.complete_updates()
    ow.complete_updates()
    Gg, Lg, lg = gw.evaluate_gl()
    Go, Lo, lo = ow.evaluate_gl()
    assert rel_err(lg, lo) < RTOL64
    assert rel_err(Gg, Go) < 1e-8 and rel_err(Lg, Lo) < 1e-8
    assert rel_err(gw.components(), ow.components()) < RTOL64


def test_j3_mixed_precision():
    """Mixed form with J3 (FP32 triples and per-electron sums, FP64 block
    sums): accept flags exact on the same streams; log ratios of a J3-only
    wavefunction (|U| ~ 0.1 per electron, FP32 rounding ~1e-7 relative per
    triple) median 1e-6, max 1e-4; logJ3 1e-5 relative."""
    W = 2
    seeds = H.oracle_primes(W)
    gw, ow = H.make_pair(precision=capi.PREC_MIXED, walkers=W, seeds=seeds, components=capi.WF_J3, **REF)
    gw.evaluate_log()
    ow.evaluate_log()
    assert elem_rel(gw.components()[:, 6], ow.components()[:, 6]).max() < 1e-5
    ur, de = H.host_streams(seeds, gw.N, 1, 1)
    rg = gw.sweep(1, 1, 0.5, ur=ur, delta=de, trace=True)
    ro = ow.sweep(1, 1, 0.5, ur=ur, delta=de, trace=True)
    assert np.array_equal(rg['trace'][..., 7], ro['trace'][..., 7])
    lr = np.abs(np.log(np.abs(rg['trace'][..., 0])) - np.log(np.abs(ro['trace'][..., 0]))).ravel()
    assert np.median(lr) < 1e-6, np.median(lr)
    assert lr.max() < 1e-4, lr.max()
    assert elem_rel(gw.components()[:, 6], ow.components()[:, 6]).max() < 1e-5


def test_j3_nio128_cell():
    """The 4x4x2 NiO-128 cell (1536 electrons, 128 ions) with J3 alone, FP64:
    one substep against the oracle; the lists stay within their capacity."""
    seeds = H.oracle_primes(1)
    gw, ow = H.make_pair(walkers=1, seeds=seeds, components=capi.WF_J3, tiling=(4, 4, 2), grid=(6, 6, 6))
    lg, lo = gw.evaluate_log(), ow.evaluate_log()
    assert elem_rel(lg, lo).max() < RTOL64
    ur, de = H.host_streams(seeds, gw.N, 1, 1)
    rg = gw.sweep(1, 1, 0.5, ur=ur, delta=de, trace=True)
    ro = ow.sweep(1, 1, 0.5, ur=ur, delta=de, trace=True)
    assert np.array_equal(rg['trace'][..., 7], ro['trace'][..., 7])
    check_ratios(rg['trace'][..., 0], ro['trace'][..., 0], RTOL64)
    assert elem_rel(rg['logpsi'], ro['logpsi']).max() < RTOL64


def test_j3_checkpoint_roundtrip():
    """A batch with J3 restored from its checkpoint continues exactly as the
    original (the electron lists are part of the state)."""
    seeds = H.oracle_primes(2)
    gw, _ = H.make_pair(walkers=2, delay=2, seeds=seeds, components=ALL_J3, **REF)
    gw.evaluate_log()
    gw.sweep(1, 1, 0.5)
    blob = gw.checkpoint()
    a = gw.sweep(1, 1, 0.5, trace=True)
    gw.restore(blob)
    b = gw.sweep(1, 1, 0.5, trace=True)
    assert np.array_equal(a['trace'], b['trace'])
    assert np.array_equal(a['logpsi'], b['logpsi'])


@pytest.mark.parametrize('form', [capi.NLPP_SPHERE, capi.NLPP_DRIVER])
def test_j3_nlpp_fp64(form):
    """NonLocalPP ratios with J3 (ThreeBodyJastrow::evaluateRatios through
    computeU at each quadrature point) against the oracle: same points,
    ratios within the determinant's bound on this cell."""
    gw, ow = H.make_pair(walkers=2, delay=4, components=ALL_J3, **REF)
    gw.evaluate_log()
    ow.evaluate_log()
    ng, wg, rg = gw.nlpp(1.7, form, max_ratios=1 << 14)
    no, wo, ro = ow.nlpp(1.7, form, max_ratios=1 << 14)
    assert np.array_equal(ng, no) and ng[0] > 0
    m = int(ng[0])
    check_ratios(rg[:m], ro[:m], 2e-9)
    assert elem_rel(wg, wo).max() < 1e-9


def test_j3_nlpp_jastrow_only_exact():
    """J1 * J2 * J3 alone: the quadrature-point ratios agree to rounding."""
    gw, ow = H.make_pair(walkers=1, components=capi.WF_J1 | capi.WF_J2 | capi.WF_J3, **REF)
    gw.evaluate_log()
    ow.evaluate_log()
    ng, wg, rg = gw.nlpp(1.7, capi.NLPP_SPHERE, max_ratios=1 << 14)
    no, wo, ro = ow.nlpp(1.7, capi.NLPP_SPHERE, max_ratios=1 << 14)
    assert np.array_equal(ng, no)
    m = int(ng[0])
    assert elem_rel(rg[:m], ro[:m]).max() < 1e-12
    # the J3-only ratios are not trivially one
    assert np.abs(np.log(np.abs(ro[:m]))).max() > 1e-2


def test_j3_nlpp_mixed():
    gw, ow = H.make_pair(precision=capi.PREC_MIXED, walkers=1, delay=4, components=ALL_J3, **REF)
    gw.evaluate_log()
    ow.evaluate_log()
    ng, wg, rg = gw.nlpp(1.7, capi.NLPP_SPHERE, max_ratios=1 << 14)
    no, wo, ro = ow.nlpp(1.7, capi.NLPP_SPHERE, max_ratios=1 << 14)
    assert np.array_equal(ng, no)
    m = int(ng[0])
    e = elem_rel(rg[:m], ro[:m])
    assert np.median(e) < 1e-4 and np.percentile(e, 99) < 1e-2, (np.median(e), np.percentile(e, 99))


def test_j3_capacity_is_reported():
    """A three-body cutoff of 30 bohr on the NiO-128 cell puts every electron
    inside every ion's cutoff: more than the 128 a list holds, and more than
    64 ions around a point.  evaluateLog reports QMC_ERR_CAPACITY; the lists
    and the near-ion buffers are written only within their bounds."""
    lib = H.product()
    spec = api.SystemSpec(lib, cell=capi.NIO_PRIM4, tiling=(4, 4, 2), grid=(6, 6, 6), components=capi.WF_J3,
                          jastrow='synthetic')
    big = lib.j3_functor(30.0, np.zeros(capi.J3_PARAMS))
    for g in range(spec.ions['n_groups']):
        spec.desc.j3_same[g] = big
        spec.desc.j3_diff[g] = big
    w = api.Walkers(api.System(lib, spec), 1, 1)
    w.init_random(H.oracle_primes(1))
    with pytest.raises(api.QMCError) as ei:
        w.evaluate_log()
    assert capi.STATUS[ei.value.status] == 'QMC_ERR_CAPACITY'
