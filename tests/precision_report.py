"""Per-quantity error of the mixed-precision form (and of the FP64 form)
against the FP64 oracle at the NiO-128 size: SPO values / gradients /
Hessians, log-ratios and gradients of one MC step of all 1536 electrons, and
the post-sweep drift of the log-determinant accumulated through the ratios
from a fresh FP64 evaluation at the final positions.

    python tests/precision_report.py [--grid 24,24,12] [--delay 32] > report.json

Needs a GPU.  The oracle is the checker: both sides see the same
FP32-rounded spline table and the same random streams."""
import argparse
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from miniqmc_b200 import api, capi  # noqa: E402
from tests import gpu_helpers as H  # noqa: E402


def stats(e):
    e = np.asarray(e, dtype=float).ravel()
    return {'median': float(np.median(e)), 'p99': float(np.percentile(e, 99)), 'max': float(e.max())}


def normwise(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def spo_errors(gs, os_, rng):
    pos = rng.uniform(size=(256, 3)) @ np.array(gs.spec.desc.lattice[:]).reshape(3, 3)
    vg, gg, hg = gs.spo_vgh(pos)
    vo, go, ho = os_.spo_vgh(pos)
    return {'v_normwise': normwise(vg, vo), 'g_normwise': normwise(gg, go), 'h_normwise': normwise(hg, ho)}


def step_errors(gw, ow, seeds):
    gw.evaluate_log()
    ow.evaluate_log()
    ur, de = H.host_streams(seeds, gw.N, 1, 1)
    rg = gw.sweep(1, 1, 0.5, ur=ur, delta=de, trace=True)
    ro = ow.sweep(1, 1, 0.5, ur=ur, delta=de, trace=True)
    tg, to = rg['trace'].reshape(-1, 8), ro['trace'].reshape(-1, 8)
    lr = np.abs(np.log(np.abs(tg[:, 0])) - np.log(np.abs(to[:, 0])))
    gerr = np.linalg.norm(tg[:, 1:4] - to[:, 1:4], axis=1) / np.maximum(np.linalg.norm(to[:, 1:4], axis=1), 1e-300)
    same_accepts = bool(np.array_equal(tg[:, 7], to[:, 7]))
    # log|det| accumulated through the step's ratios vs a fresh FP64 evaluation
    cg = gw.components()[0]
    ow.evaluate_log()
    co = ow.components()[0]
    drift = [abs(cg[s] - co[s]) / abs(co[s]) for s in (0, 1)]
    return {'log_ratio_abs': stats(lr), 'grad_rel': stats(gerr), 'accept_sequence_identical': same_accepts,
            'logdet_drift_rel': drift, 'logpsi_rel': float(abs(rg['logpsi'][0] - ro['logpsi'][0]) /
                                                             abs(ro['logpsi'][0]))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--grid', default='24,24,12')
    ap.add_argument('--delay', type=int, default=32)
    args = ap.parse_args()
    grid = tuple(int(x) for x in args.grid.split(','))
    seeds = H.oracle_primes(1)
    rng = np.random.default_rng(17)
    out = {'system': 'NiO 4x4x2 of the 4-atom cell (1536 e-, 768 orbitals/spin)', 'grid': grid,
           'delay': args.delay, 'walkers': 1, 'moves': 1536}
    for name, prec, tc in (('mixed_tensor_core_flush', capi.PREC_MIXED, 1), ('mixed_cuda_core_flush', capi.PREC_MIXED, 0),
                           ('fp64', capi.PREC_FP64, None)):
        gw, ow = H.make_pair(precision=prec, walkers=1, delay=args.delay, tiling=(4, 4, 2), grid=grid,
                             jastrow='synthetic', seeds=seeds)
        if tc is not None:
            H.product().call('walkers_set_tensor_cores', gw.h, tc)
        res = {'spo': spo_errors(gw.sys, ow.sys, rng)}
        res.update(step_errors(gw, ow, seeds))
        out[name] = res
        print(name, json.dumps(res), file=sys.stderr, flush=True)
    print(json.dumps(out), flush=True)


if __name__ == '__main__':
    main()
