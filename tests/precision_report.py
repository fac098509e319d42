"""Per-quantity error of the mixed-precision form against FP64 at the NiO-128
size, and the attribution of that error.

Measured, on the same FP32-rounded spline table, positions and random
streams: SPO values / gradients / Hessians, the log-ratio and gradient of
every move (with per-step statistics), and the drift of the log-determinant
accumulated through the ratios from a fresh FP64 evaluation at the same
positions, after the first MC step and after the last (no refresh between).

    python tests/precision_report.py [--grid 148,148,74] [--delays 16,32,64]
        [--walkers 4] [--steps 8] [--oracle-variants spo32,det32,ref_mixed]
        [--oracle-steps 2] > report.json

Product forms ('tc': mixed with the tensor-core flush, 'simt': mixed with the
CUDA-core flush) are measured against the product's FP64 form on the mixed
form's table (QMC_FILL_UNIFORM_F32: the same coefficients rounded to FP32,
evaluated in FP64; the FP64 parity tests pin it to the oracle at 1e-10).

Oracle variants restate pieces of the reference's own mixed-precision build
in the CPU oracle (qmc_oracle.hpp ARITH_*) and are measured against the FP64
oracle on the same table: 'spo32' FP32 orbital evaluation with an FP64
determinant; 'det32' FP64 orbitals with the FP32 determinant algebra
(DelayedUpdate<float, double>: FP32 inverse, delayed rows, Binv, GEMVs and
GEMMs; FP64 LU); 'ref_mixed' both plus the FP32 log|det| accumulation, i.e.
the reference's mixed build of this path (DelayedUpdate.h:28-50,
DiracMatrix.h:93-119, DiracDeterminant.cpp:129-146).  Needs a GPU."""
import argparse
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from miniqmc_b200 import api, capi, precision  # noqa: E402
from tests import gpu_helpers as H  # noqa: E402
from tests import oracle_lib  # noqa: E402

ORACLE_ARITH = {'spo32': oracle_lib.ARITH_SPO32, 'det32': oracle_lib.ARITH_DET32,
                'ref_mixed': oracle_lib.ARITH_REFERENCE_MIXED}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--grid', default='148,148,74')
    ap.add_argument('--tiling', default='4,4,2')
    ap.add_argument('--delays', default='16,32,64')
    ap.add_argument('--walkers', type=int, default=4)
    ap.add_argument('--steps', type=int, default=8)
    ap.add_argument('--forms', default='tc,simt')
    ap.add_argument('--oracle-variants', default='spo32,det32,ref_mixed')
    ap.add_argument('--oracle-steps', type=int, default=2)
    ap.add_argument('--oracle-delay', type=int, default=32)
    args = ap.parse_args()
    grid = tuple(int(x) for x in args.grid.split(','))
    tiling = tuple(int(x) for x in args.tiling.split(','))
    W, S = args.walkers, args.steps
    lib = H.product()
    seeds = (np.arange(W, dtype=np.uint32) * 7919 + 1009).astype(np.uint32)
    kw = dict(cell=capi.NIO_PRIM4, tiling=tiling, grid=grid, spo_seed=11, jastrow='synthetic')
    sm_spec = api.SystemSpec(lib, fill=capi.FILL_UNIFORM, **kw)
    sm = api.System(lib, sm_spec, capi.PREC_MIXED)
    sr = api.System(lib, api.SystemSpec(lib, fill=capi.FILL_UNIFORM_F32, **kw), capi.PREC_FP64)
    N = sm_spec.n_elec
    rs = np.random.default_rng(23)
    ur = rs.uniform(size=(S, W, 1, N))
    de = rs.normal(size=(S, W, 1, N, 3))
    pts = rs.uniform(size=(256, 3)) @ np.array(sm_spec.ions['spo_lattice']).reshape(3, 3)
    out = {'system': 'NiO %s of the 4-atom cell (%d e-, %d orbitals/spin)' % (args.tiling, N, sm_spec.n_orb),
           'grid': grid, 'walkers': W, 'steps': S, 'moves_per_step': N,
           'spo_mixed_vs_fp64': precision.spo_errors(sm, sr, pts), 'product': {}, 'oracle': {}}
    forms = [f for f in args.forms.split(',') if f]
    for k in (int(x) for x in args.delays.split(',')):
        for form in forms:
            wt = api.Walkers(sm, W, k)
            if form == 'simt':
                lib.call('walkers_set_tensor_cores', wt.h, 0)
            else:
                try:
                    lib.call('walkers_set_tensor_cores', wt.h, 1)
                except api.QMCError:
                    wt.close()
                    continue  # the tensor-core flush takes k <= 32
            wr = api.Walkers(sr, W, k)
            for w in (wt, wr):
                w.init_random(seeds)
            res = precision.sweep_errors(wt, wr, ur, de, checkpoints=(1, S))
            name = '%s_k%d' % (form, k)
            out['product'][name] = res
            print(name, json.dumps(res), file=sys.stderr, flush=True)
            wt.close()
            wr.close()
    sm.close()
    sr.close()
    variants = [v for v in args.oracle_variants.split(',') if v]
    if variants:
        olib = H.oracle()
        so = api.System(olib, api.SystemSpec(olib, fill=capi.FILL_UNIFORM_F32, **kw), capi.PREC_FP64)
        So = args.oracle_steps
        for v in variants:
            olib.call('system_set_arith', so.h, ORACLE_ARITH[v])
            wt = api.Walkers(so, W, args.oracle_delay)
            olib.call('system_set_arith', so.h, 0)
            wr = api.Walkers(so, W, args.oracle_delay)
            for w in (wt, wr):
                w.init_random(seeds)
            res = precision.sweep_errors(wt, wr, ur[:So], de[:So], checkpoints=(1, So))
            name = '%s_k%d' % (v, args.oracle_delay)
            out['oracle'][name] = res
            print('oracle', name, json.dumps(res), file=sys.stderr, flush=True)
            wt.close()
            wr.close()
    print(json.dumps(out), flush=True)


if __name__ == '__main__':
    main()
