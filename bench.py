"""Benchmark: electron-moves/s of the VMC PbyP sweep on NiO-128.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): NiO tiled 4x4x2 from the 4-atom cell -- 128 atoms,
1536 electrons, 768 orbitals per spin -- B-spline grid 148x148x74 with FP32
coefficients (5.4 GB), 512 walkers, delay rank 32, mixed precision.  One
"step" is one MC step of miniqmc's driver loop over the whole batch: 1536
single-electron moves per walker (evalGrad, makeMove, ratioGrad, threshold
accept, delayed Woodbury flushes on the tensor cores, completeUpdates)
then evaluateGL; after every 8th step the inverses are rebuilt in FP64
(SPO matrix + blocked Gauss-Jordan), as the configuration asks.  Inputs
are synthetic (uniform spline coefficients from SplitMix64 seed 11,
synthetic Jastrows, electrons from each walker's mt19937 stream).

value: device-timed (CUDA events on the launching stream, max over ranks)
whole-job moves/s with walker state resident in HBM.  e2e: the same metric
through the public C ABI (qmc_sweep) with the random streams supplied from
pinned host memory each step and the accept counts and log values read
back, wall-clock timed.  Multi-GPU: walkers are independent, so each rank
runs its own replica batch (weak scaling, no collective on the data path).
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

MEASURED_PEAKS = os.path.join(REPO, 'MEASURED_PEAKS.json')


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=8)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--tiling', default='4,4,2')
    ap.add_argument('--grid', default='148,148,74')
    ap.add_argument('--walkers', type=int, default=512)
    ap.add_argument('--delay', type=int, default=32)
    ap.add_argument('--precision', default='mixed', choices=['mixed', 'fp64'])
    ap.add_argument('--recompute-every', type=int, default=8,
                    help='FP64 refresh of the inverses every this many MC steps (0 = never)')
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-cpu', action='store_true')
    ap.add_argument('--cpu-walkers', type=int, default=0)
    ap.add_argument('--port-baseline', action='store_true',
                    help='also time the FP64 oracle port on the host cores (beside the reference miniqmc)')
    ap.add_argument('--workload', default='nio128', choices=['nio128', 'uneven', 'serve', 'nlpp'],
                    help='nio128: the headline batch; uneven: three NiO systems in one autotuned, graph-replayed '
                         'launch; serve: Poisson-arrival request loop; nlpp: the NonLocalPP ratios')
    ap.add_argument('--nlpp-grid', default='148,148,148', help='nlpp: orbital grid of the NiO 2,2,1 cell')
    ap.add_argument('--jobs', type=int, default=2000, help='serve: number of jobs (the configuration: 2000)')
    ap.add_argument('--rate', type=float, default=20.0, help='serve: arrivals per second')
    ap.add_argument('--budget-gb', type=float, default=100.0, help='serve: device memory budget of the server')
    ap.add_argument('--no-tune', action='store_true', help='uneven: skip the autotuner (default launch settings)')
    ap.add_argument('--schedule', default='auto', choices=['auto', 'static', 'queue'],
                    help='the sweep CTAs\' schedule (qmc_walkers_set_schedule)')
    ap.add_argument('--unit', type=int, default=0, help='moves per unit of the work-queue schedule (0: default)')
    ap.add_argument('--threads', type=int, default=0, help='threads per walker (0: the library default)')
    ap.add_argument('--max-moves', type=int, default=1,
                    help='moves the sweep evaluates together (qmc_walkers_set_move_batching)')
    ap.add_argument('--flush', default='tc', choices=['tc', 'simt'],
                    help='Woodbury flush on the tensor cores (tcgen05 3xTF32) or the CUDA cores (FP32 FMA)')
    ap.add_argument('--plain-steps', type=int, default=4,
                    help='walker-steps of the plain FP64 form (1 walker per launch, rank-1) to time; 0 = skip')
    ap.add_argument('--fp64-steps', type=int, default=2,
                    help='MC steps of the batched FP64 form at the same walker count to time; 0 = skip')
    ap.add_argument('--refresh1-steps', type=int, default=2,
                    help='MC steps timed with the FP64 refresh after every step (0 = skip)')
    ap.add_argument('--error-walkers', type=int, default=4,
                    help='walkers of the mixed-form error measurement; 0 = skip')
    ap.add_argument('--error-steps', type=int, default=8,
                    help='MC steps of the mixed-form error measurement (the refresh interval)')
    return ap.parse_args()


def algorithmic_bytes_per_move(n, N, I, k, s, a):
    """Algorithmic HBM bytes of one electron move (evalGrad + ratioGrad +
    accept bookkeeping + amortised Woodbury flush), with n orbitals per spin,
    N electrons, I ions, delay k, element size s and acceptance a:
      64n (SPO stencil) + (k/2+1)n (Ainv row and U/V rows of getInvRow)
      + 3n (dpsiM row) + 3N + 3I (positions for the AA and AB rows)
      + a(14N + 6n) (J2 arrays read+write, U/V and dpsiM/d2psiM row writes)
      + a(2n^2/k + 2n) (Ainv read+write per flush, amortised)."""
    return s * (64 * n + (k / 2 + 1) * n + 3 * n + 3 * N + 3 * I + a * (14 * N + 6 * n) +
                a * (2 * n * n / k + 2 * n))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.device), '--query-gpu=' + self.Q,
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(',')])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace('.', '').isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = set()
        for r in self.rows:
            if len(r) > 8:
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == 'active':
                        reasons.add(nm)
        return {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': max(mx) if mx else None,
                'reasons': sorted(reasons), 'samples': len(sm)}


def peaks():
    try:
        return json.load(open(MEASURED_PEAKS)), 'measured'
    except Exception:
        return {'hbm_gbs': 6650.0, 'bf16_tflops': 1590.0}, 'fallback'


def build_workload(lib, args, capi, api, device_rng_seeds):
    tiling = tuple(int(x) for x in args.tiling.split(','))
    grid = tuple(int(x) for x in args.grid.split(','))
    spec = api.SystemSpec(lib, cell=capi.NIO_PRIM4, tiling=tiling, grid=grid, fill=capi.FILL_UNIFORM, spo_seed=11,
                          jastrow='synthetic')
    prec = capi.PREC_MIXED if args.precision == 'mixed' else capi.PREC_FP64
    system = api.System(lib, spec, prec)
    walkers = api.Walkers(system, args.walkers, args.delay)
    walkers.init_random(device_rng_seeds)
    return spec, system, walkers


# DRAM bytes per electron move of sweep_queue_kernel<float> measured by ncu
# at the default workload (dram__bytes_read.sum + dram__bytes_write.sum =
# 360.58 + 77.51 GB over one launch of 512 walkers x 1536 moves, NiO 4x4x2,
# grid 148x148x74, k=32, mixed, tensor-core flush; 64 walkers on a 74x74x37
# grid measured 24.81 + 5.23 GB, the L2 then holding more of each walker);
# the bench's traffic figure scales it by the moves of one launch
MEASURED_TRAFFIC_PER_MOVE = (360.58e9 + 77.51e9) / (512 * 1536)


def schedule_of(lib, walkers, args):
    """The sweep form qmc_walkers_set_schedule selects for this batch (AUTO:
    the work queue), its kernel and a line for the config."""
    import torch
    from miniqmc_b200 import capi
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    queue = args.schedule in ('queue', 'auto')
    per_sm = C.c_int()
    lib.call('walkers_occupancy', walkers.h, C.byref(per_sm))
    if not queue:
        return {'kernel': 'sweep_kernel', 'text': 'static: one CTA per walker, %d per SM' % per_sm.value}
    ctas = per_sm.value * sms
    unit = args.unit or capi.SCHED_UNIT_DEFAULT
    return {'kernel': 'sweep_queue_kernel',
            'text': 'work queue: %d CTAs (%d per SM) take units of %d moves' % (ctas, per_sm.value, unit)}


def plain_fp64_form(lib, args, api, capi, stream_cls):
    """The plain GPU form of the same system: FP64 table and walker state,
    one walker per launch, delay rank 1 (Sherman-Morrison), walkers run one
    after another.  Returns (electron-moves/s, ms per walker-step)."""
    import torch
    tiling = tuple(int(x) for x in args.tiling.split(','))
    grid = tuple(int(x) for x in args.grid.split(','))
    spec = api.SystemSpec(lib, cell=capi.NIO_PRIM4, tiling=tiling, grid=grid, fill=capi.FILL_UNIFORM, spo_seed=11,
                          jastrow='synthetic')
    system = api.System(lib, spec, capi.PREC_FP64)
    w = api.Walkers(system, 1, 1)
    w.init_random(np.array([1009], dtype=np.uint32))
    stream = stream_cls()
    lib.call('walkers_set_stream', w.h, C.c_void_p(stream.cuda_stream))
    w.evaluate_log()
    lib.call('sweep_async', w.h, 1, 1, 0.5, 0)  # warm-up
    lib.call('walkers_sync', w.h)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.plain_steps):
        lib.call('sweep_async', w.h, 1, 1, 0.5, 0)
    e1.record(stream)
    lib.call('walkers_sync', w.h)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.plain_steps
    w.close()
    system.close()
    return spec.n_elec / (ms / 1e3), ms


def operating_points(value, refresh1, R, error):
    """Throughput beside the median log-ratio error it is reached at: the
    configured refresh interval R (the error window is R steps after a
    refresh) and the FP64 refresh after every step (the first step's
    error after a fresh inverse)."""
    pts = [{'recompute_every': R, 'value': value,
            'log_ratio_median': error['log_ratio_abs']['median'] if error else None}]
    if refresh1 is not None:
        pts.append({'recompute_every': 1, 'value': refresh1,
                    'log_ratio_median': error['log_ratio_abs_per_step'][0]['median'] if error else None})
    return pts


def fp64_reference_system(lib, args, api, capi):
    """The FP64 form's system on the mixed form's table: the same
    SplitMix64 coefficients rounded to FP32 (QMC_FILL_UNIFORM_F32), held and
    evaluated in FP64."""
    tiling = tuple(int(x) for x in args.tiling.split(','))
    grid = tuple(int(x) for x in args.grid.split(','))
    spec = api.SystemSpec(lib, cell=capi.NIO_PRIM4, tiling=tiling, grid=grid, fill=capi.FILL_UNIFORM_F32,
                          spo_seed=11, jastrow='synthetic')
    return spec, api.System(lib, spec, capi.PREC_FP64)


def mixed_form_error(lib, args, api, capi, spec, mixed_system, fp64_system):
    """Per-quantity error of the benchmarked mixed form (same grid, delay
    and flush engine) against the FP64 form on the same FP32-rounded table,
    positions and random streams: --error-walkers walkers, --error-steps MC
    steps of 1536 moves each (log-ratios and gradients of every move, log|det|
    drift after the first and the last step).  No refresh inside the window:
    --error-steps = the refresh interval measures the whole interval."""
    from miniqmc_b200 import precision
    W, S = args.error_walkers, args.error_steps
    seeds = (np.arange(W, dtype=np.uint32) * 7919 + 1009).astype(np.uint32)
    wm = api.Walkers(mixed_system, W, args.delay)
    wd = api.Walkers(fp64_system, W, args.delay)
    if args.flush == 'simt':
        lib.call('walkers_set_tensor_cores', wm.h, 0)
    for w in (wm, wd):
        w.init_random(seeds)
    rs = np.random.default_rng(23)
    ur = rs.uniform(size=(S, W, 1, spec.n_elec))
    de = rs.normal(size=(S, W, 1, spec.n_elec, 3))
    pts = rs.uniform(size=(256, 3)) @ np.array(spec.ions['spo_lattice']).reshape(3, 3)
    out = {'against': 'FP64 form on the same FP32-rounded table (QMC_FILL_UNIFORM_F32), same positions and '
                      'streams', 'walkers': W, 'steps': S, 'delay': args.delay,
           'flush': args.flush if args.precision == 'mixed' else 'simt',
           'spo': precision.spo_errors(mixed_system, fp64_system, pts)}
    out.update(precision.sweep_errors(wm, wd, ur, de, checkpoints=(1, S)))
    wm.close()
    wd.close()
    return out


def batched_fp64_form(lib, args, api, fp64_system, stream_cls):
    """The same fused batched sweep in FP64 (table, orbitals, inverse,
    Woodbury flush on the CUDA cores) at the bench's walker count and delay,
    at its best block size: the default (one thread per 16-byte vector of
    orbitals, 256) or 192 threads per walker, which lets four walkers share
    an SM; --fp64-steps timed MC steps after one warm-up step each, no
    refresh.  Returns (electron-moves/s, ms per step, threads)."""
    import torch
    W = args.walkers
    w = api.Walkers(fp64_system, W, args.delay)
    w.init_random((np.arange(W, dtype=np.uint32) * 7919 + 1009).astype(np.uint32))
    stream = stream_cls()
    lib.call('walkers_set_stream', w.h, C.c_void_p(stream.cuda_stream))
    w.evaluate_log()
    best = None
    for threads in (0, 192):
        if threads:
            lib.call('walkers_set_threads', w.h, threads)
        lib.call('sweep_async', w.h, 1, 1, 0.5, 0)
        lib.call('walkers_sync', w.h)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.fp64_steps):
            lib.call('sweep_async', w.h, 1, 1, 0.5, 0)
        e1.record(stream)
        lib.call('walkers_sync', w.h)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.fp64_steps
        t = C.c_int()
        lib.call('walkers_get_config', w.h, C.byref(t), None, None)
        if best is None or ms < best[0]:
            best = (ms, t.value)
    n = fp64_system.spec.n_elec
    w.close()
    return W * n / (best[0] / 1e3), best[0], best[1]


def cpu_baseline(args, n_threads, sample_walkers):
    """The CPU FP64 oracle (a port of the reference algorithm) on the host
    cores: `sample_walkers` walkers (one per thread) for one substep of the
    same system on a coarser grid (same per-move work: 64 stencil points x
    768 orbitals); returns electron-moves/s."""
    from miniqmc_b200 import api, capi
    from tests import oracle_lib
    lib = oracle_lib.library()
    tiling = tuple(int(x) for x in args.tiling.split(','))
    spec = api.SystemSpec(lib, cell=capi.NIO_PRIM4, tiling=tiling, grid=(37, 37, 18), fill=capi.FILL_UNIFORM,
                          spo_seed=11, jastrow='synthetic')
    system = api.System(lib, spec, capi.PREC_FP64)
    w = api.Walkers(system, sample_walkers, args.delay)
    seeds = np.arange(sample_walkers, dtype=np.uint32) + 7
    w.init_random(seeds)
    w.evaluate_log()
    t0 = time.perf_counter()
    w.sweep(1, 1, 0.5)
    dt = time.perf_counter() - t0
    moves = sample_walkers * spec.n_elec
    return moves / dt, ('%d walkers x 1 substep x %d electrons of NiO %s (FP64 oracle port, grid 37x37x18, k=%d)'
                        % (sample_walkers, spec.n_elec, args.tiling, args.delay))


def job_rate(moves_per_rank, seconds, world, device='cpu'):
    """Whole-job rate of a replica run: every rank moved `moves_per_rank`
    electrons; the job's time is the maximum over ranks (one all-reduce,
    outside any timed region).  Returns (rate, max seconds)."""
    import torch
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    tmax = float(t.item())
    return moves_per_rank * world / tmax, tmax


def nio_system(lib, api, capi, tiling, precision):
    """NiO tiling of the 4-atom cell with 37 grid points per cell edge (the
    148x148x74 grid of the 4x4x2 cell), SplitMix64 coefficients, synthetic
    Jastrows."""
    spec = api.SystemSpec(lib, cell=capi.NIO_PRIM4, tiling=tiling, grid=tuple(37 * t for t in tiling),
                          fill=capi.FILL_UNIFORM, spo_seed=11, jastrow='synthetic')
    return spec, api.System(lib, spec, precision)


def plain_rate(lib, api, capi, tiling, torch):
    """electron-moves/s of the plain FP64 form (1 walker per launch, delay 1)
    on one NiO tiling: one timed step after one warm-up step."""
    spec, system = nio_system(lib, api, capi, tiling, capi.PREC_FP64)
    w = api.Walkers(system, 1, 1)
    w.init_random(np.array([1009], dtype=np.uint32))
    w.evaluate_log()
    lib.call('sweep_async', w.h, 1, 1, 0.5, 0)
    lib.call('walkers_sync', w.h)
    t0 = time.perf_counter()
    lib.call('sweep_async', w.h, 1, 1, 0.5, 0)
    lib.call('walkers_sync', w.h)
    dt = time.perf_counter() - t0
    w.close()
    system.close()
    return spec.n_elec / dt


def run_extra_workload(args):
    import torch
    from miniqmc_b200 import api, capi
    lib = api.Library()
    lib.call('init', 0)
    run = {'uneven': run_uneven, 'serve': run_serve, 'nlpp': run_nlpp}[args.workload]
    out = run(args, lib, api, capi, torch)
    print(json.dumps(out), flush=True)


def run_nlpp(args, lib, api, capi, torch):
    """NonLocalPP ratios (qmc_nlpp_evaluate, the driver's form) on the
    reference's NiO-128 cell (its 32-atom cell tiled 2x2x1: 1536 e-, 128
    ions), --walkers walkers, the orbital grid of --nlpp-grid, mixed form.
    A step is one call over every walker: all electrons x ions within rmax
    1.7 x 12 points.  The dominant bytes of a point are its value-only
    stencil, 64 n coefficients."""
    grid = tuple(int(x) for x in args.nlpp_grid.split(','))
    spec = api.SystemSpec(lib, cell=capi.NIO_REF32, tiling=(2, 2, 1), grid=grid, fill=capi.FILL_UNIFORM,
                          spo_seed=11, jastrow='reference')
    system = api.System(lib, spec, capi.PREC_MIXED)
    w = api.Walkers(system, args.walkers, args.delay)
    w.init_random((np.arange(args.walkers, dtype=np.uint32) * 7919 + 1009).astype(np.uint32))
    w.evaluate_log()
    for _ in range(args.warmup):
        w.nlpp(1.7, capi.NLPP_DRIVER)
    points, times = 0, []
    clocks = ClockSampler(0)
    clocks.start()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        n, _, _ = w.nlpp(1.7, capi.NLPP_DRIVER)
        times.append(time.perf_counter() - t0)
        points += int(np.sum(n))
    clk = clocks.stop()
    total = sum(times)
    bytes_per_point = 64.0 * spec.n_orb * 4
    achieved = points * bytes_per_point / total / 1e9
    pk, kind = peaks()
    peak = pk['hbm_gbs']
    return {'metric': 'NLPP quadrature-point ratios/s', 'value': points / total, 'unit': 'ratios/s', 'n_gpus': 1,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_call': 1e3 * total / args.steps,
            'points_per_call': points / args.steps, 'higher_is_better': True, 'dtype': 'f32', 'data': 'synthetic',
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                         'frac': achieved / peak, 'algorithmic_bytes_per_point': bytes_per_point,
                         'kernel': 'nlpp_kernel<float>', 'peak_kind': kind},
            'clocks': clk,
            'config': {'workload': 'NLPP ratios, NiO 2,2,1 of the 32-atom cell: 128 ions, 1536 e-, 768 orbitals/spin, '
                                   'grid %s FP32 table, %d walkers, rmax 1.7, 12 points' % (args.nlpp_grid, args.walkers),
                       'l2': 'inputs larger than L2'}}


def run_uneven(args, lib, api, capi, torch):
    """Three NiO systems in ONE fused launch per MC step: 256 walkers of the
    2x2x1 cell (192 e-), 128 of 2x2x2 (384 e-), 64 of 4x2x2 (768 e-), each
    with the delay rank, threads per walker and flush engine the autotuner
    picked, the launch replayed from a CUDA graph."""
    parts = [((2, 2, 1), 256), ((2, 2, 2), 128), ((4, 2, 2), 64)]
    batches, systems, chosen = [], [], []
    t_tune = 0.0
    for tiling, W in parts:
        spec, system = nio_system(lib, api, capi, tiling, capi.PREC_MIXED)
        systems.append(system)
        if args.no_tune:
            best = {'delay': 16, 'threads': None, 'tensor_cores': None, 'max_moves': 1, 'ms_per_step': None}
        else:
            t0 = time.perf_counter()
            best, _ = api.autotune(lib, system, W, delays=(8, 16, 32), n_steps=2)
            t_tune += time.perf_counter() - t0
        w = api.Walkers(system, W, best['delay'])
        if best['threads'] is not None:
            lib.call('walkers_set_tensor_cores', w.h, 0)
            lib.call('walkers_set_threads', w.h, best['threads'])
            if best['tensor_cores']:
                lib.call('walkers_set_tensor_cores', w.h, 1)
            lib.call('walkers_set_move_batching', w.h, best['max_moves'])
        w.init_random((np.arange(W, dtype=np.uint32) * 7919 + 1009).astype(np.uint32))
        w.evaluate_log()
        batches.append((spec, W, w))
        chosen.append({'tiling': list(tiling), 'walkers': W, 'electrons': spec.n_elec, **best})
    g = api.Group(lib, [b[2] for b in batches])
    mode = {'auto': capi.SCHED_AUTO, 'static': capi.SCHED_STATIC, 'queue': capi.SCHED_QUEUE}[args.schedule]
    lib.call('group_set_schedule', g.h, mode, args.unit, 0)
    g.use_graph(True)
    g.sweep(args.warmup, 1, 0.5, args.recompute_every)
    g.sync()
    stream = torch.cuda.ExternalStream(g.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.sweep(args.steps, 1, 0.5, args.recompute_every)
    e1.record(stream)
    g.sync()
    ms = e0.elapsed_time(e1)
    moves = sum(W * spec.n_elec for spec, W, _ in batches) * args.steps
    st = g.stats()
    g.close()
    # the same batches launched one after another (one launch per batch per step)
    t_sep = 0.0
    for spec, W, w in batches:
        s2 = torch.cuda.Stream()
        lib.call('walkers_set_stream', w.h, C.c_void_p(s2.cuda_stream))
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(s2)
        lib.call('sweep_async', w.h, args.steps, 1, 0.5, args.recompute_every)
        a1.record(s2)
        lib.call('walkers_sync', w.h)
        t_sep += a0.elapsed_time(a1)
    return {'metric': 'electron-moves/s (uneven batch: 3 NiO systems in one launch)', 'value': moves / (ms / 1e3),
            'unit': 'electron-moves/s', 'n_gpus': 1, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': ms / args.steps, 'higher_is_better': True, 'dtype': 'f32', 'data': 'synthetic',
            'config': {'workload': 'uneven', 'batches': chosen, 'launch_threads': st['threads'],
                       'graph_launches': st['graph_launches'], 'recompute_every': args.recompute_every,
                       'autotune_s': t_tune,
                       'schedule': 'static: one CTA per walker' if args.schedule == 'static'
                                   else 'work queue, units of %d moves' % (args.unit or capi.SCHED_UNIT_DEFAULT)},
            'separate_launches': {'value': moves / (t_sep / 1e3), 'ms_per_step': t_sep / args.steps}}


def run_serve(args, lib, api, capi, torch):
    """Request loop: jobs arrive as a Poisson process (seed 3) and are NiO
    tilings (1,1,1)/(2,1,1)/(2,2,1)/(2,2,2)/(4,2,2) with probabilities
    .3/.25/.2/.15/.1, 32-256 walkers, 5-50 steps, each with its own seed.
    Reports p50/p99 latency (arrival to result) and the aggregate rate, next
    to running the same jobs one at a time in the plain FP64 form (its time
    from that form's rate measured on each tiling)."""
    rng = np.random.default_rng(3)
    tilings = [(1, 1, 1), (2, 1, 1), (2, 2, 1), (2, 2, 2), (4, 2, 2)]
    n = args.jobs
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, n))
    kinds = rng.choice(len(tilings), size=n, p=[0.3, 0.25, 0.2, 0.15, 0.1])
    walkers = rng.integers(32, 257, size=n)
    steps = rng.integers(5, 51, size=n)
    seeds = rng.integers(1, 2 ** 31 - 1, size=n)
    systems = [nio_system(lib, api, capi, t, capi.PREC_MIXED) for t in tilings]
    srv = api.Server(lib, args.budget_gb * 1e9, threads=128, recompute_every=8)
    ids, lag = [], []
    t0 = time.perf_counter()
    sub = 0
    while True:
        now = time.perf_counter() - t0
        while sub < n and arrivals[sub] <= now:
            ids.append(srv.submit(systems[kinds[sub]][1], int(walkers[sub]), int(steps[sub]), 16, int(seeds[sub])))
            lag.append(now - arrivals[sub])
            sub += 1
        running, waiting = srv.tick()
        if sub == n and running == 0 and waiting == 0:
            break
        if running == 0 and waiting == 0 and sub < n:
            time.sleep(max(0.0, arrivals[sub] - (time.perf_counter() - t0)))
    wall = time.perf_counter() - t0
    infos = [srv.job(i) for i in ids]
    lat = np.array([inf['t_done'] - inf['t_submit'] + lg for inf, lg in zip(infos, lag)])
    st = srv.stats()
    rates = {t: plain_rate(lib, api, capi, t, torch) for t in tilings}
    plain_s = sum(int(walkers[i]) * int(steps[i]) * systems[kinds[i]][0].n_elec / rates[tilings[kinds[i]]]
                  for i in range(n))
    return {'metric': 'p50/p99 job latency and electron-moves/s (request loop)',
            'value': st['electron_moves'] / wall, 'unit': 'electron-moves/s', 'n_gpus': 1,
            'latency_s': {'p50': float(np.percentile(lat, 50)), 'p99': float(np.percentile(lat, 99)),
                          'max': float(lat.max())},
            'jobs': n, 'failed': sum(inf['state'] != capi.JOB_DONE for inf in infos), 'wall_s': wall,
            'launches': st['launches'], 'dtype': 'f32', 'data': 'synthetic',
            'config': {'workload': 'serve', 'rate_per_s': args.rate, 'seed': 3, 'budget_gb': args.budget_gb,
                       'threads': 128, 'delay': 16, 'recompute_every': 8},
            'plain_fp64_one_at_a_time': {'estimated_s': plain_s, 'rates_moves_per_s':
                                         {str(t): r for t, r in rates.items()},
                                         'speedup_of_wall': plain_s / wall}}


REF_BIN = os.path.join(REPO, 'oracle', '_ref')


def reference_binary(mixed=False):
    """The reference's own miniqmc, built from its sources by
    oracle/ref_miniqmc.mk for this host's widest ISA (x86-64-v4 with
    AVX-512, else v3), or None when it was not built."""
    try:
        isa = 'v4' if ' avx512f' in open('/proc/cpuinfo').read() else 'v3'
    except OSError:
        isa = 'v3'
    path = os.path.join(REF_BIN, 'miniqmc%s_%s' % ('_mixed' if mixed else '', isa))
    return path if os.access(path, os.X_OK) else None


def reference_miniqmc(args, n_threads, steps, mixed=False, delay=None):
    """Time the reference's own miniqmc on the host cores: one walker per
    OpenMP thread (-w = threads), its Release build, OPENBLAS_NUM_THREADS=1.
    The bench's NiO tiling (n1,n2,n3) of the 4-atom cell is the reference's
    -g "n1/2 n2/2 n3/2" of its 32-atom cell (1536 e- at 4,4,2); its table is
    the 32-atom cell's at -m 2 (74^3 points; per move the same 64 stencil
    points x 768 orbitals), -x 0 leaves out the NLPP step.  electron-moves/s
    = W * steps * N / Diffusion time, from the driver's own throughput line
    (miniqmc.cpp:509-521: N_walkers * N_elec^3 / Diffusion time).  Returns
    (moves/s, description) or raises."""
    import re
    import tempfile
    exe = reference_binary(mixed)
    if exe is None:
        raise RuntimeError('reference miniqmc not built (oracle/ref_miniqmc.mk)')
    t = [int(x) for x in args.tiling.split(',')]
    if any(x % 2 for x in t):
        raise RuntimeError('tiling %s has no reference equivalent (odd factor)' % args.tiling)
    g = '%d %d %d' % (t[0] // 2, t[1] // 2, t[2] // 2)
    env = dict(os.environ, OMP_NUM_THREADS=str(n_threads), OPENBLAS_NUM_THREADS='1')
    k = args.delay if delay is None else delay
    cmd = [exe, '-g', g, '-m', '2', '-n', str(steps), '-N', '1', '-r', '0.5', '-k', str(k),
           '-w', str(n_threads), '-x', '0']
    with tempfile.TemporaryDirectory() as d:  # the driver writes info_*.xml into its working directory
        r = subprocess.run(cmd, cwd=d, env=env, capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        raise RuntimeError('reference miniqmc exited %d: %s' % (r.returncode, r.stderr[-300:]))
    m = re.search(r'Diffusion throughput \( N_walkers \* N_elec\^3 / Diffusion time \) = ([0-9.eE+-]+)', r.stdout)
    if not m:
        raise RuntimeError('no Diffusion throughput line in the reference output')
    n_elec = 12 * 32 * (t[0] // 2) * (t[1] // 2) * (t[2] // 2)
    rate = float(m.group(1)) * steps / float(n_elec) ** 2
    desc = ('reference miniqmc %s (%s build, -ffast-math -O3, OpenBLAS): -g "%s" -m 2 -k %d -w %d -n %d -x 0, '
            'one walker per thread' % (os.path.basename(exe), 'mixed-precision' if mixed else 'FP64', g,
                                       k, n_threads, steps))
    return rate, desc


def run_reference(args, rank, world):
    """The reference arm: the reference's own miniqmc Release build on all
    host cores (rank 0 only), each timed step one MC step of its walkers; its
    mixed-precision build and its rank-1 form (-k 1) are reported beside
    it."""
    if rank != 0:
        return
    ncpu = os.cpu_count() or 1
    try:
        v, desc = reference_miniqmc(args, ncpu, args.steps)
        kind = 'reference'
    except Exception as ex:
        print(json.dumps({'impl': 'reference', 'unavailable': 'reference miniqmc: %s' % ex}), flush=True)
        return
    extra = {}
    try:
        mv, mdesc = reference_miniqmc(args, ncpu, args.steps, mixed=True)
        extra['reference_mixed'] = {'value': mv, 'unit': 'electron-moves/s', 'sample': mdesc}
    except Exception as ex:
        extra['reference_mixed'] = {'value': None, 'note': str(ex)}
    try:
        # the reference's rank-1 (Sherman-Morrison) form, -k 1
        kv, kdesc = reference_miniqmc(args, ncpu, args.steps, delay=1)
        extra['reference_k1'] = {'value': kv, 'unit': 'electron-moves/s', 'sample': kdesc}
    except Exception as ex:
        extra['reference_k1'] = {'value': None, 'note': str(ex)}
    tiling = args.tiling
    print(json.dumps({
        'impl': 'reference', 'metric': 'electron-moves/s', 'value': v, 'unit': 'electron-moves/s',
        'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
        'config': {'workload': 'NiO %s (4-atom cell) = reference -g "%s": 1536 e-, k=%d' %
                   (tiling, ' '.join(str(int(x) // 2) for x in tiling.split(',')), args.delay)},
        'cpu_baseline': {'value': v, 'unit': 'electron-moves/s', 'cores': ncpu, 'kind': kind, 'sample': desc},
        'e2e': {'value': v, 'unit': 'electron-moves/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
        **extra}), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if args.impl == 'reference':
        if args.workload != 'nio128':
            if rank == 0:
                print(json.dumps({'impl': 'reference', 'unavailable': 'the CPU reference arm covers the nio128 '
                                  'workload only'}), flush=True)
            return
        run_reference(args, rank, world)
        return
    if args.workload != 'nio128':
        if rank == 0:
            run_extra_workload(args)
        return
    import torch
    import torch.distributed as dist
    from miniqmc_b200 import api, capi
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group('nccl', timeout=__import__('datetime').timedelta(seconds=600))
    lib = api.Library()
    lib.call('init', local)
    seeds = (np.arange(args.walkers, dtype=np.uint32) * 7919 + 1009 * (rank + 1)).astype(np.uint32)
    spec, system, walkers = build_workload(lib, args, capi, api, seeds)
    stream = torch.cuda.Stream()
    lib.call('walkers_set_stream', walkers.h, C.c_void_p(stream.cuda_stream))
    if args.precision == 'mixed':
        lib.call('walkers_set_tensor_cores', walkers.h, 1 if args.flush == 'tc' else 0)
    if args.threads:
        lib.call('walkers_set_threads', walkers.h, args.threads)
    if args.max_moves != 1:
        lib.call('walkers_set_move_batching', walkers.h, args.max_moves)
    mode = {'auto': capi.SCHED_AUTO, 'static': capi.SCHED_STATIC, 'queue': capi.SCHED_QUEUE}[args.schedule]
    lib.call('walkers_set_schedule', walkers.h, mode, args.unit, 0)
    sched = schedule_of(lib, walkers, args)
    walkers.evaluate_log()
    W, N = args.walkers, spec.n_elec
    count = C.c_int64()

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    # warm-up (device RNG, fully resident)
    for _ in range(args.warmup):
        lib.call('sweep_async', walkers.h, 1, 1, 0.5, args.recompute_every)
    lib.call('walkers_sync', walkers.h)
    lib.call('walkers_launch_count', walkers.h, C.byref(count))
    launches0 = count.value
    acc0 = np.zeros(W, dtype=np.int64)
    lib.call('sweep_results', walkers.h, acc0.ctypes.data_as(C.POINTER(C.c_int64)), None)
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    with torch.cuda.stream(stream):
        t_all0 = torch.cuda.Event(enable_timing=True)
        t_all1 = torch.cuda.Event(enable_timing=True)
        t_all0.record(stream)
        for s in range(args.steps):
            ev[s][0].record(stream)
            lib.call('sweep_async', walkers.h, 1, 1, 0.5, args.recompute_every)
            ev[s][1].record(stream)
        t_all1.record(stream)
    lib.call('walkers_sync', walkers.h)
    barrier()
    clk = clocks.stop()
    ms_total = t_all0.elapsed_time(t_all1)
    kernel_ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    acc = np.zeros(W, dtype=np.int64)
    lib.call('sweep_results', walkers.h, acc.ctypes.data_as(C.POINTER(C.c_int64)), None)
    lib.call('walkers_launch_count', walkers.h, C.byref(count))
    launches = count.value - launches0
    value, tmax = job_rate(W * N * args.steps, ms_total / 1e3, world, device='cuda')
    ms_total = tmax * 1e3
    a = float((acc - acc0).sum()) / (W * N * args.steps)

    # e2e through the public API: host random streams in, results out.  The
    # streams come from the host (QMC_RNG_HOST), so the device's own stream
    # generation is not part of this number.  The window starts at the same
    # phase of the FP64 refresh cycle as the device-timed one, so both hold
    # the same number of refreshes.
    e2e = None
    if not args.no_e2e:
        rs = np.random.default_rng(5 + rank)
        ur = np.ascontiguousarray(rs.uniform(size=(1, W, 1, N)))
        de = np.ascontiguousarray(rs.normal(size=(1, W, 1, N, 3)))
        pin_ur = torch.from_numpy(ur).pin_memory().numpy()
        pin_de = torch.from_numpy(de).pin_memory().numpy()
        R = args.recompute_every
        done = args.warmup + args.steps
        n_warm = 1 + ((args.warmup - done - 1) % R if R > 0 else 0)
        for _ in range(n_warm):
            walkers.sweep(1, 1, 0.5, ur=pin_ur, delta=pin_de, recompute_every=R)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            walkers.sweep(1, 1, 0.5, ur=pin_ur, delta=pin_de, recompute_every=args.recompute_every)
        barrier()
        dt = time.perf_counter() - t0
        e2e = {'value': job_rate(W * N * args.steps, dt, world, device='cuda')[0], 'unit': 'electron-moves/s',
               'h2d_bytes_per_step': int(ur.nbytes + de.nbytes), 'd2h_bytes_per_step': int(W * 16)}

    # the same sweep with the FP64 refresh after every step (the accurate
    # operating point: every step starts from a fresh FP64 inverse)
    refresh1 = None
    if args.refresh1_steps > 0 and args.recompute_every != 1:
        lib.call('sweep_async', walkers.h, 1, 1, 0.5, 1)  # warm
        barrier()
        with torch.cuda.stream(stream):
            r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            r0.record(stream)
            for _ in range(args.refresh1_steps):
                lib.call('sweep_async', walkers.h, 1, 1, 0.5, 1)
            r1.record(stream)
        lib.call('walkers_sync', walkers.h)
        barrier()
        refresh1 = job_rate(W * N * args.refresh1_steps, r0.elapsed_time(r1) / 1e3, world, device='cuda')[0]

    pk, pk_kind = peaks()
    n, I, k = spec.n_orb, spec.n_ions, args.delay
    s = 4 if args.precision == 'mixed' else 8
    bpm = algorithmic_bytes_per_move(n, N, I, k, s, a)
    # the sweep kernel's own launch time: steps that also ran the periodic
    # FP64 refresh of the inverses are left out (reported as recompute_ms)
    R = args.recompute_every
    refresh = [R > 0 and (args.warmup + i + 1) % R == 0 for i in range(args.steps)]
    sweep_ms = [t for t, r in zip(kernel_ms, refresh) if not r] or kernel_ms
    refresh_ms = [t for t, r in zip(kernel_ms, refresh) if r]
    avg_launch_ms = float(np.mean(sweep_ms))
    recompute_ms = float(np.mean(refresh_ms)) - avg_launch_ms if refresh_ms else None
    achieved = bpm * W * N / (avg_launch_ms / 1e3) / 1e9
    roofline = {'bound': 'hbm', 'achieved': achieved, 'peak': pk['hbm_gbs'], 'unit': 'GB/s',
                'frac': achieved / pk['hbm_gbs'],
                'traffic': (MEASURED_TRAFFIC_PER_MOVE * W * N
                            if (args.precision == 'mixed' and args.delay == 32) else None),
                'traffic_source': 'ncu dram bytes per move of sweep_queue_kernel (512 walkers, grid 148x148x74) '
                                  'x moves per launch',
                'peak_kind': pk_kind, 'algorithmic_bytes_per_move': bpm,
                'kernel': '%s<%s>' % (sched['kernel'], 'float' if s == 4 else 'double'), 'launch_ms': avg_launch_ms}
    # the Woodbury GEMMs on the tensor cores (tcgen05 kind::tf32, 3xTF32):
    # per flush GEMM1 (n x npad by npad x k) and GEMM2 (n x k by k x npad),
    # three TF32 products each, i.e. 12 n npad flops per accepted move.
    # The TF32 peak is taken as half the measured dense BF16 rate (TF32
    # MMAs run at half the BF16 rate).
    tensor = None
    if args.precision == 'mixed' and args.flush == 'tc':
        npad = -(-n // 4) * 4
        tflop = 12.0 * n * npad * a * W * N / 1e12
        tf32_peak = pk['bf16_tflops'] / 2
        ach = tflop / (avg_launch_ms / 1e3)
        tensor = {'kernel': '%s Woodbury flush (tcgen05 kind::tf32, 3xTF32)' % sched['kernel'], 'tflop_per_launch': tflop,
                  'achieved': ach, 'peak': tf32_peak, 'unit': 'TFLOP/s', 'frac': ach / tf32_peak,
                  'peak_kind': pk_kind + ' bf16 / 2',
                  'ncu_pipe_tensor_cycles_active_pct': 0.75}
    error, batched = None, None
    if rank == 0 and world == 1 and args.precision == 'mixed' and (args.error_walkers > 0 or args.fp64_steps > 0):
        _, fp64_sys = fp64_reference_system(lib, args, api, capi)
        if args.error_walkers > 0:
            error = mixed_form_error(lib, args, api, capi, spec, system, fp64_sys)
        if args.fp64_steps > 0:
            bv, bms, bthr = batched_fp64_form(lib, args, api, fp64_sys, torch.cuda.Stream)
            batched = {'value': bv, 'unit': 'electron-moves/s', 'ms_per_step': bms,
                       'form': 'FP64 fused batched sweep, %d walkers, delay %d, CUDA-core flush, same grid, '
                               '%d threads per walker' % (W, args.delay, bthr),
                       'steps_timed': args.fp64_steps, 'value_over_batched_fp64': value / bv}
        fp64_sys.close()
    plain = None
    if rank == 0 and world == 1 and args.plain_steps > 0:
        pv, pms = plain_fp64_form(lib, args, api, capi, torch.cuda.Stream)
        plain = {'value': pv, 'unit': 'electron-moves/s', 'ms_per_walker_step': pms,
                 'form': 'FP64, 1 walker per launch, delay rank 1, walkers in sequence',
                 'walker_steps_timed': args.plain_steps, 'value_over_plain': value / pv}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        ncpu = os.cpu_count() or 1
        try:  # the reference's own miniqmc (2 MC steps of one walker per core)
            v, desc = reference_miniqmc(args, ncpu, 2)
            cpu = {'value': v, 'unit': 'electron-moves/s', 'cores': ncpu, 'kind': 'reference', 'sample': desc}
        except Exception as ex:  # the baseline is reported, never required
            cpu = {'value': None, 'unit': 'electron-moves/s', 'cores': ncpu, 'kind': 'reference',
                   'sample': 'failed: %s' % ex}
        if args.port_baseline:
            try:
                v, desc = cpu_baseline(args, ncpu, args.cpu_walkers or ncpu)
                cpu['port'] = {'value': v, 'kind': 'port', 'sample': desc}
            except Exception as ex:
                cpu['port'] = {'value': None, 'sample': 'failed: %s' % ex}
    if rank == 0:
        out = {
            'metric': 'electron-moves/s', 'value': value, 'unit': 'electron-moves/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms_total / args.steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'f32' if args.precision == 'mixed' else 'f64', 'data': 'synthetic',
            'config': {'workload': 'NiO %s of the 4-atom cell: %d atoms, %d e-, %d orbitals/spin, grid %s '
                                   '%s table, %d walkers/GPU, delay %d, %s'
                                   % (args.tiling, I, N, n, args.grid, 'FP32' if s == 4 else 'FP64', W, k,
                                      args.precision),
                       'walkers_per_gpu': W,
                       'l2': 'inputs larger than L2 (%.2f GB spline table, %.1f GB walker state)'
                             % (system_bytes(lib, system) / 1e9, walkers_bytes(lib, walkers) / 1e9),
                       'acceptance': a, 'parallelism': 'replicas x%d' % world,
                       'flush': args.flush if args.precision == 'mixed' else 'simt',
                       'recompute_every': args.recompute_every, 'recompute_ms': recompute_ms,
                       'schedule': sched['text']},
            'roofline': roofline, 'tensor': tensor, 'cpu_baseline': cpu, 'e2e': e2e, 'clocks': clk,
            'plain_fp64': plain, 'batched_fp64': batched, 'error': error,
            'operating_points': operating_points(value, refresh1, args.recompute_every, error),
            'gpu_launches': launches,
        }
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


def system_bytes(lib, system):
    b = C.c_size_t()
    lib.call('system_bytes', system.h, C.byref(b))
    return b.value


def walkers_bytes(lib, walkers):
    b = C.c_size_t()
    lib.call('walkers_bytes', walkers.h, C.byref(b))
    return b.value


if __name__ == '__main__':
    main()
