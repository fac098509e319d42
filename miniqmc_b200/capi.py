"""ctypes declarations of the C ABI in include/qmcgpu.h.

`bind(lib, prefix)` sets argtypes/restype on every entry point of a loaded
shared library that exports the qmc_* surface under `prefix` (the product
library uses "qmc_").  The struct layouts here must match include/qmcgpu.h.
"""
import ctypes as C

QMC_OK = 0
STATUS = {0: 'QMC_OK', 1: 'QMC_ERR_ARG', 2: 'QMC_ERR_CUDA', 3: 'QMC_ERR_OOM', 4: 'QMC_ERR_SINGULAR',
          5: 'QMC_ERR_NONFINITE', 6: 'QMC_ERR_TIMEOUT', 7: 'QMC_ERR_STATE', 8: 'QMC_ERR_NODEVICE',
          9: 'QMC_ERR_ADMISSION', 10: 'QMC_ERR_CAPACITY'}
PREC_FP64, PREC_MIXED = 0, 1
NLPP_SPHERE, NLPP_DRIVER = 0, 1
NOALLOC_MAX_N = 768  # largest n of qmc_invert_transpose_noalloc
FILL_USER, FILL_REFERENCE, FILL_UNIFORM, FILL_UNIFORM_F32 = 0, 1, 2, 3
LAP_HXX, LAP_TRACE = 0, 1
WF_DET, WF_J1, WF_J2, WF_ALL, WF_J3 = 1, 2, 4, 7, 8
J3_PARAMS = 26
RNG_DEVICE, RNG_HOST = 0, 1
PREFETCH_AUTO, PREFETCH_OFF, PREFETCH_ON = 0, 1, 2
SCHED_AUTO, SCHED_STATIC, SCHED_QUEUE = 0, 1, 2
SCHED_UNIT_DEFAULT = 16
NIO_REF32, NIO_PRIM4 = 0, 1
NIO_QUIRK_UNIT_IONS, NIO_QUIRK_ONE_GROUP = 1, 2
MAX_FUNCTOR_COEFS = 32
MAX_ION_GROUPS = 4


class Functor(C.Structure):
    _fields_ = [('n_coefs', C.c_int), ('cutoff', C.c_double), ('delta_r_inv', C.c_double),
                ('coefs', C.c_double * MAX_FUNCTOR_COEFS)]


class J3Functor(C.Structure):
    _fields_ = [('cutoff', C.c_double), ('gamma', C.c_double * 64)]


class SystemDesc(C.Structure):
    _fields_ = [('lattice', C.c_double * 9), ('n_ions', C.c_int), ('n_ion_groups', C.c_int),
                ('ion_pos', C.POINTER(C.c_double)), ('ion_group', C.POINTER(C.c_int)),
                ('n_elec', C.c_int), ('n_up', C.c_int), ('spo_lattice', C.c_double * 9),
                ('grid', C.c_int * 3), ('n_orb', C.c_int), ('spo_fill', C.c_int),
                ('spo_seed', C.c_uint64), ('spo_user_coefs', C.POINTER(C.c_double)),
                ('lap_mode', C.c_int), ('components', C.c_int),
                ('j1', Functor * MAX_ION_GROUPS), ('j2_uu', Functor), ('j2_ud', Functor),
                ('j3_same', J3Functor * MAX_ION_GROUPS), ('j3_diff', J3Functor * MAX_ION_GROUPS)]


class SweepOpts(C.Structure):
    _fields_ = [('n_steps', C.c_int), ('n_substeps', C.c_int), ('accept', C.c_double),
                ('rng_mode', C.c_int), ('ur', C.POINTER(C.c_double)), ('delta', C.POINTER(C.c_double)),
                ('recompute_every', C.c_int), ('trace', C.POINTER(C.c_double)),
                ('n_accepted', C.POINTER(C.c_int64)), ('logpsi', C.POINTER(C.c_double))]


class TuneResult(C.Structure):
    _fields_ = [('delay', C.c_int), ('threads', C.c_int), ('tensor_cores', C.c_int), ('max_moves', C.c_int),
                ('ms_per_step', C.c_double)]


JOB_WAITING, JOB_RUNNING, JOB_DONE, JOB_FAILED = 0, 1, 2, 3


class JobInfo(C.Structure):
    _fields_ = [('state', C.c_int), ('status', C.c_int), ('steps_done', C.c_int), ('n_accepted', C.c_int64),
                ('logpsi_mean', C.c_double), ('t_submit', C.c_double), ('t_start', C.c_double),
                ('t_done', C.c_double)]


P = C.c_void_p
PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int)
I = C.c_int
D = C.c_double

# name -> (restype, argtypes); names without the prefix
SIGNATURES = {
    'nio_count': (I, [I, I, I, I, PI]),
    'nio_build': (I, [I, I, I, I, I, PD, PD, PI, PI, PD]),
    'nio_jastrows': (I, [PD, C.POINTER(Functor), C.POINTER(Functor), C.POINTER(Functor), C.POINTER(Functor)]),
    'functor_setup': (I, [I, D, D, PD, C.POINTER(Functor)]),
    'nio_j3': (I, [PD, C.POINTER(J3Functor), C.POINTER(J3Functor)]),
    'j3_functor_setup': (I, [D, PD, C.POINTER(J3Functor)]),
    'lattice_ws_radius': (I, [PD, PD]),
    'system_create': (I, [C.POINTER(SystemDesc), I, C.POINTER(P)]),
    'system_destroy': (I, [P]),
    'spo_evaluate_vgh': (I, [P, I, PD, PD, PD, PD]),
    'spo_evaluate_v': (I, [P, I, PD, PD]),
    'walkers_create': (I, [P, I, I, C.POINTER(P)]),
    'walkers_destroy': (I, [P]),
    'walkers_init_random': (I, [P, C.POINTER(C.c_uint32)]),
    'walkers_set_positions': (I, [P, PD]),
    'walkers_get_positions': (I, [P, PD]),
    'pset_make_move': (I, [P, I, PD]),
    'pset_accept_reject': (I, [P, I, PI]),
    'pset_get_temp_rows': (I, [P, PD, PD, PD, PD]),
    'wf_evaluate_log': (I, [P, PD]),
    'wf_eval_grad': (I, [P, I, PD]),
    'wf_ratio_grad': (I, [P, I, PD, PD]),
    'wf_ratio': (I, [P, I, PD]),
    'wf_evaluate_ratios': (I, [P, I, I, I, PD, PD]),
    'wf_accept_restore': (I, [P, I, PI]),
    'wf_complete_updates': (I, [P]),
    'wf_evaluate_gl': (I, [P, PD, PD, PD]),
    'wf_components': (I, [P, PD]),
    'wf_get_inverse': (I, [P, I, I, PD]),
    'sweep': (I, [P, C.POINTER(SweepOpts)]),
    'detengine_create': (I, [I, I, C.POINTER(P)]),
    'detengine_destroy': (I, [P]),
    'detengine_invert_transpose': (I, [P, PD, PD, PD]),
    'detengine_get_inv_row': (I, [P, I, PD]),
    'detengine_accept_row': (I, [P, I, PD]),
    'detengine_update_inv_mat': (I, [P]),
    'detengine_get_ainv': (I, [P, PD]),
    'nlpp_evaluate': (I, [P, D, I, C.POINTER(C.c_int64), PD, PD, I]),
    'nlpp_sphere': (I, [I, PD]),
}

# entry points only the product library exports
PRODUCT_ONLY = {
    'status_string': (C.c_char_p, [I]),
    'last_error': (C.c_char_p, []),
    'init': (I, [I]),
    'system_bytes': (I, [P, C.POINTER(C.c_size_t)]),
    'walkers_bytes': (I, [P, C.POINTER(C.c_size_t)]),
    'walkers_set_stream': (I, [P, P]),
    'pset_update': (I, [P]),
    'pset_set_active': (I, [P, I]),
    'pset_done': (I, [P]),
    'detengine_create_prec': (I, [I, I, I, C.POINTER(P)]),
    'detengine_set_tensor_cores': (I, [P, I]),
    'walkers_set_tensor_cores': (I, [P, I]),
    'walkers_set_wait_limit': (I, [P, C.c_longlong]),
    'walkers_set_move_batching': (I, [P, I]),
    'walkers_set_threads': (I, [P, I]),
    'walkers_set_prefetch': (I, [P, I]),
    'walkers_set_schedule': (I, [P, I, I, I]),
    'group_set_schedule': (I, [P, I, I, I]),
    'local_kinetic': (I, [P, PD]),
    'walkers_checkpoint_bytes': (I, [P, C.POINTER(C.c_size_t)]),
    'walkers_checkpoint': (I, [P, P, C.c_size_t]),
    'walkers_restore': (I, [P, P, C.c_size_t]),
    'walkers_get_config': (I, [P, PI, PI, PI]),
    'walkers_occupancy': (I, [P, PI]),
    'group_create': (I, [C.POINTER(P), I, C.POINTER(P)]),
    'group_destroy': (I, [P]),
    'group_set_threads': (I, [P, I]),
    'group_use_graph': (I, [P, I]),
    'group_sweep': (I, [P, I, I, D, I]),
    'group_sync': (I, [P]),
    'group_stream': (I, [P, C.POINTER(P)]),
    'group_stats': (I, [P, PI, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    'autotune': (I, [P, I, PI, I, I, C.POINTER(TuneResult), I, PI, C.POINTER(TuneResult)]),
    'server_create': (I, [C.c_size_t, I, I, C.POINTER(P)]),
    'server_destroy': (I, [P]),
    'server_submit': (I, [P, P, I, I, I, C.c_uint32, C.POINTER(C.c_int64)]),
    'server_tick': (I, [P, PI, PI]),
    'server_job': (I, [P, C.c_int64, C.POINTER(JobInfo)]),
    'server_stats': (I, [P, C.POINTER(C.c_size_t), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    'invert_transpose_noalloc': (I, [I, P, P, PD, PD, P]),
    'sweep_async': (I, [P, I, I, D, I]),
    'step': (I, [P, I, D, PD, PD, PI]),
    'spo_evaluate_batch': (I, [P, I, P, P, P]),
    'walkers_sync': (I, [P]),
    'sweep_results': (I, [P, C.POINTER(C.c_int64), PD]),
    'walkers_launch_count': (I, [P, C.POINTER(C.c_int64)]),
    'walkers_enable_timers': (I, [P, I]),
    'walkers_phase_times': (I, [P, PD, PI]),
}
PHASES = ['random', 'getInvRow', 'spo+det dots', 'jastrow sums', 'reduce+ratio', 'acceptRow', 'woodbury flush',
          'J2 accept', 'position', 'completeUpdates', 'evaluateGL', 'move setup',
          'flush U2 image', 'flush GEMM1']


def bind(lib, prefix, extra=None):
    """Attach ctypes signatures; returns {short_name: function}."""
    table = dict(SIGNATURES)
    if extra:
        table.update(extra)
    out = {}
    for name, (res, args) in table.items():
        fn = getattr(lib, prefix + name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
        out[name] = fn
    return out
