"""Loader for the CPU FP64 oracle (oracle/liboracle.so) -- the checker.

The oracle exports the same surface as the product's C ABI with the prefix
oracle_, so it plugs into miniqmc_b200.api.Library unchanged.  Built on
demand with oracle/Makefile.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from miniqmc_b200 import api, capi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(REPO, 'oracle', 'liboracle.so')
GOLDEN = os.path.join(REPO, 'tests', 'golden')

_lib = None

# arithmetic of the oracle's orbital and determinant path (qmc_oracle.hpp
# ARITH_*): FP32 orbitals, FP32 determinant algebra, FP32 log|det|
# accumulation; all three together restate the reference's mixed-precision
# build of that path
ARITH_SPO32, ARITH_DET32, ARITH_LOG32 = 1, 2, 4
ARITH_REFERENCE_MIXED = ARITH_SPO32 | ARITH_DET32 | ARITH_LOG32


def build():
    src = [os.path.join(REPO, 'oracle', f) for f in ('oracle_capi.cpp', 'qmc_oracle.hpp')]
    if (not os.path.exists(ORACLE_SO)
            or max(os.path.getmtime(s) for s in src) > os.path.getmtime(ORACLE_SO)):
        subprocess.check_call(['make', '-s', '-C', os.path.join(REPO, 'oracle')])


def library():
    global _lib
    if _lib is None:
        build()
        extra = {
            'rng_uniform': (C.c_int, [C.c_uint32, C.c_int, capi.PD]),
            'rng_normal': (C.c_int, [C.c_uint32, C.c_int, C.c_int, capi.PD]),
            'rng_words': (C.c_int, [C.c_uint32, C.c_int, C.POINTER(C.c_uint32)]),
            'primes': (C.c_int, [C.c_int, C.POINTER(C.c_uint32)]),
            'splitmix_uniform': (C.c_double, [C.c_uint64, C.c_uint64]),
            'distance_row': (C.c_int, [capi.PD, capi.PD, capi.PD, C.c_int, C.c_int, capi.PD, capi.PD]),
            'functor_eval': (C.c_int, [C.POINTER(capi.Functor), C.c_double, capi.PD]),
            'j3_functor_eval': (C.c_int, [C.POINTER(capi.J3Functor), C.c_double, C.c_double, C.c_double,
                                          capi.PD]),
            'walkers_skip': (C.c_int, [C.c_void_p, C.c_int]),
            'num_threads': (C.c_int, []),
            'detengine_delay_count': (C.c_int, [C.c_void_p]),
            'system_set_arith': (C.c_int, [C.c_void_p, C.c_int]),
        }
        _lib = api.Library(ORACLE_SO, prefix='oracle_', extra=extra)
    return _lib


def pd(a):
    return a.ctypes.data_as(capi.PD)
