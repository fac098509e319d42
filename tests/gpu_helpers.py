"""Shared setup for the GPU parity tests: the product library (CUDA path)
and the oracle (checker) driven through the same API calls."""
import numpy as np
import pytest

from miniqmc_b200 import api, capi
from tests import oracle_lib

_prod = None


def product():
    """The product library; the GPU tests fail (not skip) if it is missing."""
    global _prod
    if _prod is None:
        from miniqmc_b200 import build
        build.build()
        _prod = api.Library()
        _prod.call('init', 0)
    return _prod


def oracle():
    return oracle_lib.library()


def spec_pair(cell=capi.NIO_PRIM4, tiling=(1, 1, 1), quirks=0, grid=(12, 12, 12), fill=capi.FILL_UNIFORM,
              jastrow='reference', components=capi.WF_ALL, lap_mode=capi.LAP_HXX, n_orb=None, spo_seed=11):
    kw = dict(cell=cell, tiling=tiling, quirks=quirks, grid=grid, fill=fill, jastrow=jastrow,
              components=components, lap_mode=lap_mode, n_orb=n_orb, spo_seed=spo_seed)
    return api.SystemSpec(product(), **kw), api.SystemSpec(oracle(), **kw)


def make_pair(precision=capi.PREC_FP64, walkers=1, delay=1, seeds=None, **kw):
    sp, so = spec_pair(**kw)
    gs = api.System(product(), sp, precision)
    os_ = api.System(oracle(), so, precision)
    gw = api.Walkers(gs, walkers, delay)
    ow = api.Walkers(os_, walkers, delay)
    if seeds is None:
        seeds = oracle_primes(walkers)
    gw.init_random(seeds)
    ow.init_random(seeds)
    return gw, ow


def oracle_primes(n):
    import ctypes as C
    p = np.zeros(n, dtype=np.uint32)
    oracle().fn['primes'](n, p.ctypes.data_as(C.POINTER(C.c_uint32)))
    return p


def host_streams(seeds, N, n_steps, n_substeps):
    """ur[n_steps][W][nsub][N], delta[n_steps][W][nsub][N][3] from each walker's
    oracle stream after build_els (3N uniforms), in the driver's draw order."""
    W = len(seeds)
    ur = np.zeros((n_steps, W, n_substeps, N))
    de = np.zeros((n_steps, W, n_substeps, N, 3))
    lib = oracle()
    for w, s in enumerate(seeds):
        # total draws: 3N (positions) then per substep N uniforms + 3N normals
        per = N + 2 * ((3 * N + 1) // 2)
        tot = 3 * N + n_steps * n_substeps * per
        u = np.zeros(tot)
        lib.fn['rng_uniform'](int(s), tot, oracle_lib.pd(u))
        off = 3 * N
        for st in range(n_steps):
            for l in range(n_substeps):
                ur[st, w, l] = u[off:off + N]
                off += N
                nrm = np.zeros(3 * N)
                lib.fn['rng_normal'](int(s), off, 3 * N, oracle_lib.pd(nrm))
                de[st, w, l] = nrm.reshape(N, 3)
                off += 2 * ((3 * N + 1) // 2)
    return ur, de


gpu = pytest.mark.gpu
