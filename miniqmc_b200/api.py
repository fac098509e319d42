"""Python mirror of miniqmc's ParticleSet / SPOSet / WaveFunction interface.

The classes below call a shared library that exports the C ABI of
include/qmcgpu.h.  `Library()` loads the product library (libqmcgpu.so,
built in-tree by miniqmc_b200/build.py); there is no CPU fallback -- if the
library or a CUDA device is missing, the calls fail loudly.

Reference interface each method mirrors (QMCPACK/miniqmc):
  Walkers.make_move / accept_reject     ParticleSet::flex_makeMove, acceptMove,
                                        rejectMove (ParticleSet.cpp:316-378)
  Walkers.evaluate_log / eval_grad /    WaveFunction::evaluateLog, evalGrad,
  ratio_grad / ratio / accept_restore / ratioGrad, ratio, acceptMove, restore,
  complete_updates / evaluate_gl        completeUpdates, evaluateGL
                                        (WaveFunction.cpp:178-279)
  System.spo_vgh / spo_v                SPOSet::evaluate (SPOSet.h:55-66)
  Walkers.sweep                         the PbyP loop of miniqmc.cpp:406-468
"""
import ctypes as C
import os

import numpy as np

from . import capi

_HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIB = os.path.join(_HERE, 'libqmcgpu.so')


class QMCError(RuntimeError):
    def __init__(self, status, where, detail=''):
        self.status = status
        super().__init__('%s failed: %s %s' % (where, capi.STATUS.get(status, status), detail))


def _pd(a):
    return None if a is None else a.ctypes.data_as(capi.PD)


def _pi(a):
    return None if a is None else a.ctypes.data_as(capi.PI)


class Library:
    """A loaded qmc_* C-ABI library."""

    def __init__(self, path=None, prefix='qmc_', extra=None):
        path = path or DEFAULT_LIB
        if not os.path.exists(path):
            raise FileNotFoundError('%s not built; run miniqmc_b200/build.py (or __graft_entry__.build())'
                                    % path)
        self.path = path
        self.prefix = prefix
        self.lib = C.CDLL(path)
        if extra is None and prefix == 'qmc_':
            extra = capi.PRODUCT_ONLY
        self.fn = capi.bind(self.lib, prefix, extra)

    def call(self, name, *args):
        st = self.fn[name](*args)
        if st != capi.QMC_OK:
            detail = ''
            if 'last_error' in self.fn:
                detail = (self.fn['last_error']() or b'').decode()
            raise QMCError(st, self.prefix + name, detail)
        return st

    def has(self, name):
        return name in self.fn

    # ---- builders --------------------------------------------------------
    def nio(self, cell=capi.NIO_PRIM4, tiling=(1, 1, 1), quirks=0):
        n = C.c_int()
        self.call('nio_count', cell, tiling[0], tiling[1], tiling[2], C.byref(n))
        lat = np.zeros(9)
        spo_lat = np.zeros(9)
        pos = np.zeros((n.value, 3))
        grp = np.zeros(n.value, dtype=np.int32)
        ng = C.c_int()
        st = self.fn['nio_build'](cell, tiling[0], tiling[1], tiling[2], quirks, _pd(lat), _pd(pos), _pi(grp),
                                  C.byref(ng), _pd(spo_lat))
        if st < 0:
            raise QMCError(-st, 'nio_build')
        return dict(lattice=lat, ion_pos=pos, ion_group=grp, n_groups=ng.value, spo_lattice=spo_lat)

    def functor(self, n_params, rcut, cusp, params):
        f = capi.Functor()
        p = np.ascontiguousarray(params, dtype=np.float64)
        self.call('functor_setup', n_params, rcut, cusp, _pd(p), C.byref(f))
        return f

    def nio_jastrows(self, lattice):
        fs = [capi.Functor() for _ in range(4)]
        lat = np.ascontiguousarray(lattice, dtype=np.float64)
        self.call('nio_jastrows', _pd(lat), *[C.byref(f) for f in fs])
        return dict(j1=[fs[0], fs[1]], j2_uu=fs[2], j2_ud=fs[3])

    def nio_j3(self, lattice):
        """buildJeeI's functors: dict(same=[species 0, 1], diff=[species 0, 1])."""
        same = (capi.J3Functor * 2)()
        diff = (capi.J3Functor * 2)()
        lat = np.ascontiguousarray(lattice, dtype=np.float64)
        self.call('nio_j3', _pd(lat), same, diff)
        return dict(same=[same[0], same[1]], diff=[diff[0], diff[1]])

    def j3_functor(self, rcut, params):
        f = capi.J3Functor()
        p = np.ascontiguousarray(params, dtype=np.float64)
        assert p.size == capi.J3_PARAMS
        self.call('j3_functor_setup', rcut, _pd(p), C.byref(f))
        return f

    def ws_radius(self, lattice):
        ws = C.c_double()
        lat = np.ascontiguousarray(lattice, dtype=np.float64)
        self.call('lattice_ws_radius', _pd(lat), C.byref(ws))
        return ws.value


_M64 = (1 << 64) - 1


def splitmix_uniform(seed, index):
    """SplitMix64 (Steele, Lea & Flood 2014) mapped to [0,1) with 53 bits."""
    z = (seed + (index + 1) * 0x9E3779B97F4A7C15) & _M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    z ^= z >> 31
    return (z >> 11) * (1.0 / 9007199254740992.0)


def synthetic_jastrows(lib, lattice, n_ion_groups=2, seed=13, n_params=8):
    """Jastrows of the synthetic NiO workloads (same values as the C entry
    point qmc_synthetic_jastrows): knot i of functor f is uniform in
    [-0.1, 0.1) from SplitMix64(seed, 64 f + i), f = 0 (uu), 1 (ud), 2 + g
    (ion species g); cutoff = half the Wigner-Seitz radius; cusp 0 (J2) and
    -0.25 (J1) as the reference's tables."""
    rc = 0.5 * lib.ws_radius(lattice)

    def knots(f):
        return [0.2 * splitmix_uniform(seed, 64 * f + i) - 0.1 for i in range(n_params)]
    j2_uu = lib.functor(n_params, rc, 0.0, knots(0))
    j2_ud = lib.functor(n_params, rc, 0.0, knots(1))
    j1 = [lib.functor(n_params, rc, -0.25, knots(2 + g)) for g in range(n_ion_groups)]
    return dict(j1=j1, j2_uu=j2_uu, j2_ud=j2_ud)


class SystemSpec:
    """Host description of one system (qmc_system_desc plus the arrays it
    points to, kept alive here)."""

    def __init__(self, lib, cell=capi.NIO_PRIM4, tiling=(1, 1, 1), quirks=0, grid=(37, 37, 37),
                 fill=capi.FILL_UNIFORM, spo_seed=11, jastrow='reference', components=capi.WF_ALL,
                 lap_mode=capi.LAP_HXX, user_coefs=None, n_orb=None):
        ions = lib.nio(cell, tiling, quirks)
        self.ions = ions
        n_ions = len(ions['ion_group'])
        n_elec = 12 * n_ions  # count_electrons (nio.hpp:16-20)
        self.n_elec = n_elec
        self.n_up = n_elec // 2
        self.n_orb = n_orb or self.n_up
        self.n_ions = n_ions
        self.grid = tuple(grid)
        d = capi.SystemDesc()
        d.lattice[:] = ions['lattice']
        d.n_ions = n_ions
        d.n_ion_groups = ions['n_groups']
        self._pos = np.ascontiguousarray(ions['ion_pos'])
        self._grp = np.ascontiguousarray(ions['ion_group'], dtype=np.int32)
        d.ion_pos = _pd(self._pos)
        d.ion_group = _pi(self._grp)
        d.n_elec = n_elec
        d.n_up = self.n_up
        d.spo_lattice[:] = ions['spo_lattice']
        d.grid[:] = grid
        d.n_orb = self.n_orb
        d.spo_fill = fill
        d.spo_seed = spo_seed
        self._coefs = None
        if user_coefs is not None:
            self._coefs = np.ascontiguousarray(user_coefs, dtype=np.float64)
            d.spo_user_coefs = _pd(self._coefs)
        d.lap_mode = lap_mode
        d.components = components
        if jastrow == 'reference':
            js = lib.nio_jastrows(ions['lattice'])
        else:
            js = synthetic_jastrows(lib, ions['lattice'], ions['n_groups'])
        for g in range(min(len(js['j1']), capi.MAX_ION_GROUPS)):
            d.j1[g] = js['j1'][g]
        d.j2_uu = js['j2_uu']
        d.j2_ud = js['j2_ud']
        if components & capi.WF_J3:
            # buildJeeI's tables (species 0 and 1; a third or fourth species
            # reuses species 1's functors)
            j3 = lib.nio_j3(ions['lattice'])
            for g in range(ions['n_groups']):
                d.j3_same[g] = j3['same'][min(g, 1)]
                d.j3_diff[g] = j3['diff'][min(g, 1)]
            js = dict(js, j3=j3)
        self.desc = d
        self.jastrows = js


class System:
    def __init__(self, lib, spec, precision=capi.PREC_FP64):
        self.lib = lib
        self.spec = spec
        self.precision = precision
        h = C.c_void_p()
        lib.call('system_create', C.byref(spec.desc), precision, C.byref(h))
        self.h = h

    def close(self):
        if self.h:
            self.lib.call('system_destroy', self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def spo_vgh(self, pos):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        n, norb = len(pos), self.spec.n_orb
        v = np.zeros((n, norb))
        g = np.zeros((n, 3, norb))
        h = np.zeros((n, 6, norb))
        self.lib.call('spo_evaluate_vgh', self.h, n, _pd(pos), _pd(v), _pd(g), _pd(h))
        return v, g, h

    def spo_v(self, pos):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        v = np.zeros((len(pos), self.spec.n_orb))
        self.lib.call('spo_evaluate_v', self.h, len(pos), _pd(pos), _pd(v))
        return v


class Walkers:
    """A batch of W walkers of one system (device-resident in the product)."""

    def __init__(self, system, n_walkers, delay_rank=1):
        self.sys = system
        self.lib = system.lib
        self.W = n_walkers
        self.k = delay_rank
        self.N = system.spec.n_elec
        h = C.c_void_p()
        self.lib.call('walkers_create', system.h, n_walkers, delay_rank, C.byref(h))
        self.h = h

    def close(self):
        if self.h:
            self.lib.call('walkers_destroy', self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_random(self, seeds):
        s = np.ascontiguousarray(seeds, dtype=np.uint32)
        self.lib.call('walkers_init_random', self.h, s.ctypes.data_as(C.POINTER(C.c_uint32)))

    def positions(self):
        R = np.zeros((self.W, self.N, 3))
        self.lib.call('walkers_get_positions', self.h, _pd(R))
        return R

    def set_positions(self, R):
        R = np.ascontiguousarray(R, dtype=np.float64)
        self.lib.call('walkers_set_positions', self.h, _pd(R))

    # ParticleSet
    def make_move(self, iat, displ):
        d = np.ascontiguousarray(displ, dtype=np.float64).reshape(self.W, 3)
        self.lib.call('pset_make_move', self.h, iat, _pd(d))

    def accept_reject(self, iat, accept):
        a = np.ascontiguousarray(accept, dtype=np.int32)
        self.lib.call('pset_accept_reject', self.h, iat, _pi(a))

    def temp_rows(self):
        I = self.sys.spec.n_ions
        aa_r = np.zeros((self.W, self.N))
        aa_dr = np.zeros((self.W, self.N, 3))
        ab_r = np.zeros((self.W, I))
        ab_dr = np.zeros((self.W, I, 3))
        self.lib.call('pset_get_temp_rows', self.h, _pd(aa_r), _pd(aa_dr), _pd(ab_r), _pd(ab_dr))
        return aa_r, aa_dr, ab_r, ab_dr

    # WaveFunction
    def evaluate_log(self):
        out = np.zeros(self.W)
        self.lib.call('wf_evaluate_log', self.h, _pd(out))
        return out

    def eval_grad(self, iat):
        g = np.zeros((self.W, 3))
        self.lib.call('wf_eval_grad', self.h, iat, _pd(g))
        return g

    def ratio_grad(self, iat):
        r = np.zeros(self.W)
        g = np.zeros((self.W, 3))
        self.lib.call('wf_ratio_grad', self.h, iat, _pd(r), _pd(g))
        return r, g

    def ratio(self, iat):
        r = np.zeros(self.W)
        self.lib.call('wf_ratio', self.h, iat, _pd(r))
        return r

    def set_schedule(self, mode=capi.SCHED_AUTO, unit_moves=0, ctas=0):
        """qmc_walkers_set_schedule: the fused sweep's CTAs in the work-queue
        form (AUTO, QUEUE) or one per walker (STATIC)."""
        self.lib.call('walkers_set_schedule', self.h, mode, unit_moves, ctas)

    def evaluate_ratios(self, walker, iat, pos):
        """WaveFunction::evaluateRatios: one walker's ratios of electron iat
        at absolute positions pos[n][3]."""
        p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        r = np.zeros(len(p))
        self.lib.call('wf_evaluate_ratios', self.h, walker, iat, len(p), _pd(p), _pd(r))
        return r

    def accept_restore(self, iat, accept):
        a = np.ascontiguousarray(accept, dtype=np.int32)
        self.lib.call('wf_accept_restore', self.h, iat, _pi(a))

    def complete_updates(self):
        self.lib.call('wf_complete_updates', self.h)

    def step(self, iat, accept, ur, delta):
        """qmc_step: the fused move of electron iat for every walker; returns
        the accept flags [W]."""
        u = np.ascontiguousarray(ur, dtype=np.float64).reshape(self.W)
        d = np.ascontiguousarray(delta, dtype=np.float64).reshape(self.W, 3)
        acc = np.zeros(self.W, dtype=np.int32)
        self.lib.call('step', self.h, iat, accept, _pd(u), _pd(d), _pi(acc))
        return acc

    def evaluate_gl(self):
        G = np.zeros((self.W, self.N, 3))
        L = np.zeros((self.W, self.N))
        lp = np.zeros(self.W)
        self.lib.call('wf_evaluate_gl', self.h, _pd(G), _pd(L), _pd(lp))
        return G, L, lp

    def local_kinetic(self):
        ke = np.zeros(self.W)
        self.lib.call('local_kinetic', self.h, _pd(ke))
        return ke

    def checkpoint(self):
        """The batch's persistent state as bytes (qmc_walkers_checkpoint)."""
        n = C.c_size_t()
        self.lib.call('walkers_checkpoint_bytes', self.h, C.byref(n))
        buf = (C.c_ubyte * n.value)()
        self.lib.call('walkers_checkpoint', self.h, C.cast(buf, C.c_void_p), n)
        return bytes(buf)

    def restore(self, data):
        buf = (C.c_ubyte * len(data)).from_buffer_copy(data)
        self.lib.call('walkers_restore', self.h, C.cast(buf, C.c_void_p), C.c_size_t(len(data)))

    def nlpp(self, rmax=1.7, form=capi.NLPP_SPHERE, max_ratios=0):
        """NonLocalPP ratios (qmc_nlpp_evaluate): (n_points[W], wsum[W],
        walker 0's ratios or None)."""
        n = np.zeros(self.W, dtype=np.int64)
        ws = np.zeros(self.W)
        r = np.zeros(max_ratios) if max_ratios else None
        self.lib.call('nlpp_evaluate', self.h, rmax, form, n.ctypes.data_as(C.POINTER(C.c_int64)), _pd(ws),
                      _pd(r) if r is not None else None, max_ratios)
        return n, ws, r

    def components(self):
        c = np.zeros((self.W, 7))
        self.lib.call('wf_components', self.h, _pd(c))
        return c

    def inverse(self, walker, spin):
        n = self.sys.spec.n_orb
        m = np.zeros((n, n))
        self.lib.call('wf_get_inverse', self.h, walker, spin, _pd(m))
        return m

    def sweep(self, n_steps=1, n_substeps=1, accept=0.5, ur=None, delta=None, recompute_every=0,
              trace=False):
        o = capi.SweepOpts()
        o.n_steps = n_steps
        o.n_substeps = n_substeps
        o.accept = accept
        keep = []
        if ur is not None:
            o.rng_mode = capi.RNG_HOST
            ur = np.ascontiguousarray(ur, dtype=np.float64)
            delta = np.ascontiguousarray(delta, dtype=np.float64)
            keep += [ur, delta]
            o.ur = _pd(ur)
            o.delta = _pd(delta)
        else:
            o.rng_mode = capi.RNG_DEVICE
        o.recompute_every = recompute_every
        tr = None
        if trace:
            tr = np.zeros((n_steps, self.W, n_substeps, self.N, 8))
            o.trace = _pd(tr)
        acc = np.zeros(self.W, dtype=np.int64)
        lp = np.zeros(self.W)
        o.n_accepted = acc.ctypes.data_as(C.POINTER(C.c_int64))
        o.logpsi = _pd(lp)
        self.lib.call('sweep', self.h, C.byref(o))
        return dict(accepted=acc, logpsi=lp, trace=tr)


class DetEngine:
    """DelayedUpdate + DiracMatrix on one n x n inverse (DelayedUpdate.h:28-231)."""

    def __init__(self, lib, n, delay, precision=None):
        self.lib = lib
        self.n = n
        h = C.c_void_p()
        if precision is None:
            lib.call('detengine_create', n, delay, C.byref(h))
        else:
            lib.call('detengine_create_prec', n, delay, precision, C.byref(h))
        self.h = h

    def close(self):
        if self.h:
            self.lib.call('detengine_destroy', self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def invert_transpose(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        lg, ph = C.c_double(), C.c_double()
        self.lib.call('detengine_invert_transpose', self.h, _pd(a), C.byref(lg), C.byref(ph))
        return lg.value, ph.value

    def get_inv_row(self, row):
        r = np.zeros(self.n)
        self.lib.call('detengine_get_inv_row', self.h, row, _pd(r))
        return r

    def accept_row(self, row, psiv):
        p = np.ascontiguousarray(psiv, dtype=np.float64)
        self.lib.call('detengine_accept_row', self.h, row, _pd(p))

    def update_inv_mat(self):
        self.lib.call('detengine_update_inv_mat', self.h)

    def ainv(self):
        m = np.zeros((self.n, self.n))
        self.lib.call('detengine_get_ainv', self.h, _pd(m))
        return m


class Group:
    """Several walker batches (possibly of different systems) advanced by one
    fused launch per MC step (qmc_group_*)."""

    def __init__(self, lib, batches):
        self.lib = lib
        self.batches = list(batches)
        arr = (C.c_void_p * len(self.batches))(*[b.h.value if isinstance(b.h, C.c_void_p) else b.h
                                                  for b in self.batches])
        h = C.c_void_p()
        lib.call('group_create', arr, len(self.batches), C.byref(h))
        self.h = h

    def close(self):
        if self.h:
            self.lib.call('group_destroy', self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_threads(self, threads):
        self.lib.call('group_set_threads', self.h, threads)

    def use_graph(self, enable=True):
        self.lib.call('group_use_graph', self.h, 1 if enable else 0)

    def set_schedule(self, mode=capi.SCHED_AUTO, unit_moves=0, ctas=0):
        self.lib.call('group_set_schedule', self.h, mode, unit_moves, ctas)

    def sweep(self, n_steps=1, n_substeps=1, accept=0.5, recompute_every=0):
        self.lib.call('group_sweep', self.h, n_steps, n_substeps, accept, recompute_every)

    def sync(self):
        self.lib.call('group_sync', self.h)

    def stream(self):
        s = C.c_void_p()
        self.lib.call('group_stream', self.h, C.byref(s))
        return s.value

    def stats(self):
        t, l, gl = C.c_int(), C.c_int64(), C.c_int64()
        self.lib.call('group_stats', self.h, C.byref(t), C.byref(l), C.byref(gl))
        return dict(threads=t.value, launches=l.value, graph_launches=gl.value)


def autotune(lib, system, n_walkers, delays=(8, 16, 32), n_steps=2):
    """qmc_autotune: (best, all) as dicts."""
    d = (C.c_int * len(delays))(*delays)
    res = (capi.TuneResult * 64)()
    n = C.c_int()
    best = capi.TuneResult()
    lib.call('autotune', system.h, n_walkers, d, len(delays), n_steps, res, 64, C.byref(n), C.byref(best))

    def as_dict(r):
        return dict(delay=r.delay, threads=r.threads, tensor_cores=r.tensor_cores, max_moves=r.max_moves,
                    ms_per_step=r.ms_per_step)
    return as_dict(best), [as_dict(res[i]) for i in range(min(n.value, 64))]


class Server:
    """The request loop (qmc_server_*): jobs admitted by device footprint,
    every running job's walkers moved by one shared launch per tick."""

    def __init__(self, lib, memory_budget, threads=128, recompute_every=0):
        self.lib = lib
        h = C.c_void_p()
        lib.call('server_create', C.c_size_t(int(memory_budget)), threads, recompute_every, C.byref(h))
        self.h = h

    def close(self):
        if self.h:
            self.lib.call('server_destroy', self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, system, n_walkers, n_steps, delay, seed):
        j = C.c_int64()
        self.lib.call('server_submit', self.h, system.h, n_walkers, n_steps, delay, C.c_uint32(seed), C.byref(j))
        return j.value

    def tick(self):
        r, w = C.c_int(), C.c_int()
        self.lib.call('server_tick', self.h, C.byref(r), C.byref(w))
        return r.value, w.value

    def job(self, job_id):
        info = capi.JobInfo()
        self.lib.call('server_job', self.h, C.c_int64(job_id), C.byref(info))
        return dict(state=info.state, status=info.status, steps_done=info.steps_done, n_accepted=info.n_accepted,
                    logpsi_mean=info.logpsi_mean, t_submit=info.t_submit, t_start=info.t_start, t_done=info.t_done)

    def stats(self):
        b, l, m = C.c_size_t(), C.c_int64(), C.c_int64()
        self.lib.call('server_stats', self.h, C.byref(b), C.byref(l), C.byref(m))
        return dict(bytes_in_use=b.value, launches=l.value, electron_moves=m.value)
