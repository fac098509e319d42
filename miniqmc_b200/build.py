"""Build libqmcgpu.so in-tree with nvcc for sm_100a, and the miniqmc driver.

    python miniqmc_b200/build.py [--force] [--verbose]

Each .cu under miniqmc_b200/csrc compiles to an object in miniqmc_b200/_build
(in parallel); the objects link into miniqmc_b200/libqmcgpu.so with the CUDA
runtime linked statically, so the library needs only the driver at run time.
miniqmc_b200/drivers/*.cpp (the miniqmc command-line driver on the C ABI)
build with g++ into miniqmc_b200/bin/, linked against the in-tree library.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
BUILD = os.path.join(HERE, '_build')
LIB = os.path.join(HERE, 'libqmcgpu.so')
DRIVERS = os.path.join(HERE, 'drivers')
BIN = os.path.join(HERE, 'bin')
CXX = os.environ.get('CXX', '/usr/bin/g++')
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr',
         '-Xcudafe', '--diag_suppress=177']


def _deps():
    return [os.path.join(HERE, '..', 'include', 'qmcgpu.h')] + glob.glob(os.path.join(CSRC, '*.cuh')) + \
        glob.glob(os.path.join(CSRC, '*.hpp'))


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(force=False, verbose=False, extra_flags=()):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, '*.cu')))
    deps = _deps()
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + '.o')
        objs.append(o)
        if force or _stale(o, [s] + deps):
            cmd = [NVCC] + ARCH + FLAGS + list(extra_flags) + ['-c', s, '-o', o]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(' '.join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, r in ex.map(run, jobs):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError('nvcc failed: %s' % os.path.basename(cmd[-3]))
            if verbose and (r.stderr.strip()):
                sys.stderr.write(r.stderr)
    if force or jobs or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ['-shared', '-o', LIB] + objs + ['-cudart', 'static']
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError('link failed')
    build_drivers(force)
    return LIB


def build_drivers(force=False):
    """Command-line drivers over the C ABI (no CUDA headers needed)."""
    os.makedirs(BIN, exist_ok=True)
    include = os.path.join(HERE, '..', 'include')
    for src in sorted(glob.glob(os.path.join(DRIVERS, '*.cpp'))):  # driver_common.hpp is a header
        exe = os.path.join(BIN, os.path.basename(src)[:-4])
        if not force and not _stale(exe, [src, LIB, os.path.join(include, 'qmcgpu.h'),
                                          os.path.join(DRIVERS, 'driver_common.hpp')]):
            continue
        cmd = [CXX, '-O2', '-std=c++17', '-I', include, src, '-L', HERE, '-lqmcgpu',
               '-Wl,-rpath,$ORIGIN/..', '-o', exe]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError('driver build failed: %s' % os.path.basename(src))


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--force', action='store_true')
    ap.add_argument('--verbose', action='store_true')
    a = ap.parse_args()
    print(build(a.force, a.verbose))
