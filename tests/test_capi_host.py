"""CPU-only checks of the product C ABI: the library builds for sm_100a,
loads, exports every entry point include/qmcgpu.h declares, and its host-side
builders (NiO input, functors, Wigner-Seitz radius, synthetic Jastrows)
agree with the oracle.  No CUDA device is touched."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from miniqmc_b200 import api, capi
from tests import oracle_lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, 'include', 'qmcgpu.h')


@pytest.fixture(scope='module')
def prod():
    from miniqmc_b200 import build
    build.build()
    return api.Library()


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r'/\*.*?\*/', '', txt, flags=re.S)
    return sorted(set(re.findall(r'\b(qmc_\w+)\s*\(', txt)))


def test_header_symbols_exported(prod):
    names = declared_functions()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(prod.lib, n)]
    assert not missing, missing


def test_status_strings(prod):
    prod.lib.qmc_status_string.restype = C.c_char_p
    assert prod.lib.qmc_status_string(4) == b'QMC_ERR_SINGULAR'


@pytest.mark.parametrize('cell,tiling,quirks', [(capi.NIO_REF32, (1, 1, 1), 3), (capi.NIO_REF32, (2, 1, 1), 3),
                                                (capi.NIO_REF32, (1, 1, 2), 0), (capi.NIO_PRIM4, (2, 2, 1), 0),
                                                (capi.NIO_PRIM4, (4, 4, 2), 0)])
def test_nio_builder_matches_oracle(prod, cell, tiling, quirks):
    orc = oracle_lib.library()
    a = prod.nio(cell, tiling, quirks)
    b = orc.nio(cell, tiling, quirks)
    for k in ('lattice', 'ion_pos', 'spo_lattice'):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(a['ion_group'], b['ion_group'])
    assert prod.ws_radius(a['lattice']) == orc.ws_radius(b['lattice'])


def test_prim4_is_reference_tiling(prod):
    """The 4-atom cell tiled 2x2x2 is the reference's 32-atom cell: same
    lattice and the same set of sites (the site order differs)."""
    a = prod.nio(capi.NIO_PRIM4, (2, 2, 2))
    b = prod.nio(capi.NIO_REF32, (1, 1, 1))
    assert np.allclose(a['lattice'], b['lattice'])
    G = np.linalg.inv(a['lattice'].reshape(3, 3))
    ua = np.round((a['ion_pos'] @ G) % 1.0, 9) % 1.0
    ub = np.round((b['ion_pos'] @ G) % 1.0, 9) % 1.0
    sa = sorted(map(tuple, np.c_[ua, a['ion_group']]))
    sb = sorted(map(tuple, np.c_[ub, b['ion_group']]))
    assert np.allclose(np.array(sa), np.array(sb))


def test_functors_and_jastrows_match_oracle(prod):
    orc = oracle_lib.library()
    lat = prod.nio(capi.NIO_REF32, (1, 1, 1), 3)['lattice']
    ja, jb = prod.nio_jastrows(lat), orc.nio_jastrows(lat)
    for fa, fb in [(ja['j2_uu'], jb['j2_uu']), (ja['j2_ud'], jb['j2_ud']), (ja['j1'][0], jb['j1'][0]),
                   (ja['j1'][1], jb['j1'][1])]:
        assert fa.n_coefs == fb.n_coefs and fa.cutoff == fb.cutoff and fa.delta_r_inv == fb.delta_r_inv
        assert list(fa.coefs) == list(fb.coefs)


def test_j3_functors_match_reference(prod):
    """The product's PolynomialFunctor3D::reset_gamma restatement and its
    buildJeeI tables against the gammas the reference printed, on two cells
    (the reference's 32-atom cell and the 4x4x2 NiO-128 cell)."""
    import json
    gold = json.load(open(os.path.join(oracle_lib.GOLDEN, 'reference_dump.json')))
    lat = prod.nio(capi.NIO_REF32, (1, 1, 1), 3)['lattice']
    j3 = prod.nio_j3(lat)
    assert j3['same'][0].cutoff == gold['j3_rcut']
    for key, f in (('j3_gamma_uu0', j3['same'][0]), ('j3_gamma_ud0', j3['diff'][0]),
                   ('j3_gamma_uu1', j3['same'][1]), ('j3_gamma_ud1', j3['diff'][1])):
        np.testing.assert_allclose(list(f.gamma), gold[key], rtol=1e-12, atol=1e-15)
    orc = oracle_lib.library()
    lat = prod.nio(capi.NIO_PRIM4, (4, 4, 2), 0)['lattice']
    ja, jb = prod.nio_j3(lat), orc.nio_j3(lat)
    for s in range(2):
        for kind in ('same', 'diff'):
            assert ja[kind][s].cutoff == jb[kind][s].cutoff
            np.testing.assert_allclose(list(ja[kind][s].gamma), list(jb[kind][s].gamma), rtol=1e-12, atol=1e-15)


def test_synthetic_jastrows_c_equals_python(prod):
    lat = prod.nio(capi.NIO_PRIM4, (2, 2, 1))['lattice']
    py = api.synthetic_jastrows(prod, lat, 2, 13, 8)
    j1 = (capi.Functor * 4)()
    uu, ud = capi.Functor(), capi.Functor()
    latc = np.ascontiguousarray(lat)
    fn = prod.lib.qmc_synthetic_jastrows
    fn.argtypes = [capi.PD, C.c_int, C.c_uint64, C.c_int, C.POINTER(capi.Functor), C.POINTER(capi.Functor),
                   C.POINTER(capi.Functor)]
    assert fn(latc.ctypes.data_as(capi.PD), 2, 13, 8, j1, C.byref(uu), C.byref(ud)) == 0
    assert list(uu.coefs) == list(py['j2_uu'].coefs)
    assert list(ud.coefs) == list(py['j2_ud'].coefs)
    assert list(j1[1].coefs) == list(py['j1'][1].coefs)


def test_splitmix_python_equals_oracle():
    orc = oracle_lib.library()
    for i in (0, 1, 17, 123456789):
        assert api.splitmix_uniform(11, i) == orc.fn['splitmix_uniform'](11, i)


def test_nlpp_spheres_match_reference(prod):
    """The product's host-side NonLocalPP sphere stream (no GPU needed)."""
    import json
    import os
    gold = json.load(open(os.path.join(os.path.dirname(__file__), 'golden', 'reference_dump.json')))
    out = np.zeros(3 * 36)
    prod.call('nlpp_sphere', 3, out.ctypes.data_as(capi.PD))
    np.testing.assert_allclose(out, np.array(gold['nlpp_spheres']), rtol=0, atol=1e-15)
