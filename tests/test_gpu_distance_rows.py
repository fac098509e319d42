"""Distance rows on the GPU against the reference's own values.

qmc_pset_get_temp_rows returns the temporary AA and AB rows of the active
move (DistanceTableAA::move / DistanceTableBA::move, DistanceTableAA.h:85-95,
DistanceTableBA.h:83-97) computed by the device's minimum-image code (reduced
basis, -floor wrap, 8-corner search, the sign flip from the active index on:
ParticleBConds.h:153-217).  The golden rows were printed by the reference's
own ParticleSet / DTD_BConds code on its 32-atom NiO cell
(tests/golden/reference_dump.json): the row of electron 5 after setActive(5)
and the temp rows of makeMove(7, (0.3, -0.7, 1.1))."""
import json
import os

import numpy as np
import pytest

from miniqmc_b200 import api, capi
from tests import gpu_helpers as H
from tests import oracle_lib

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(oracle_lib.GOLDEN, 'reference_dump.json')))
REJECT = np.zeros(2, dtype=np.int32)


def close(a, b, rtol=1e-12, atol=1e-12):
    np.testing.assert_allclose(np.asarray(a, dtype=float), np.asarray(b, dtype=float), rtol=rtol, atol=atol)


def _walkers(lib, seeds):
    spec = api.SystemSpec(lib, cell=capi.NIO_REF32, tiling=(1, 1, 1),
                          quirks=capi.NIO_QUIRK_UNIT_IONS | capi.NIO_QUIRK_ONE_GROUP, grid=(8, 8, 8),
                          fill=capi.FILL_REFERENCE, jastrow='reference', components=capi.WF_J1 | capi.WF_J2)
    system = api.System(lib, spec, capi.PREC_FP64)
    w = api.Walkers(system, len(seeds), 1)
    w.init_random(np.array(seeds, dtype=np.uint32))
    return spec, system, w


def test_temp_rows_match_reference_dump():
    spec, system, w = _walkers(H.product(), [3, 5])
    R = w.positions()
    close(R[0].ravel(), GOLD['els_111_p0'])
    # makeMove(7, d): the temp rows of the AA and AB tables
    w.make_move(7, np.array([[0.3, -0.7, 1.1], [0.3, -0.7, 1.1]]))
    aa_r, aa_dr, ab_r, ab_dr = w.temp_rows()
    close(aa_r[0], GOLD['aa_move7_r'])
    close(aa_dr[0].ravel(), GOLD['aa_move7_dr'])
    close(ab_r[0], GOLD['ab_move7_r'])
    close(ab_dr[0].ravel(), GOLD['ab_move7_dr'])
    w.accept_reject(7, REJECT)
    # setActive(5)'s row: electron 5 at its current position, flip index 5;
    # the table's diagonal holds max T (dumped as -1), the temp row a 0
    w.make_move(5, np.zeros((2, 3)))
    aa_r, aa_dr, _, _ = w.temp_rows()
    gold_r = np.array(GOLD['aa_row5_r'])
    keep = np.arange(spec.n_elec) != 5
    close(aa_r[0][keep], gold_r[keep])
    close(aa_dr[0].ravel(), GOLD['aa_row5_dr'])
    assert aa_r[0][5] == 0.0
    w.accept_reject(5, REJECT)
    w.close()
    system.close()


def test_temp_rows_second_walker_and_sign_contract():
    """Walker 1 (another stream) against the oracle's rows, and the
    displacement sign contract dr_ij = -dr_ji of the flip: entry j of i's
    row (i at rest) against entry i of j's row (j at rest)."""
    _, s_g, wg = _walkers(H.product(), [3, 5])
    _, s_o, wo = _walkers(H.oracle(), [3, 5])
    d = np.array([[0.0, 0.0, 0.0], [-0.4, 0.25, 0.9]])
    for w in (wg, wo):
        w.make_move(11, d)
    rg, ro = wg.temp_rows(), wo.temp_rows()
    for a, b in zip(rg, ro):
        close(a[1], b[1])
    wg.accept_reject(11, REJECT)
    wo.accept_reject(11, REJECT)
    wg.make_move(11, np.zeros((2, 3)))
    r11, dr11, _, _ = wg.temp_rows()
    wg.accept_reject(11, REJECT)
    wg.make_move(20, np.zeros((2, 3)))
    r20, dr20, _, _ = wg.temp_rows()
    wg.accept_reject(20, REJECT)
    close(r11[:, 20], r20[:, 11])
    close(dr11[:, 20], -dr20[:, 11])
    for w, s in ((wg, s_g), (wo, s_o)):
        w.close()
        s.close()
