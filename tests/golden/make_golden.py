"""Regenerate the golden fixtures in tests/golden from the reference.

Run where the reference source tree is (its root given by --reference or the
MINIQMC_REFERENCE environment variable); the GPU runs do not need it because
the fixtures are committed.  Two sources:

1. reference_dump.json -- output of oracle/_ref/ref_harness, which is built by
   oracle/ref_harness.mk from the reference's own ParticleSet, distance-table,
   lattice, einspline SPO, BsplineFunctor, One/TwoBodyJastrow, StdRandom and
   NiO-input code (FP64, no fast-math); reference_det_dump.json -- output of
   oracle/_ref/ref_det_harness: the reference's DiracDeterminant /
   DelayedUpdate / DiracMatrix over OpenBLAS on a well-conditioned table.
2. known_answers.json -- the numbers the reference's Catch unit tests assert,
   read from the test sources as text:
     src/QMCWaveFunctions/tests/test_dirac_matrix.cpp  (3x3 inverse, log|det|,
       rank-1 row update ratio and updated inverse)
     src/QMCWaveFunctions/tests/test_dirac_det.cpp     (FakeSPO matrices used
       for sequential rank-1 and delay-2 updates)
     src/Particle/tests/test_particle.cpp               (PBC AA distance)
     src/Utilities/tests/test_PrimeNumberSet.cpp        (primes)

Usage:  python tests/golden/make_golden.py [--reference <reference root>]
"""
import argparse
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _test_case_blocks(text):
    parts = re.split(r'TEST_CASE\("([^"]+)"', text)
    return {parts[i]: parts[i + 1] for i in range(1, len(parts), 2)}


def _matrix_assignments(block):
    """Collect `name(i, j) = value;` and `name[i] = value;` in source order."""
    out = {}
    for m in re.finditer(r'(\w+)\((\d+),\s*(\d+)\)\s*=\s*([-+0-9.eE]+)\s*;', block):
        out.setdefault(m.group(1), []).append((int(m.group(2)), int(m.group(3)), float(m.group(4))))
    for m in re.finditer(r'(\w+)\[(\d+)\]\s*=\s*([-+0-9.eE]+)\s*;', block):
        out.setdefault(m.group(1), []).append((int(m.group(2)), float(m.group(3))))
    return out


def _dense(entries, rows, cols):
    a = [[0.0] * cols for _ in range(rows)]
    for i, j, v in entries:
        a[i][j] = v
    return a


def known_answers(ref):
    src = os.path.join(ref, 'src')
    ka = {}
    txt = open(os.path.join(src, 'QMCWaveFunctions/tests/test_dirac_matrix.cpp')).read()
    blocks = _test_case_blocks(txt)
    inv = _matrix_assignments(blocks['DiracMatrix_inverse'])
    ka['dm_a'] = _dense(inv['a'], 3, 3)
    ka['dm_a_inv'] = _dense(inv['b'], 3, 3)
    ka['dm_logdet'] = float(re.search(r'LogValue == ValueApprox\(([-0-9.eE]+)\)',
                                      blocks['DiracMatrix_inverse']).group(1))
    upd = blocks['DiracMatrix_update_row']
    ua = _matrix_assignments(upd)
    ka['dm_update_v'] = [v for _, v in sorted(ua['v'])]
    ka['dm_update_ratio'] = float(re.search(r'det_ratio = ([-0-9.eE]+);', upd).group(1))
    ka['dm_update_inv'] = _dense(ua['b'], 3, 3)

    txt = open(os.path.join(src, 'QMCWaveFunctions/tests/test_dirac_det.cpp')).read()
    ctor = txt[txt.index('FakeSPO::FakeSPO()'):txt.index('void FakeSPO::setOrbitalSetSize')]
    fs = _matrix_assignments(ctor)
    ka['fake_a'] = _dense(fs['a'], 3, 3)
    ka['fake_v'] = [v for _, v in sorted(fs['v'])]
    ka['fake_a2'] = _dense(fs['a2'], 4, 4)
    ka['fake_v2'] = _dense(fs['v2'], 3, 4)
    first = _test_case_blocks(txt)['DiracDeterminant_first']
    fb = _matrix_assignments(first)['b']
    ka['det_first_inv'] = _dense(fb[:9], 3, 3)
    ka['det_first_ratio'] = float(re.search(r'det_ratio1 = ([-0-9.eE]+);', first).group(1))
    ka['det_first_updated_inv'] = _dense(fb[9:], 3, 3)

    txt = open(os.path.join(src, 'Particle/tests/test_particle.cpp')).read()
    m = re.search(r'grid\.R = ParticleSet::Tensor_t\(([^)]*)\)', txt, re.S)
    ka['pbc_lattice'] = [float(x) for x in m.group(1).replace('\n', ' ').split(',')]
    ka['pbc_R'] = [[float(x) for x in g.split(',')]
                   for g in re.findall(r'source\.R\[\d\] = ParticleSet::PosType\(([^)]*)\)', txt)]
    ka['pbc_dist_12'] = float(re.search(r'Distances\[1\]\[2\] == Approx\(([-0-9.eE]+)\)', txt).group(1))
    ka['pbc_displ_12'] = [float(x) for x in re.findall(
        r'Displacements\[1\]\[2\]\[\d\] == Approx\(([-0-9.eE]+)\)', txt)]
    ka['pbc_displ_21'] = [float(x) for x in re.findall(
        r'Displacements\[2\]\[1\]\[\d\] == Approx\(([-0-9.eE]+)\)', txt)]

    txt = open(os.path.join(src, 'Utilities/tests/test_PrimeNumberSet.cpp')).read()
    ka['primes_checked'] = [[int(i), int(v)] for i, v in
                            re.findall(r'myPrimes\[(\d+)\] == (\d+)', txt)]
    ka['_sources'] = {
        'dm_*': 'src/QMCWaveFunctions/tests/test_dirac_matrix.cpp:69-160',
        'fake_*, det_first_*': 'src/QMCWaveFunctions/tests/test_dirac_det.cpp:75-248',
        'pbc_*': 'src/Particle/tests/test_particle.cpp:31-61',
        'primes_checked': 'src/Utilities/tests/test_PrimeNumberSet.cpp',
    }
    return ka


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', default=os.environ.get('MINIQMC_REFERENCE'),
                    help='root of the reference source tree (default: $MINIQMC_REFERENCE)')
    args = ap.parse_args()
    if not args.reference or not os.path.isdir(os.path.join(args.reference, 'src')):
        sys.exit('reference tree not found: pass --reference or set MINIQMC_REFERENCE')
    subprocess.check_call(['make', '-s', '-f', os.path.join(REPO, 'oracle', 'ref_harness.mk'),
                           'MINIQMC_REFERENCE=%s' % args.reference])
    dump = subprocess.check_output([os.path.join(REPO, 'oracle', '_ref', 'ref_harness')])
    dump = json.loads(dump)
    dump['_generator'] = 'oracle/ref_harness.cpp compiled from the reference sources'
    with open(os.path.join(HERE, 'reference_dump.json'), 'w') as f:
        json.dump(dump, f)
    # the determinant path (DiracDeterminant + DelayedUpdate + DiracMatrix
    # over OpenBLAS) on a well-conditioned table, delay ranks 1 and 32
    det = subprocess.check_output([os.path.join(REPO, 'oracle', '_ref', 'ref_det_harness')],
                                  env=dict(os.environ, OPENBLAS_NUM_THREADS='1'))
    with open(os.path.join(HERE, 'reference_det_dump.json'), 'w') as f:
        json.dump(json.loads(det), f)
    with open(os.path.join(HERE, 'known_answers.json'), 'w') as f:
        json.dump(known_answers(args.reference), f, indent=1)
    print('wrote', os.path.join(HERE, 'reference_dump.json'), 'and known_answers.json')


if __name__ == '__main__':
    main()
