"""The CPU oracle's determinant path (DelayedUpdate at delay ranks 1 and 32,
the FP64 inverse, DiracDeterminant's ratios, gradients and log|det|) against
the reference's own code on a well-conditioned table (tests/det_golden.py).
CPU only."""
import pytest

from tests import det_golden, oracle_lib


@pytest.mark.parametrize('delay', [1, 32])
def test_oracle_matches_reference_determinant(delay):
    det_golden.check(oracle_lib.library(), delay)
