"""The product's FP64 determinant path (the fused sweep's getInvRow,
acceptRow and Woodbury flush at delay ranks 1 and 32, the FP64 Gauss-Jordan
inverse, the ratios, gradients and log|det|) against the reference's own
DiracDeterminant / DelayedUpdate / DiracMatrix on a well-conditioned table
(tests/det_golden.py)."""
import pytest

from tests import det_golden
from tests import gpu_helpers as H

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('delay', [1, 32])
def test_product_matches_reference_determinant(delay):
    det_golden.check(H.product(), delay)
