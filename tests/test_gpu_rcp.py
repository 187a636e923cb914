"""The FP64 reciprocal of the Riemann solvers (Newton-Raphson refinement of the
hardware approximation, physics.cuh rcp_nr) against CUDA's IEEE reciprocal and
quotient over random doubles of both signs and exponents in [-300, 300]."""
import os
import sys

import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "kfvm-kokkos_b200"))


@pytest.mark.gpu
def test_rcp_within_one_ulp():
    import kfvm
    max_ulp, max_rel = kfvm.selftest_rcp(1 << 24, seed=5)
    # the refined reciprocal is within one ulp of the correctly rounded 1/y, so
    # x * rcp(y) is within about 1.5 ulp (2^-53 = 1.1e-16 relative) of x / y
    assert max_ulp <= 1, max_ulp
    assert max_rel <= 2.5e-16, max_rel
