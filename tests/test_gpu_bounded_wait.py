"""Failure detection without a GPU fault: the tensor-core kernels wait on
mbarriers with a time limit and report a timeout instead of hanging.  Here the
wait is made to run out on purpose (an mbarrier that nothing completes, 20 ms
limit); the kernel must give up, return, and leave the context usable."""
import numpy as np
import pytest

import kfvm_abi as abi

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_survives(product_lib, gpu):
    import kfvm
    gave_up, waited = kfvm.selftest_wait(0.02)
    assert gave_up
    assert 0.02 <= waited < 0.5, waited
    # the context still runs the tensor-core path afterwards
    cfg, ic = abi.workload("isentropic_vortex", scale=32, steps=2)
    s = kfvm.Solver(cfg)
    s.set_precision(abi.KFVM_PREC_TF32X3)
    s.init_ic(ic)
    info = s.take_step()
    assert info.accepted == 1 and np.isfinite(s.get_state()).all()
    s.close()


def test_bounded_wait_arguments(product_lib, gpu):
    import kfvm
    with pytest.raises(kfvm.KfvmError):
        kfvm.selftest_wait(0.0)
    with pytest.raises(kfvm.KfvmError):
        kfvm.selftest_wait(5.0)
