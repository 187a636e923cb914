"""C-ABI checks that need no GPU: the library loads and exports every entry point
declared in include/kfvm_b200.h, the host weight precompute matches the oracle
bit for bit, and configuration errors are reported without touching a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import kfvm_abi as abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "kfvm_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(kfvm_[a-z_0-9]+)\s*\(", text)))


def test_exports_every_declared_symbol(product_lib):
    L = product_lib.lib()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n


WORKLOADS = ["isentropic_vortex", "sod3d", "kelvin_helmholtz", "taylor_green", "orszag_tang"]


@pytest.mark.parametrize("name", WORKLOADS)
def test_weights_bitwise_equal_oracle(name, product_lib, oracle_lib):
    cfg, _ = abi.workload(name, scale=24)
    a = product_lib.stencil(cfg)
    b = oracle_lib.stencil(cfg)
    assert bytes(a) == bytes(b)


@pytest.mark.parametrize("lfac", [2.0, 5.0, 20.0])
@pytest.mark.parametrize("dim", [2, 3])
def test_weights_other_lfac(dim, lfac, product_lib, oracle_lib):
    cfg, _ = abi.workload("isentropic_vortex" if dim == 2 else "sod3d", scale=16)
    cfg.lfac = lfac
    assert bytes(product_lib.stencil(cfg)) == bytes(oracle_lib.stencil(cfg))


def test_default_config(product_lib):
    c = abi.KfvmConfig()
    product_lib.lib().kfvm_default_config(C.byref(c))
    d = abi.default_config()
    for f, _ in abi.KfvmConfig._fields_:
        if f in ("bc", "cfl"):
            continue
        a, b = getattr(c, f), getattr(d, f)
        if f in ("nb", "block"):
            a, b = list(a), list(b)
        assert a == b, f


@pytest.mark.parametrize("mutate,msg", [
    (lambda c: setattr(c, "dim", 4), "dim"),
    (lambda c: setattr(c, "nq", 4), "NUM_QUAD_PTS"),
    # three points in 3D for every system but SR
    (lambda c: (setattr(c, "dim", 3), setattr(c, "nz", 16), setattr(c, "nq", 3), setattr(c, "eq", abi.KFVM_EQ_SRHYDRO),
                setattr(c, "rs", abi.KFVM_RS_HLL)), "NUM_QUAD_PTS"),
    (lambda c: (c.bc.__setitem__(0, 6), c.bc.__setitem__(1, 6)), "unknown boundary"),
    (lambda c: (setattr(c, "eq", abi.KFVM_EQ_MHD_GLM), setattr(c, "rs", abi.KFVM_RS_HLLC)), "HLLC"),
    (lambda c: (setattr(c, "eq", abi.KFVM_EQ_SRHYDRO), setattr(c, "rs", abi.KFVM_RS_HLLC)), "HLL and LLF"),
    (lambda c: (setattr(c, "eq", abi.KFVM_EQ_SRHYDRO), setattr(c, "rs", abi.KFVM_RS_HLL),
                setattr(c, "indicator", abi.KFVM_IND_MLP)), "learned"),
    (lambda c: setattr(c, "eq", 4), "equation"),
    (lambda c: c.bc.__setitem__(1, abi.KFVM_BC_OUTFLOW), "pairs"),
    (lambda c: setattr(c, "rk", 9), "RK"),
    (lambda c: setattr(c, "nx", 2), "small"),
])
def test_create_rejects_bad_config(mutate, msg, product_lib):
    cfg, _ = abi.workload("kelvin_helmholtz", scale=16)
    mutate(cfg)
    with pytest.raises(product_lib.KfvmError, match=msg):
        product_lib.Solver(cfg)


def test_stof_rounding():
    """Reals from an .init file are rounded through float as std::stof does."""
    cfg, _ = abi.workload("isentropic_vortex", scale=8)
    assert cfg.gamma == float(np.float32(1.4)) != 1.4
    assert cfg.cfl == float(np.float32(0.8))
