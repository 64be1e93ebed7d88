"""The pybind11 module `my_module` (ip_cu_lbm_b200/pybind/my_module.cpp): the
reference prototype's Python boundary (ref: pybind_LockExchange/run.py:1-13,
wrapper.cpp:11-61) working, plus the LockExchange stepping class."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(HERE), "ip_cu_lbm_b200")


def _mod():
    if PKG not in sys.path:
        sys.path.insert(0, PKG)
    import my_module

    return my_module


def test_module_imports_and_exposes_the_api():
    m = _mod()
    assert {"GPUMemory", "compute_on_gpu", "LockExchange"} <= set(dir(m))


@pytest.mark.gpu
def test_run_py_semantics(cuda):
    m = _mod()
    arr = np.arange(10, dtype=np.float32)
    mem = m.GPUMemory(10)
    assert mem.size() == 10
    mem.set(arr)
    m.compute_on_gpu(mem)
    np.testing.assert_array_equal(mem.get(), arr + 5.0)
    with pytest.raises(RuntimeError):
        mem.set(np.zeros(3, np.float32))


@pytest.mark.gpu
def test_lockexchange_class_matches_sim(cuda):
    from ip_cu_lbm_b200 import Sim

    m = _mod()
    nx, nz = 96, 32
    S0 = (np.arange(nx)[None, :] < nx // 2) * np.ones((nz, 1), float)
    a = m.LockExchange(nx=nx, nz=nz, q_scalar=5, geometry="uniform", wall="bb", mrt=False, g_bouss=1e-4,
                       rho_sal=1e-4, tau=0.53, taus=0.503, s0=S0.ravel().tolist())
    b = Sim(nx, nz, q_scalar=5, geometry="uniform", wall="bb", mrt=False, g_bouss=1e-4, rho_sal=1e-4, tau=0.53,
            taus=0.503, s0=S0.ravel())
    a.step(25)
    b.step(25)
    for fld in ("S", "ux", "uz"):
        assert np.array_equal(a.get(fld), b.get(fld)), fld
    assert a.cells() == nx * nz
