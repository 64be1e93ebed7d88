"""ORACLE -- test infrastructure only (tests/, __graft_entry__.smoke(),
bench.py's cpu_baseline / reference legs). Never imported by the product.

Bindings of
  * the CPU restatement of the reference kernels (oracle/_build/libipcu_oracle.so,
    built from oracle/ipcu_oracle.cpp), and
  * the reference's own CUDA kernels with a C-ABI harness
    (oracle/_ref/libipcu_ref.so, built from the reference sources by
    oracle/Makefile; present only where the reference tree was available at
    build time).
Both follow the reference kernels' argument order (ref: all.hpp:38-158).
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _load_abi_tables():
    """ip_cu_lbm_b200/_abi.py (pure-Python signature tables) loaded as a
    standalone module, so that the checkers never import the product package."""
    import importlib.util

    name = "ipcu_abi_tables"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "ip_cu_lbm_b200", "_abi.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


_abi_tables = _load_abi_tables()
Binder, ptr = _abi_tables.Binder, _abi_tables.ptr

ORACLE_SO = os.path.join(HERE, "_build", "libipcu_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libipcu_ref.so")
REF_INPUT_DIR = os.path.join(HERE, "_ref")

_oracle = None
_ref = None


class Oracle:
    """CPU restatement; all pointers are host numpy arrays."""

    def __init__(self):
        self.lib = ctypes.CDLL(ORACLE_SO)
        self.b = Binder(self.lib, "oracle_", [], restype=None)
        P, I = ctypes.c_void_p, ctypes.c_int
        for prec in ("f32", "f64"):
            f = getattr(self.lib, f"oracle_IP_process_{prec}")
            f.argtypes = [P] * 12 + [I]
            f.restype = None
        self.lib.oracle_nearest_cells_f32.argtypes = [P, P, P, ctypes.c_longlong, P, I, P]
        self.lib.oracle_nearest_cells_f32.restype = None

    def __call__(self, name, prec, *args):
        return self.b(name, prec, *args)

    def nearest_cells(self, px, py, pz, nc, posw):
        """lattice_id per marker as the case drivers search it (float32 inputs)."""
        posw = np.ascontiguousarray(posw, np.float32).ravel()
        xyz = [np.ascontiguousarray(a, np.float32) for a in (px, py, pz)]
        lid = np.zeros(posw.size // 3, np.int32)
        self.lib.oracle_nearest_cells_f32(*[ptr(a) for a in xyz], int(nc), ptr(posw), posw.size // 3, ptr(lid))
        return lid

    def IP_process(self, prec, items, neib, f, feq, ftmp, fout, nextB, nextK, px, py, dX, dY, slip):
        getattr(self.lib, f"oracle_IP_process_{prec}")(
            *[ptr(a) for a in (items, neib, f, feq, ftmp, fout, nextB, nextK, px, py, dX, dY)], int(slip))


class Ref:
    """The reference's CUDA kernels; pointers are device addresses, each call
    launches <<<ceil(n/64), 64>>> on the legacy default stream and synchronises."""

    def __init__(self):
        self.lib = ctypes.CDLL(REF_SO)
        self.b = Binder(self.lib, "ref_", [ctypes.c_int64], restype=ctypes.c_int)
        P, I, I64, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
        for prec in ("f32", "f64"):
            f = getattr(self.lib, f"ref_IP_process_{prec}")
            f.argtypes = [P] * 12 + [I, I64]
            f.restype = I
        sig = {
            "ref_setc": ([I, D, D, I, P, P, P, P, P, P, P], None),
            "ref_set_M_f64": ([ctypes.c_char_p, I, P, P, P, P], I),
            "ref_set_neibghor_wall_f32": ([I, I, I, I, I, P, P, P, P, P, P, I64, P, P, P], I64),
            "ref_set_walln_f32": ([P, I, P, I64, I64, P, P], I),
            "ref_set_bound_f32": ([I, P, I, I, P, I64, P, P], I),
            "ref_set_quaternionS_f32": ([ctypes.c_float] * 4 + [P], None),
            "ref_le_steps_f32": ([P, P, P], I),
            "ref_ibm_steps_f32": ([P, P, P], I),
            "ref_buf_count": ([], I),
        }
        for name, (a, r) in sig.items():
            f = getattr(self.lib, name)
            f.argtypes, f.restype = a, r

    def __call__(self, name, prec, *args, n):
        return self.b(name, prec, *args, tail=(int(n),))

    def IP_process(self, prec, items, neib, f, feq, ftmp, fout, nextB, nextK, px, py, dX, dY, slip, n):
        return getattr(self.lib, f"ref_IP_process_{prec}")(
            *[ptr(a) for a in (items, neib, f, feq, ftmp, fout, nextB, nextK, px, py, dX, dY)], int(slip), int(n))


def oracle() -> Oracle:
    global _oracle
    if _oracle is None:
        _oracle = Oracle()
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref() -> Ref:
    global _ref
    if _ref is None:
        _ref = Ref()
    return _ref


# slot order of the harness's step-chain buffer table (ref_harness.cu enum RefBuf)
REF_BUFS = ["items", "neib", "nextB", "nextK", "f", "ftmp", "fout", "feq", "Fk", "g", "p", "sal", "phi", "tau",
            "taus", "Fx", "Fy", "Fz", "rho", "posx", "posy", "posz", "delX", "delY", "u", "v", "w", "M", "Minv",
            "S", "MM", "w1", "w2", "w3", "w4", "w5", "w6",
            "lid", "uo", "vo", "wo", "massB", "densB", "inertia", "FB", "posB", "Torque", "velB", "quat",
            "quaS", "angleVB", "posw", "oposw", "Gw", "velw", "nB", "onB", "quatold"]
