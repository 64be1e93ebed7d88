"""Signature tables of the reference kernel-entry API and a ctypes binder.

The same per-kernel argument lists describe three libraries that share the
reference's calling convention (ref: all.hpp:38-158):
  * libipcu.so          -- the product: ipcu_<name>_<f32|f64>(..., int64 nthreads, stream)
  * oracle CPU library   -- test infrastructure: oracle_<name>_<f32|f64>(...)
  * oracle/_ref harness  -- test infrastructure: ref_<name>_<f32|f64>(..., int64 n)

Argument codes: P pointer, i int, T scalar of the precision, f float.
"""
from __future__ import annotations

import ctypes

# kernel name -> argument codes, in the reference's order
LEGACY = {
    "equ_f": "PPPPPP",                      # collision.cu:3
    "equ_g": "PPPPPP",                      # collision.cu:16
    "wall_function": "PPPiiiiPPPPPPP",      # collision.cu:28
    "Force": "PiPPPPPPPPPPPPPPPPPPPP",      # collision.cu:57
    "col_f_MRT": "PPPPPPPPPP",              # collision.cu:115
    "col_f_SRT": "PPPPPP",                  # collision.cu:151
    "col_g_reg": "PPPPPPPPP",               # collision.cu:167
    "col_PF": "PPPPPPPPPPPPPPPPP",          # collision.cu:190
    "update_scalar": "PPP",                 # collision.cu:225
    "update_rho": "PTTPPPPPPPPPPP",         # collision.cu:238
    "resetF": "PPPPi",                      # collision.cu:258
    "set_wall_f": "PPP",                    # adv.cu:3
    "set_out": "PPPPPPPPPP",                # adv.cu:50
    "set_fin": "PPPPP",                     # adv.cu:148
    "reset_f": "PPPP",                      # adv.cu:176
    "set_wall_f_inv": "PPPPP",              # adv.cu:188
    "set_tmp": "PPPPPP",                    # adv.cu:234
    "set_wall_propagation": "PiPPPP",       # set_bound.cu:164
    "propagation": "PPPP",                  # propagation.cu:2
    "reset_wall_fin": "PPP",                # basic.cu:274
    "set_wall_rho": "PPP",                  # basic.cu:254
    "reset_pressure": "PPPPPPT",            # basic.cu:262
    "LES": "PPPPPPTTPPPPPP",                # basic.cu:285
    "get_IBMGw2": "PPPPPPPPPPPPPPPPPPPT",   # ibm.cu:124
    "update_velIBM": "PPPPPPPPPPPPPPP",     # ibm.cu:346
    "update_IBbody": "PiPPPPPPPPPPPPPT",    # ibm.cu:367
    "update_IBpoint": "PiPPPPPPPPP",        # ibm.cu:426
    "search_IBlattice": "PiPPPPPP",         # ibm.cu:449
    "SPM": "PTPPPPPPPPPPPPP",               # ibm.cu:68
}
FLOAT_ONLY = {
    "IB_directForcing": "PPPPPPPPPPPPPPP",  # ibm.cu:276
    "SPM_ellipse": "PffPPPPPPPPPPPP",       # ibm.cu:87
}
# kernels the reference instantiates in float only (search_IBlattice, ibm.cu:483)
REF_FLOAT_ONLY = {"search_IBlattice"}


def _ctype(code: str, prec: str):
    if code == "P":
        return ctypes.c_void_p
    if code == "i":
        return ctypes.c_int
    if code == "f":
        return ctypes.c_float
    if code == "T":
        return ctypes.c_float if prec == "f32" else ctypes.c_double
    raise ValueError(code)


def ptr(x):
    """Address of a numpy array, torch tensor, int or None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    raise TypeError(f"cannot take the address of {type(x)}")


class Binder:
    """Binds `<prefix><name>_<prec>` from a CDLL with the signature table and
    a fixed tail of extra argument types (e.g. nthreads + stream)."""

    def __init__(self, lib: ctypes.CDLL, prefix: str, tail: list, restype=ctypes.c_int):
        self.lib, self.prefix, self.tail, self.restype = lib, prefix, tail, restype
        self._cache = {}

    def fn(self, name: str, prec: str):
        key = (name, prec)
        if key not in self._cache:
            codes = LEGACY.get(name) or FLOAT_ONLY.get(name)
            if codes is None:
                raise KeyError(name)
            f = getattr(self.lib, f"{self.prefix}{name}_{prec}")
            f.argtypes = [_ctype(c, prec) for c in codes] + list(self.tail)
            f.restype = self.restype
            self._cache[key] = f
        return self._cache[key]

    def __call__(self, name: str, prec: str, *args, tail=()):
        codes = LEGACY.get(name) or FLOAT_ONLY.get(name)
        if len(args) != len(codes):
            raise TypeError(f"{name} takes {len(codes)} arguments, got {len(args)}")
        conv = [ptr(a) if c == "P" else a for c, a in zip(codes, args)]
        return self.fn(name, prec)(*conv, *tail)
