"""Loader of libipcu.so, the compiled sm_100a library of this package.

The library is built in-tree (``make -C ip_cu_lbm_b200/csrc``, or
``__graft_entry__.build()``) and loaded from the package directory. There
is no fallback: if the library is missing or fails to load, importing the
GPU entry points raises.
"""
from __future__ import annotations

import ctypes
import os

from ._abi import Binder

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libipcu.so")

IPCU_OK = 0
STATUS = {
    0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "out of device memory",
    -4: "output capacity too small", -5: "non-finite value detected",
    -6: "unsupported configuration", -7: "file I/O error", -8: "device wait timed out",
}

_lib = None


class IpcuError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        super().__init__(f"{what}: {STATUS.get(code, 'status %d' % code)}")


def lib() -> ctypes.CDLL:
    """The loaded libipcu.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"libipcu.so not found at {LIB_PATH}; build it with "
                "`make -C ip_cu_lbm_b200/csrc -j` (nvcc, sm_100a)")
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def check(code: int, what: str = "ipcu") -> int:
    if code != IPCU_OK:
        raise IpcuError(code, what)
    return code


def legacy() -> Binder:
    """Binder for the reference-compatible launchers: ipcu_<name>_<prec>(..., nthreads, stream)."""
    return Binder(lib(), "ipcu_", [ctypes.c_int64, ctypes.c_void_p])


class SimConfig(ctypes.Structure):
    """Mirror of ipcu_sim_config (include/ipcu_sim.h)."""
    _fields_ = [
        ("nx", ctypes.c_int32), ("nz", ctypes.c_int32), ("q_scalar", ctypes.c_int32),
        ("geometry", ctypes.c_int32), ("storage", ctypes.c_int32), ("wall", ctypes.c_int32),
        ("mrt", ctypes.c_int32), ("scalar_kind", ctypes.c_int32),
        ("dz", ctypes.c_double), ("dt", ctypes.c_double),
        ("x", ctypes.c_void_p), ("z", ctypes.c_void_p), ("wx", ctypes.c_void_p), ("wz", ctypes.c_void_p),
        ("tau", ctypes.c_double), ("taus", ctypes.c_double),
        ("rhoL", ctypes.c_double), ("rhoH", ctypes.c_double), ("phi", ctypes.c_double),
        ("rho_sal", ctypes.c_double), ("g_bouss", ctypes.c_double), ("s_ref", ctypes.c_double),
        ("M", ctypes.c_void_p), ("Minv", ctypes.c_void_p), ("S", ctypes.c_void_p),
        ("sigma", ctypes.c_double), ("pf_width", ctypes.c_double), ("gravity", ctypes.c_double),
    ]


class IBBody2D(ctypes.Structure):
    """Mirror of ipcu_ib_body2d (include/ipcu_sim.h)."""
    _fields_ = [
        ("xc", ctypes.c_double), ("zc", ctypes.c_double), ("theta", ctypes.c_double),
        ("u", ctypes.c_double), ("w", ctypes.c_double), ("omega", ctypes.c_double),
        ("rho_s", ctypes.c_double), ("rho_f", ctypes.c_double),
        ("area", ctypes.c_double), ("inertia", ctypes.c_double),
        ("semi_a", ctypes.c_double), ("semi_b", ctypes.c_double),
        ("gravity", ctypes.c_double), ("iters", ctypes.c_int32), ("pad", ctypes.c_int32),
    ]


class IBSphere3D(ctypes.Structure):
    """Mirror of ipcu_ib_sphere3d (include/ipcu_sim3d.h)."""
    _fields_ = [
        ("xc", ctypes.c_double), ("yc", ctypes.c_double), ("zc", ctypes.c_double),
        ("u", ctypes.c_double), ("v", ctypes.c_double), ("w", ctypes.c_double),
        ("radius", ctypes.c_double), ("rho_s", ctypes.c_double), ("rho_f", ctypes.c_double),
        ("gravity", ctypes.c_double), ("iters", ctypes.c_int32), ("pad", ctypes.c_int32),
    ]


class Sim3DAxes(ctypes.Structure):
    """Mirror of ipcu_sim3d_axes (include/ipcu_sim3d.h)."""
    _fields_ = [("x", ctypes.c_void_p), ("wx", ctypes.c_void_p), ("y", ctypes.c_void_p), ("wy", ctypes.c_void_p),
                ("ns", ctypes.c_int32)]


class Sim3DConfig(ctypes.Structure):
    """Mirror of ipcu_sim3d_config (include/ipcu_sim3d.h)."""
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("mrt", ctypes.c_int32),
        ("dz", ctypes.c_double), ("dt", ctypes.c_double), ("tau", ctypes.c_double), ("taus", ctypes.c_double),
        ("rho0", ctypes.c_double), ("rho_sal", ctypes.c_double), ("g_bouss", ctypes.c_double),
        ("storage", ctypes.c_int32), ("pad", ctypes.c_int32),
    ]


def _declare(L: ctypes.CDLL) -> None:
    P, I, I64, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
    sig = {
        "ipcu_status_string": ([I], ctypes.c_char_p),
        "ipcu_last_cuda_error": ([], ctypes.c_char_p),
        "ipcu_version": ([], I),
        "ipcu_IP_process_f32": ([P, I, I, P, P, P, P, P, P, P, P, P, P, P, I, P], I),
        "ipcu_IP_process_f64": ([P, I, I, P, P, P, P, P, P, P, P, P, P, P, I, P], I),
        "ipcu_setc": ([I, D, D, I, P, P, P, P, P, P, P], I),
        "ipcu_read_M_csv": ([ctypes.c_char_p, I, P, P, P], I),
        "ipcu_set_M": ([I, P, P, P, P, P, P, P], I),
        "ipcu_set_neibghor_wall": ([I, I, I, I, I64, P, P, I64, P], I64),
        "ipcu_set_walln_f32": ([P, P, I64, P, P], I),
        "ipcu_set_walln_f64": ([P, P, I64, P, P], I),
        "ipcu_set_bound2D_f32": ([P, I, P, P, P], I),
        "ipcu_set_bound2D_f64": ([P, I, P, P, P], I),
        "ipcu_set_bound3D_f32": ([P, I, P, P, P], I),
        "ipcu_set_bound3D_f64": ([P, I, P, P, P], I),
        "ipcu_build_box_grid": ([I, I, I, I, D, D, D, P, P, P, P, P, P, P, P, P], I64),
        "ipcu_set_quaternionS_f64": ([I, D, D, D, D, P], None),
        "ipcu_set_quaternionS_f32": ([I, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, P], None),
        "ipcu_sim_create": ([ctypes.POINTER(SimConfig), P, P, ctypes.POINTER(P)], I),
        "ipcu_sim_destroy": ([P], None),
        "ipcu_sim_step": ([P, I64], I),
        "ipcu_sim_step_graph": ([P, I64, ctypes.c_int32], I),
        "ipcu_sim_get": ([P, ctypes.c_char_p, P, I64], I),
        "ipcu_sim_set_state": ([P, P, P, P, P, P], I),
        "ipcu_sim_status": ([P, ctypes.POINTER(ctypes.c_uint32)], I),
        "ipcu_sim_cells": ([P], I64),
        "ipcu_sim_device_state": ([P, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(P)], I),
        "ipcu_sim_bytes_per_cell": ([P], I64),
        "ipcu_sim_totals": ([P, ctypes.POINTER(D), ctypes.POINTER(D)], I),
        "ipcu_sim_set_lean": ([P, I], I),
        "ipcu_sim_lean": ([P], I),
        "ipcu_sim_set_push": ([P, I], I),
        "ipcu_sim_push": ([P], I),
        "ipcu_sim_upload": ([P, P, P, P], I),
        "ipcu_sim_download": ([P, P, P, P], I),
        "ipcu_sim_sync": ([P], I),
        "ipcu_sim_storage_bytes": ([P], ctypes.c_int32),
        "ipcu_sim_steps": ([P], I64),
        "ipcu_sim_save": ([P, ctypes.c_char_p], I),
        "ipcu_sim_load": ([ctypes.c_char_p, P, ctypes.POINTER(P)], I),
        "ipcu_sim_write_csv": ([P, ctypes.c_char_p], I),
        "ipcu_totals_noalloc_f32": ([P, P, P, P, I, I, P, P], I),
        "ipcu_add_scalar_f32": ([P, I64, ctypes.c_float, P], I),
        "ipcu_batch_create": ([P, ctypes.POINTER(P)], I),
        "ipcu_batch_destroy": ([P], None),
        "ipcu_batch_step": ([P, P, I, I64], I),
        "ipcu_batch_launch": ([P, P, I, I64], I),
        "ipcu_batch_launch_each": ([P, P, P, I], I),
        "ipcu_batch_sync": ([P], I),
        "ipcu_batch_mark": ([P], I),
        "ipcu_batch_wait_mark": ([P, I], I),
        "ipcu_batch_set_graph": ([P, I], I),
        "ipcu_batch_graph_stats": ([P, P, P], I),
        "ipcu_batch_set_ctas": ([P, I, I, I, I, I], I),
        "ipcu_sim_device_bytes": ([P], I64),
        "ipcu_sim_ib_attach": ([P, ctypes.POINTER(IBBody2D), P, P, ctypes.c_int32], I),
        "ipcu_sim_ib_body": ([P, P], I),
        "ipcu_sim_ib_body_at": ([P, ctypes.c_int32, P], I),
        "ipcu_sim_ib_count": ([P], ctypes.c_int32),
        "ipcu_sim_ib_markers": ([P, P, ctypes.c_int32], ctypes.c_int32),
        "ipcu_sim_ib_markers_at": ([P, ctypes.c_int32, P, ctypes.c_int32], ctypes.c_int32),
        "ipcu_sim_write_ib_csv": ([P, ctypes.c_char_p], I),
        "ipcu_sim3d_save": ([P, ctypes.c_char_p], I),
        "ipcu_sim3d_load": ([ctypes.c_char_p, P, ctypes.POINTER(P)], I),
        "ipcu_sim3d_steps": ([P], I64),
        "ipcu_sim3d_ib_attach": ([P, ctypes.POINTER(IBSphere3D), P, P, ctypes.c_int32], I),
        "ipcu_sim3d_ib_body": ([P, P], I),
        "ipcu_stream_create": ([ctypes.POINTER(P)], I),
        "ipcu_stream_destroy": ([P], I),
        "ipcu_sim3d_create": ([ctypes.POINTER(Sim3DConfig), P, P, ctypes.POINTER(P)], I),
        "ipcu_sim3d_create_stretched": ([ctypes.POINTER(Sim3DConfig), ctypes.POINTER(Sim3DAxes), P, P,
                                         ctypes.POINTER(P)], I),
        "ipcu_sim3d_destroy": ([P], None),
        "ipcu_sim3d_step": ([P, I64], I),
        "ipcu_sim3d_step_graph": ([P, I64], I),
        "ipcu_sim3d_get": ([P, ctypes.c_char_p, P, I64], I),
        "ipcu_sim3d_set_state": ([P, P, P, P], I),
        "ipcu_sim3d_upload": ([P, P, P, P], I),
        "ipcu_sim3d_download": ([P, P, P, P], I),
        "ipcu_sim3d_macro_async": ([P, P], I),

        "ipcu_sim3d_sync": ([P], I),
        "ipcu_sim3d_status": ([P, ctypes.POINTER(ctypes.c_uint32)], I),
        "ipcu_sim3d_cells": ([P], I64),
        "ipcu_sim3d_bytes_per_cell": ([P], I64),
        "ipcu_build_box_device_f32": ([I, I, I, I, D, D, D, P, P, P, P, P, P, P, P, P, I64, P,
                                       ctypes.POINTER(I64), ctypes.POINTER(I64), P], I),
        "ipcu_build_box_device_f64": ([I, I, I, I, D, D, D, P, P, P, P, P, P, P, P, P, I64, P,
                                       ctypes.POINTER(I64), ctypes.POINTER(I64), P], I),
        "ipcu_nearest_cells_f32": ([P, P, P, I64, P, I, P, P], I),
        "ipcu_nearest_cells_f64": ([P, P, P, I64, P, I, P, P], I),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
