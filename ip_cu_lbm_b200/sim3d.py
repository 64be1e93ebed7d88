"""Python front end of the 3-D structured solver (ipcu_sim3d_* in libipcu.so):
D3Q19 MRT + D3Q7 salinity on a uniform box, one fused launch per step."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


class Sim3D:
    """A 3-D box advanced by the fused sm_100a step kernel. Fields come back
    as numpy arrays shaped [nz, ny, nx] (x fastest), or [q, nz, ny, nx]."""

    def __init__(self, nx, ny, nz, *, mrt=True, dz=1.0, dt=1.0, tau=0.55, taus=0.51, rho0=1.0, rho_sal=0.0,
                 g_bouss=0.0, s0=None, stream=None, x=None, wx=None, y=None, wy=None, ns=3, storage="f32"):
        """x, wx / y, wy: cell centres and widths of stretched x / y axes
        (z stays uniform), streamed with the ns-point conservative flux form
        (ipcu_sim3d_create_stretched); all None: the uniform box kernel.
        storage: "f32", or "f16" / "bf16" (populations stored as 16-bit
        deviations from a per-cell reference equilibrium; every box then
        runs the flux-form kernel)."""
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.N = self.nx * self.ny * self.nz
        cfg = _lib.Sim3DConfig()
        cfg.nx, cfg.ny, cfg.nz, cfg.mrt = self.nx, self.ny, self.nz, 1 if mrt else 0
        cfg.dz, cfg.dt, cfg.tau, cfg.taus = dz, dt, tau, taus
        cfg.rho0, cfg.rho_sal, cfg.g_bouss = rho0, rho_sal, g_bouss
        stores = {"f32": 0, "f16": 1, "bf16": 2}
        if storage not in stores:
            raise ValueError(f"storage must be one of {sorted(stores)}")
        cfg.storage = stores[storage]
        self.storage = storage
        s0p = None
        if s0 is not None:
            self._s0 = np.ascontiguousarray(s0, dtype=np.float64).reshape(-1)
            if self._s0.size != self.N:
                raise ValueError(f"s0 needs {self.N} values")
            s0p = self._s0.ctypes.data
        h = ctypes.c_void_p()
        if any(a is not None for a in (x, wx, y, wy)):
            self._axes = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (x, wx, y, wy)]
            for a, n in zip(self._axes, (self.nx, self.nx, self.ny, self.ny)):
                if a is not None and a.size != n:
                    raise ValueError("axis arrays need one value per cell")
            ax = _lib.Sim3DAxes(*[None if a is None else a.ctypes.data for a in self._axes], int(ns))
            _lib.check(_lib.lib().ipcu_sim3d_create_stretched(ctypes.byref(cfg), ctypes.byref(ax), s0p, stream,
                                                              ctypes.byref(h)), "ipcu_sim3d_create_stretched")
        else:
            _lib.check(_lib.lib().ipcu_sim3d_create(ctypes.byref(cfg), s0p, stream, ctypes.byref(h)),
                       "ipcu_sim3d_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().ipcu_sim3d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1):
        _lib.check(_lib.lib().ipcu_sim3d_step(self._h, int(n)), "ipcu_sim3d_step")

    def step_graph(self, n):
        _lib.check(_lib.lib().ipcu_sim3d_step_graph(self._h, int(n)), "ipcu_sim3d_step_graph")

    def get(self, field):
        q = {"f": 19, "g": 7, "F": 3}.get(field, 1)
        out = np.empty(q * self.N)
        _lib.check(_lib.lib().ipcu_sim3d_get(self._h, field.encode(), out.ctypes.data, out.size), "ipcu_sim3d_get")
        shape = (self.nz, self.ny, self.nx)
        return out.reshape((q,) + shape if q > 1 else shape)

    def set_state(self, f=None, g=None, F=None):
        keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (f, g, F)]
        _lib.check(_lib.lib().ipcu_sim3d_set_state(self._h, *[None if a is None else a.ctypes.data for a in keep]),
                   "ipcu_sim3d_set_state")

    def upload(self, f=None, g=None, F=None):
        P = lambda a: None if a is None else a.data_ptr()
        _lib.check(_lib.lib().ipcu_sim3d_upload(self._h, P(f), P(g), P(F)), "ipcu_sim3d_upload")

    def download(self, f=None, g=None, F=None):
        P = lambda a: None if a is None else a.data_ptr()
        _lib.check(_lib.lib().ipcu_sim3d_download(self._h, P(f), P(g), P(F)), "ipcu_sim3d_download")

    def macro_async(self, out):
        """S, u_x, u_y, u_z ([4, N] FP32, the values of get) formed on the
        device and copied into `out` (a pinned host or device tensor)
        asynchronously on the simulation's stream."""
        if out.numel() < 4 * self.N:
            raise ValueError(f"out needs {4 * self.N} floats")
        _lib.check(_lib.lib().ipcu_sim3d_macro_async(self._h, out.data_ptr()), "ipcu_sim3d_macro_async")

    def device_bytes(self):
        """Device bytes of the state (two buffers of f, g and the force planes)."""
        return int(self.bytes_per_cell()) * self.N

    def sync(self):
        _lib.check(_lib.lib().ipcu_sim3d_sync(self._h), "ipcu_sim3d_sync")

    # ---------------------------------------------------------------- moving sphere
    def attach_sphere(self, xc, yc, zc, radius, *, markers=None, rho_s=1.5, rho_f=1.0, gravity=0.0, iters=3,
                      u=0.0, v=0.0, w=0.0):
        """Attaches a rigid sphere (physical units) with `markers` markers on
        a Fibonacci lattice (default: about one per unit area, at least 64)
        that settles under gravity by multi-direct forcing
        (ipcu_sim3d_ib_attach)."""
        from .cases import sphere_markers

        n = int(markers) if markers else max(64, int(round(4.0 * np.pi * radius * radius)))
        r0, dA = sphere_markers(radius, n)
        self._sphere = (np.ascontiguousarray(r0, dtype=np.float64), np.ascontiguousarray(dA, dtype=np.float64))
        body = _lib.IBSphere3D(xc=xc, yc=yc, zc=zc, u=u, v=v, w=w, radius=radius, rho_s=rho_s, rho_f=rho_f,
                               gravity=gravity, iters=iters, pad=0)
        _lib.check(_lib.lib().ipcu_sim3d_ib_attach(self._h, ctypes.byref(body), self._sphere[0].ctypes.data,
                                                   self._sphere[1].ctypes.data, n), "ipcu_sim3d_ib_attach")

    def body(self):
        """Sphere state: dict of X (3), U (3), omega (3), Fib (3), Tib (3)."""
        out = np.zeros(15)
        _lib.check(_lib.lib().ipcu_sim3d_ib_body(self._h, out.ctypes.data), "ipcu_sim3d_ib_body")
        return {"X": out[0:3], "U": out[3:6], "omega": out[6:9], "Fib": out[9:12], "Tib": out[12:15]}

    def status(self):
        fl = ctypes.c_uint32()
        _lib.lib().ipcu_sim3d_status(self._h, ctypes.byref(fl))
        return fl.value

    def bytes_per_cell(self):
        return int(_lib.lib().ipcu_sim3d_bytes_per_cell(self._h))

    def steps(self):
        return int(_lib.lib().ipcu_sim3d_steps(self._h))

    def save(self, path):
        """Versioned binary snapshot (ipcu_sim3d_save)."""
        _lib.check(_lib.lib().ipcu_sim3d_save(self._h, str(path).encode()), "ipcu_sim3d_save")

    @classmethod
    def load(cls, path, stream=None):
        """Restores a simulation saved with `save`."""
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().ipcu_sim3d_load(str(path).encode(), stream, ctypes.byref(h)), "ipcu_sim3d_load")
        obj = cls.__new__(cls)
        obj._h = h
        cfg = _lib.Sim3DConfig()
        with open(path, "rb") as fh:
            head = fh.read(12 + ctypes.sizeof(cfg))
        cfg = _lib.Sim3DConfig.from_buffer_copy(head[12:])
        obj.nx, obj.ny, obj.nz = cfg.nx, cfg.ny, cfg.nz
        version = int.from_bytes(head[8:12], "little")
        obj.storage = {0: "f32", 1: "f16", 2: "bf16"}[cfg.storage if version >= 2 else 0]
        obj.N = obj.nx * obj.ny * obj.nz
        return obj
