"""Python front end of the structured-grid solver (ipcu_sim_* in libipcu.so)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .cases import d2q9_mrt, ellipse_markers

GEOMETRY = {"uniform": 0, "x5": 1, "x3": 2, "z5": 3, "z3": 4}
STORAGE = {"f32": 0, "f16": 1, "bf16": 2}
WALL = {"slip": 0, "bb": 1}
SCALAR = {"salinity": 0, "phase": 1}

# the reference's constants (ref: function/collision.cu:78,251)
REF_RHO_SAL = 0.824493
REF_G_BOUSS = 0.824493 * 9.81


class Sim:
    """A 2-D box (x-z plane) advanced by the fused sm_100a step kernel.

    Fields are returned as numpy arrays shaped [nz, nx] (x fastest), or
    [q, nz, nx] for the distributions f and g.
    """

    def __init__(self, nx, nz, *, q_scalar=5, geometry="uniform", storage="f32", wall="bb", mrt=True,
                 dz=1.0, dt=1.0, x=None, z=None, wx=None, wz=None, tau=0.53, taus=0.503,
                 rhoL=1.0, rhoH=1.0, phi=1.0, rho_sal=0.0, g_bouss=1e-4, s_ref=0.5,
                 M=None, Minv=None, S=None, s0=None, stream=None, scalar="salinity", sigma=0.0, pf_width=4.0,
                 gravity=0.0):
        L = _lib.lib()
        self.nx, self.nz, self.q_scalar = int(nx), int(nz), int(q_scalar)
        self._keep = []

        def arr(a, n):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float64)
            if a.size != n:
                raise ValueError(f"expected {n} values, got {a.size}")
            self._keep.append(a)
            return a.ctypes.data

        if mrt and M is None:
            M, Minv, S = d2q9_mrt()
        cfg = _lib.SimConfig()
        cfg.nx, cfg.nz, cfg.q_scalar = self.nx, self.nz, self.q_scalar
        cfg.geometry = GEOMETRY[geometry] if isinstance(geometry, str) else int(geometry)
        cfg.storage = STORAGE[storage] if isinstance(storage, str) else int(storage)
        cfg.wall = WALL[wall] if isinstance(wall, str) else int(wall)
        cfg.mrt = 1 if mrt else 0
        cfg.dz, cfg.dt = dz, dt
        cfg.x, cfg.z, cfg.wx, cfg.wz = arr(x, nx), arr(z, nz), arr(wx, nx), arr(wz, nz)
        cfg.tau, cfg.taus = tau, taus
        cfg.rhoL, cfg.rhoH, cfg.phi = rhoL, rhoH, phi
        cfg.rho_sal, cfg.g_bouss, cfg.s_ref = rho_sal, g_bouss, s_ref
        cfg.scalar_kind = SCALAR[scalar] if isinstance(scalar, str) else int(scalar)
        cfg.sigma, cfg.pf_width, cfg.gravity = sigma, pf_width, gravity
        if mrt:
            cfg.M, cfg.Minv, cfg.S = arr(M, 81), arr(Minv, 81), arr(S, 9)
        s0p = arr(s0, nx * nz)
        h = ctypes.c_void_p()
        _lib.check(L.ipcu_sim_create(ctypes.byref(cfg), s0p, stream, ctypes.byref(h)), "ipcu_sim_create")
        self._h = h
        self.N = self.nx * self.nz
        self.storage = storage
        # (storage, scalar lattice, geometry, scalar kind): the batched kernel class
        self.kernel_class = (int(cfg.storage), int(cfg.q_scalar), int(cfg.geometry), int(cfg.scalar_kind))

    # ---------------------------------------------------------------- lifecycle
    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().ipcu_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- stepping
    def step(self, n=1):
        _lib.check(_lib.lib().ipcu_sim_step(self._h, int(n)), "ipcu_sim_step")

    def step_graph(self, n, chunk=64):
        _lib.check(_lib.lib().ipcu_sim_step_graph(self._h, int(n), int(chunk)), "ipcu_sim_step_graph")

    # ---------------------------------------------------------------- immersed body
    def attach_ellipse(self, xc, zc, a, b, *, markers=240, theta=0.0, rho_s=1.1, rho_f=1.0, gravity=0.0,
                       iters=3, u=0.0, w=0.0, omega=0.0):
        """Attaches a rigid ellipse (semi-axes a along the body x axis, b along
        its z axis, physical units) with `markers` markers at equal arc length;
        it settles under gravity by multi-direct forcing (ipcu_sim_ib_attach).
        Each call adds a body (index 0, 1, ...); bodies must stay at least 6
        cells apart."""
        X0, dS = ellipse_markers(a, b, markers)
        body = _lib.IBBody2D(xc=xc, zc=zc, theta=theta, u=u, w=w, omega=omega, rho_s=rho_s, rho_f=rho_f,
                             area=np.pi * a * b, inertia=np.pi * a * b * (a * a + b * b) / 4, semi_a=a, semi_b=b,
                             gravity=gravity, iters=iters, pad=0)
        X0 = np.ascontiguousarray(X0, dtype=np.float64)
        dS = np.ascontiguousarray(dS, dtype=np.float64)
        _lib.check(_lib.lib().ipcu_sim_ib_attach(self._h, ctypes.byref(body), X0.ctypes.data, dS.ctypes.data,
                                                 len(dS)), "ipcu_sim_ib_attach")

    @property
    def n_bodies(self):
        """Bodies attached."""
        return int(_lib.lib().ipcu_sim_ib_count(self._h))

    def body(self, index=0):
        """State of body `index`: dict of x, z, u, w, theta, omega, Fx, Fz, T
        (the IB force and torque on the fluid in the last step)."""
        out = np.zeros(9)
        _lib.check(_lib.lib().ipcu_sim_ib_body_at(self._h, int(index), out.ctypes.data), "ipcu_sim_ib_body_at")
        return dict(zip(("x", "z", "u", "w", "theta", "omega", "Fx", "Fz", "T"), out.tolist()))

    def markers(self, index=0):
        """Markers of body `index`, [n, 9]: x, y, z, u, v, w, Fx, Fy, Fz
        (position, velocity, force on the fluid in the last update)."""
        cap = 4096
        out = np.zeros(9 * cap)
        n = _lib.lib().ipcu_sim_ib_markers_at(self._h, int(index), out.ctypes.data, cap)
        if n < 0:
            _lib.check(n, "ipcu_sim_ib_markers_at")
        return out.reshape(cap, 9)[:n].copy()

    def write_ib_csv(self, path):
        """The markers as the reference's IB_csv writes them (ibm.cu:3-14)."""
        _lib.check(_lib.lib().ipcu_sim_write_ib_csv(self._h, str(path).encode()), "ipcu_sim_write_ib_csv")

    # ---------------------------------------------------------------- fields
    def get(self, field):
        n = self.N * (9 if field == "f" else (self.q_scalar if field == "g" else 1))
        out = np.zeros(n)
        _lib.check(_lib.lib().ipcu_sim_get(self._h, field.encode(), out.ctypes.data, n), f"get {field}")
        if field in ("f", "g"):
            return out.reshape(-1, self.nz, self.nx)
        return out.reshape(self.nz, self.nx)

    def set_state(self, f=None, g=None, S=None, ux=None, uz=None):
        keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (f, g, S, ux, uz)]
        p = [None if a is None else a.ctypes.data for a in keep]
        _lib.check(_lib.lib().ipcu_sim_set_state(self._h, *p), "ipcu_sim_set_state")

    def status(self):
        fl = ctypes.c_uint32()
        _lib.lib().ipcu_sim_status(self._h, ctypes.byref(fl))
        return fl.value

    def totals(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        _lib.check(_lib.lib().ipcu_sim_totals(self._h, ctypes.byref(a), ctypes.byref(b)), "ipcu_sim_totals")
        return a.value, b.value

    def set_lean(self, on=True):
        """Turns the lean flow-only step on or off (ipcu_sim_set_lean)."""
        _lib.check(_lib.lib().ipcu_sim_set_lean(self._h, 1 if on else 0), "ipcu_sim_set_lean")

    def lean(self):
        """True while the step kernel runs the lean flow-only step."""
        return bool(_lib.lib().ipcu_sim_lean(self._h))

    def set_push(self, on=True):
        """Selects the push form (on) or the tile form (off) of the lean step
        (ipcu_sim_set_push)."""
        _lib.check(_lib.lib().ipcu_sim_set_push(self._h, 1 if on else 0), "ipcu_sim_set_push")

    def push(self):
        """True while the lean step runs in its push form."""
        return bool(_lib.lib().ipcu_sim_push(self._h))

    def bytes_per_cell(self):
        return int(_lib.lib().ipcu_sim_bytes_per_cell(self._h))

    def mac_planes(self):
        """FP32 macroscopic planes of the raw state: S, u_x, u_z (+ p* with 16-bit storage)."""
        return 3 if self.storage_bytes() == 4 else 4

    def upload(self, f=None, g=None, mac=None):
        """Asynchronous raw upload from (ideally pinned) host buffers in the storage layout."""
        P = lambda a: None if a is None else (a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data)
        _lib.check(_lib.lib().ipcu_sim_upload(self._h, P(f), P(g), P(mac)), "ipcu_sim_upload")

    def download(self, f=None, g=None, mac=None):
        P = lambda a: None if a is None else (a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data)
        _lib.check(_lib.lib().ipcu_sim_download(self._h, P(f), P(g), P(mac)), "ipcu_sim_download")

    def sync(self):
        _lib.check(_lib.lib().ipcu_sim_sync(self._h), "ipcu_sim_sync")

    def storage_bytes(self):
        return int(_lib.lib().ipcu_sim_storage_bytes(self._h))

    def device_bytes(self):
        return int(_lib.lib().ipcu_sim_device_bytes(self._h))

    def steps(self):
        return int(_lib.lib().ipcu_sim_steps(self._h))

    def save(self, path):
        _lib.check(_lib.lib().ipcu_sim_save(self._h, str(path).encode()), "ipcu_sim_save")

    @classmethod
    def load(cls, path, stream=None):
        """Restores a simulation saved with `save`."""
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().ipcu_sim_load(str(path).encode(), stream, ctypes.byref(h)), "ipcu_sim_load")
        obj = cls.__new__(cls)
        obj._h, obj._keep = h, []
        obj.N = int(_lib.lib().ipcu_sim_cells(h))
        obj._dims_from_file(path)
        return obj

    def _dims_from_file(self, path):
        # snapshot header: 8-byte magic, int32 version, then the configuration struct
        with open(path, "rb") as fh:
            head = fh.read(8 + 4 + ctypes.sizeof(_lib.SimConfig))
        cfg = _lib.SimConfig.from_buffer_copy(head[12:])
        self.nx, self.nz, self.q_scalar = cfg.nx, cfg.nz, cfg.q_scalar
        self.storage = {0: "f32", 1: "f16", 2: "bf16"}[cfg.storage]

    def write_csv(self, path):
        _lib.check(_lib.lib().ipcu_sim_write_csv(self._h, str(path).encode()), "ipcu_sim_write_csv")

    def device_state(self):
        f, g, m = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        _lib.check(_lib.lib().ipcu_sim_device_state(self._h, ctypes.byref(f), ctypes.byref(g), ctypes.byref(m)))
        return f.value, g.value, m.value
