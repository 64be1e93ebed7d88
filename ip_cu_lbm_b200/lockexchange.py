"""The reference case drivers' per-step kernel order on the reference-
compatible entries of libipcu (the drop-in path).

`le_step` replays LockExchange (ref: LockExchange/LockExchange.cu:214-278)
and `ibm_step` the moving-IBM drivers (ref:
EllipticalFall2/EllipticalFallxz.cu:344-430). Both take a `call(name,
*args)` that launches one kernel of the reference API and an `ip(f, feq,
ftmp, fout)` that runs the streaming pass, so the same order drives this
library, the reference build or a CPU restatement.

`LockExchange` owns the device buffers (torch tensors, used as plain
device memory) of one compacted-grid case and steps it through libipcu.
"""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from . import _lib


def le_step(call, ip, B, *, mrt=True, scalar=True, wall_function=False, boussi=1, rhoL=1.0, rhoH=1000.0,
            num_F=None, wall_sizes=(0, 0, 0, 0, 0, 0)):
    if wall_function:
        w1, w2, w3, w4, w5, w6 = wall_sizes
        call("wall_function", B.items, B.delX, B.delY, 1, 0, 0, w1, B.w1, B.v, B.w, B.u, B.Fy, B.Fz, B.rho)
        call("wall_function", B.items, B.delX, B.delY, 1, 0, 0, w3, B.w3, B.v, B.w, B.u, B.Fy, B.Fz, B.rho)
        call("wall_function", B.items, B.delX, B.delY, 0, 0, 1, w5, B.w5, B.u, B.v, B.w, B.Fx, B.Fy, B.rho)
        call("wall_function", B.items, B.delX, B.delY, 0, 0, 1, w6, B.w6, B.u, B.v, B.w, B.Fx, B.Fy, B.rho)
        call("wall_function", B.items, B.delX, B.delY, 0, 1, 0, w2, B.w2, B.u, B.w, B.v, B.Fx, B.Fz, B.rho)
        call("wall_function", B.items, B.delX, B.delY, 0, 1, 0, w4, B.w4, B.u, B.w, B.v, B.Fx, B.Fz, B.rho)
    call("equ_f", B.items, B.feq, B.p, B.u, B.v, B.w)
    call("Force", B.items, int(boussi), B.neib, B.f, B.feq, B.tau, B.Fk, B.Fx, B.Fy, B.Fz, B.p, B.rho, B.sal, B.phi,
         B.u, B.v, B.w, B.delX, B.delY, B.posx, B.posy, B.posz)
    if mrt:
        call("col_f_MRT", B.items, B.tau, B.f, B.ftmp, B.feq, B.Fk, B.M, B.Minv, B.S, B.MM)
    else:
        call("col_f_SRT", B.items, B.tau, B.f, B.ftmp, B.feq, B.Fk)
    ip(B.f, B.feq, B.ftmp, B.fout)
    if scalar:
        call("col_g_reg", B.items, B.taus, B.g, B.ftmp, B.feq, B.sal, B.u, B.v, B.w)
        ip(B.g, B.feq, B.ftmp, B.fout)
        call("update_scalar", B.items, B.g, B.sal)
    call("update_rho", B.items, rhoL, rhoH, B.f, B.Fx, B.Fy, B.Fz, B.p, B.sal, B.phi, B.rho, B.u, B.v, B.w)
    call("set_wall_rho", B.items, B.neib, B.rho)
    call("resetF", B.items, B.Fx, B.Fy, B.Fz, int(num_F))


def pf_step(call, ip, B, *, mrt=True, rhoL=1.0, rhoH=3.0, num_F=None):
    """One step of the reference's two-phase driver order (ref:
    RTinstability/RTinstability.cu:177-206): equilibrium, force with surface
    tension and the mixture's weight (Boussi_flag off), MRT collision and
    interpolated streaming of f, conservative Allen-Cahn collision and
    streaming of the phase field g, phi = sum g, moments, ghost rho and phi."""
    call("equ_f", B.items, B.feq, B.p, B.u, B.v, B.w)
    call("Force", B.items, 0, B.neib, B.f, B.feq, B.tau, B.Fk, B.Fx, B.Fy, B.Fz, B.p, B.rho, B.sal, B.phi,
         B.u, B.v, B.w, B.delX, B.delY, B.posx, B.posy, B.posz)
    if mrt:
        call("col_f_MRT", B.items, B.tau, B.f, B.ftmp, B.feq, B.Fk, B.M, B.Minv, B.S, B.MM)
    else:
        call("col_f_SRT", B.items, B.tau, B.f, B.ftmp, B.feq, B.Fk)
    ip(B.f, B.feq, B.ftmp, B.fout)
    call("col_PF", B.items, B.neib, B.taus, B.g, B.ftmp, B.feq, B.phi, B.u, B.v, B.w, B.phiold, B.uold, B.vold,
         B.wold, B.posx, B.posy, B.posz)
    ip(B.g, B.feq, B.ftmp, B.fout)
    call("update_scalar", B.items, B.g, B.phi)
    call("update_rho", B.items, rhoL, rhoH, B.f, B.Fx, B.Fy, B.Fz, B.p, B.sal, B.phi, B.rho, B.u, B.v, B.w)
    call("set_wall_rho", B.items, B.neib, B.rho)
    call("set_wall_rho", B.items, B.neib, B.phi)
    call("resetF", B.items, B.Fx, B.Fy, B.Fz, int(num_F))


def ibm_step(call, ip, B, *, mrt=False, boussi=1, rhoL=1.0, rhoH=1000.0, num_F=None, num_Gw=None):
    call("equ_f", B.items, B.feq, B.p, B.u, B.v, B.w)
    call("Force", B.items, int(boussi), B.neib, B.f, B.feq, B.tau, B.Fk, B.Fx, B.Fy, B.Fz, B.p, B.rho, B.sal, B.phi,
         B.u, B.v, B.w, B.delX, B.delY, B.posx, B.posy, B.posz)
    if mrt:
        call("col_f_MRT", B.items, B.tau, B.f, B.ftmp, B.feq, B.Fk, B.M, B.Minv, B.S, B.MM)
    else:
        call("col_f_SRT", B.items, B.tau, B.f, B.ftmp, B.feq, B.Fk)
    ip(B.f, B.feq, B.ftmp, B.fout)
    call("update_rho", B.items, rhoL, rhoH, B.f, B.Fx, B.Fy, B.Fz, B.p, B.sal, B.phi, B.rho, B.u, B.v, B.w)
    call("resetF", B.items, B.Fx, B.Fy, B.Fz, int(num_F))
    B.copy_f_ftmp()  # driver-local set_f_ftmp (EllipticalFallxz.cu:4-13)
    call("get_IBMGw2", B.items, B.lid, B.neib, B.f, B.tau, B.posx, B.posy, B.posz, B.posw, B.posB, B.nB, B.u, B.v,
         B.w, B.velw, B.Fx, B.Fy, B.Fz, B.Gw, rhoH)
    call("update_velIBM", B.items, B.lid, B.f, B.ftmp, B.p, B.tau, B.u, B.v, B.w, B.uo, B.vo, B.wo, B.Fx, B.Fy, B.Fz)
    call("update_IBbody", B.items, 0, B.massB, B.densB, B.inertia, B.FB, B.posB, B.Torque, B.velB, B.quat, B.quaS,
         B.angleVB, B.posw, B.Gw, B.quatold, rhoH)
    call("update_IBpoint", B.items, 0, B.posB, B.velB, B.angleVB, B.quaS, B.posw, B.oposw, B.nB, B.onB, B.velw)
    call("search_IBlattice", B.items, 0, B.lid, B.neib, B.posx, B.posy, B.posz, B.posw)
    call("resetF", B.items, B.Fx, B.Fy, B.Fz, int(num_F))
    call("resetF", B.items, B.Gw, B.Gw, B.Gw, int(num_Gw))


class LockExchange:
    """A LockExchange-ordered run on the reference-compatible entries of
    libipcu, with device buffers held as torch tensors.

    `case` comes from `cases.box_case`; `state` maps the reference driver's
    per-cell arrays (f, g, p, sal, phi, rho, tau, taus, u, v, w over all
    Nt cells; f, g with Q per cell) to host numpy arrays."""

    def __init__(self, case, state, *, slip=1, mrt=True, scalar=True, wall_function=False, boussi=1,
                 rhoL=1.0, rhoH=1000.0, M=None, Minv=None, S=None, MM=None, device="cuda", stream=None):
        import torch

        self.torch = torch
        self.case, self.prec = case, ("f32" if case["dtype"] == np.float32 else "f64")
        dt = torch.float32 if self.prec == "f32" else torch.float64
        dev = torch.device(device)
        T = lambda a, d=dt: torch.as_tensor(np.ascontiguousarray(a), dtype=d, device=dev)
        nt, Q = case["nt"], case["Q"]
        z = lambda n: torch.zeros(n, dtype=dt, device=dev)
        B = SimpleNamespace()
        B.items, B.neib = T(case["items"]), T(case["neib"], torch.int32)
        B.nextB, B.nextK = T(case["nextB"], torch.int32), T(case["nextK"], torch.int32)
        for k in ("posx", "posy", "posz", "delX", "delY"):
            setattr(B, k, T(case[k]))
        for k in ("f", "g", "p", "sal", "phi", "rho", "tau", "taus", "u", "v", "w"):
            setattr(B, k, T(state[k]))
        B.ftmp, B.fout, B.feq, B.Fk = T(state["f"]), T(state["f"]), z(nt * Q), z(nt * Q)
        B.Fx, B.Fy, B.Fz = z(nt), z(nt), z(nt)
        if mrt:
            B.M, B.Minv, B.S, B.MM = T(M), T(Minv), T(S), T(MM)
        else:
            B.M = B.Minv = B.S = B.MM = None
        for a, wl in enumerate(case["walls"]):
            setattr(B, f"w{a + 1}", T(wl if len(wl) else np.zeros(1, np.int32), torch.int32))
        self.B = B
        self.kw = dict(mrt=mrt, scalar=scalar, wall_function=wall_function, boussi=boussi, rhoL=rhoL, rhoH=rhoH,
                       num_F=nt, wall_sizes=tuple(len(w) for w in case["walls"]))
        self.slip, self.nt = slip, nt
        self.stream = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
        self.L = _lib.legacy()

    def _call(self, name, *args):
        _lib.check(self.L(name, self.prec, *args, tail=(self.nt, self.stream)), name)

    def _ip(self, f, feq, ftmp, fout):
        B = self.B
        fn = getattr(_lib.lib(), f"ipcu_IP_process_{self.prec}")
        nb = (self.nt + 63) // 64
        _lib.check(fn(B.items.data_ptr(), nb, 64, B.neib.data_ptr(), f.data_ptr(), feq.data_ptr(),
                      ftmp.data_ptr(), fout.data_ptr(), B.nextB.data_ptr(), B.nextK.data_ptr(), B.posx.data_ptr(),
                      B.posy.data_ptr(), B.delX.data_ptr(), B.delY.data_ptr(), int(self.slip), self.stream),
                   "IP_process")

    def step(self, n=1):
        for _ in range(int(n)):
            le_step(self._call, self._ip, self.B, **self.kw)

    def get(self, name):
        self.torch.cuda.synchronize()
        return getattr(self.B, name).detach().cpu().numpy().copy()
