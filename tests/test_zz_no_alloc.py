"""The allocation-free totals entry point (ipcu_totals_noalloc_f32).

Some callers cannot allocate device memory where they need the domain
totals: hosts that hand all device memory to their own pool, loops that must
not enter the driver's allocator.
For them the library keeps the reduction's scratch in a fixed device array.
This file checks, through the C ABI, that two calls in a row return the same
totals as the allocating path (ipcu_sim_totals, same FP64 reduction) within
1e-12 relative, that a call captured in a CUDA graph replays to the same
totals, and that fields beyond the fixed scratch are rejected. It is
collected last (test_zz_...) so a failure here comes after every other test,
and it runs alone in a fresh process as well as after the others.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sim(nx, nz):
    from ip_cu_lbm_b200 import Sim

    wz = np.linspace(1.0, 3.0, nz)
    z = np.cumsum(wz) - wz / 2
    S0 = np.where(np.arange(nx)[None, :] < nx // 3, 1.0, 0.25) * np.ones((nz, 1))
    s = Sim(nx, nz, q_scalar=5, geometry="z3", z=z, wz=wz, g_bouss=1e-3, rho_sal=1e-3, tau=0.55, taus=0.52,
            s0=S0.ravel())
    s.step(40)
    return s, wz


def test_noalloc_totals_match_allocating_path(cuda):
    import torch

    from ip_cu_lbm_b200 import _lib

    L = _lib.lib()
    fn = L.ipcu_totals_noalloc_f32
    fn.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    nx, nz = 300, 70
    s, wz = _sim(nx, nz)
    ref_p, ref_s = s.totals()
    f_ptr, _, mac_ptr = s.device_state()
    wx_d = torch.ones(nx, dtype=torch.float32, device=cuda)
    wz_d = torch.as_tensor(wz.astype(np.float32), device=cuda)
    out = torch.zeros(2, dtype=torch.float64, device=cuda)
    stream = torch.cuda.current_stream(cuda)
    s.sync()
    # p* totals cancel (positive and negative populations): compare against the
    # magnitude of the summands, not of the sum
    area = np.outer(wz, np.ones(nx))
    p_scale = float((np.abs(s.get("p")) * area).sum())
    for call in range(2):
        out.fill_(float("nan"))
        rc = fn(f_ptr, mac_ptr, wx_d.data_ptr(), wz_d.data_ptr(), nx, nz, out.data_ptr(), stream.cuda_stream)
        assert rc == 0, f"call {call}: status {rc}"
        torch.cuda.synchronize()
        got_p, got_s = out.cpu().tolist()
        assert abs(got_s - ref_s) <= 1e-12 * abs(ref_s), (call, got_s, ref_s)
        assert abs(got_p - ref_p) <= 1e-12 * p_scale, (call, got_p, ref_p, p_scale)
    # the launches can be captured once the scratch address is resolved: a
    # graph replay gives the same totals
    graph = torch.cuda.CUDAGraph()
    cs = torch.cuda.Stream(cuda)
    with torch.cuda.graph(graph, stream=cs):
        rc = fn(f_ptr, mac_ptr, wx_d.data_ptr(), wz_d.data_ptr(), nx, nz, out.data_ptr(), cs.cuda_stream)
    assert rc == 0, f"captured call: status {rc}"
    out.fill_(float("nan"))
    torch.cuda.synchronize()
    graph.replay()
    torch.cuda.synchronize()
    got_p, got_s = out.cpu().tolist()
    assert abs(got_s - ref_s) <= 1e-12 * abs(ref_s), ("replay", got_s, ref_s)
    assert abs(got_p - ref_p) <= 1e-12 * p_scale, ("replay", got_p, ref_p, p_scale)
    del graph
    # beyond the fixed scratch: rejected before any launch
    rc = fn(f_ptr, mac_ptr, wx_d.data_ptr(), wz_d.data_ptr(), 8192, 4097, out.data_ptr(), stream.cuda_stream)
    assert rc == -4, rc  # IPCU_ERR_CAPACITY
    s.close()
