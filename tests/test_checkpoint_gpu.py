"""Checkpoint/restore and the reference-format CSV writer of the structured
solver: a run restored from a snapshot continues bit-identically (FP32 and
FP16 storage), and the CSV has the reference's header, columns and cell
order (ref: function/basic.cu:16-28)."""
import numpy as np
import pytest

from ip_cu_lbm_b200 import Sim

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_restore_continues_bit_identically(cuda, tmp_path, storage):
    nx, nz = 80, 40
    wz = np.linspace(1.0, 2.0, nz)
    kw = dict(q_scalar=5, geometry="z3", storage=storage, z=np.cumsum(wz) - wz / 2, wz=wz, g_bouss=1e-3,
              rho_sal=1e-3, tau=0.55, taus=0.52)
    S0 = (np.arange(nx)[None, :] < nx // 2) * np.ones((nz, 1), float)
    a = Sim(nx, nz, s0=S0.ravel(), **kw)
    a.step(20)
    snap = tmp_path / "state.ipcu"
    a.save(snap)
    a.step(30)
    b = Sim.load(snap)
    assert b.steps() == 20 and (b.nx, b.nz) == (nx, nz)
    b.step(30)
    assert a.steps() == b.steps() == 50
    for fld in ("f", "g", "S", "ux", "uz"):
        assert np.array_equal(a.get(fld), b.get(fld)), fld


def test_csv_in_reference_format(cuda, tmp_path):
    nx, nz = 12, 5
    s = Sim(nx, nz, q_scalar=5, s0=np.linspace(0, 1, nx * nz), g_bouss=1e-3, rho_sal=1e-3)
    s.step(3)
    path = tmp_path / "Fakhari_LBM0001.csv"
    s.write_csv(path)
    lines = path.read_text().splitlines()
    assert lines[0] == f"num_calc,{nx * nz}"
    assert [c.strip() for c in lines[1].split(",")] == ["x", "y", "z", "delx", "dely", "pressure", "salinity", "phi",
                                                        "rho", "u", "v", "w", "Fx", "Fy", "Fz"]
    rows = np.array([[float(v) for v in ln.split(",")] for ln in lines[2:]])
    assert rows.shape == (nx * nz, 15)
    # reference cell order: x-major, z fastest
    np.testing.assert_allclose(rows[:nz, 0], 0.5)
    np.testing.assert_allclose(rows[:nz, 2], np.arange(nz) + 0.5)
    np.testing.assert_allclose(rows[:, 6], s.get("S").T.ravel(), atol=1e-6)
