"""Checkpoint/restore and the reference-format CSV writers of the structured
solvers: a run restored from a snapshot continues bit-identically (FP32 and
FP16 storage, with a moving body, and the 3-D solver), the field CSV has the
reference's header, columns and cell order (ref: function/basic.cu:16-28)
and the marker CSV its IB_csv columns (ref: function/ibm.cu:3-14)."""
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


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_restore_with_moving_body_continues_bit_identically(cuda, tmp_path, storage):
    """The snapshot holds the attached body (its description and device
    state: rigid-body state, previous stencil footprints, force density,
    tile flags), so a settling ellipse resumes bit for bit."""
    from ip_cu_lbm_b200.cases import d2q9_mrt

    M, Minv, S = d2q9_mrt()
    kw = dict(q_scalar=0, geometry="uniform", wall="bb", tau=0.56, rho_sal=0.0, g_bouss=0.0, storage=storage, M=M,
              Minv=Minv, S=S)
    a = Sim(64, 96, **kw)
    a.attach_ellipse(32.0, 60.0, 8.0, 4.0, markers=48, theta=np.pi / 4, rho_s=1.5, gravity=1e-4)
    a.step(40)
    snap = tmp_path / "body.ipcu"
    a.save(snap)
    a.step(30)
    b = Sim.load(snap)
    assert b.steps() == 40
    b.step(30)
    assert a.body() == b.body()
    for fld in ("f", "ux", "uz", "ibfx", "ibfz"):
        assert np.array_equal(a.get(fld), b.get(fld)), fld
    assert np.array_equal(a.markers(), b.markers())
    assert a.status() == 0 and b.status() == 0


def test_ib_csv_in_reference_format(cuda, tmp_path):
    """Markers in the reference's IB_csv columns (ref: function/ibm.cu:3-14):
    position, velocity and the force each marker put on the fluid, which sum
    to the body's IB force."""
    from ip_cu_lbm_b200.cases import d2q9_mrt

    M, Minv, S = d2q9_mrt()
    s = Sim(64, 96, q_scalar=0, tau=0.56, rho_sal=0.0, g_bouss=0.0, M=M, Minv=Minv, S=S)
    s.attach_ellipse(32.0, 60.0, 8.0, 4.0, markers=48, theta=np.pi / 4, rho_s=1.5, gravity=1e-4)
    s.step(25)
    path = tmp_path / "ibm_0001.csv"
    s.write_ib_csv(path)
    lines = path.read_text().splitlines()
    assert lines[0] == "x,y,z,velx,vely,velz,ax,ay,az"
    rows = np.array([[float(v) for v in ln.split(",")] for ln in lines[1:]])
    assert rows.shape == (48, 9)
    m = s.markers()
    np.testing.assert_allclose(rows, m, rtol=1e-5, atol=1e-12)
    b = s.body()
    np.testing.assert_allclose(m[:, [0, 2]].mean(0), [b["x"], b["z"]], atol=1e-9)
    # the markers' forces sum to the body's IB force (FP64 sum of the same values)
    assert abs(m[:, 6].sum() - b["Fx"]) <= 1e-5 * np.abs(m[:, 6]).sum() + 1e-15
    assert abs(m[:, 8].sum() - b["Fz"]) <= 1e-5 * np.abs(m[:, 8]).sum() + 1e-15
    np.testing.assert_allclose(m[:, 1], 0.5)


def test_3d_restore_continues_bit_identically(cuda, tmp_path):
    from ip_cu_lbm_b200.sim3d import Sim3D
    from ip_cu_lbm_b200.workloads import centre_clustered_axis

    nx, ny, nz = 40, 24, 12
    x, wx = centre_clustered_axis(nx)
    y, wy = centre_clustered_axis(ny)
    S0 = np.linspace(0.2, 0.8, nx * ny * nz)
    a = Sim3D(nx, ny, nz, x=x, wx=wx, y=y, wy=wy, ns=3, tau=0.58, taus=0.53, rho_sal=1e-3, g_bouss=1e-4, s0=S0)
    a.step(10)
    snap = tmp_path / "box3d.ipcu"
    a.save(snap)
    a.step(10)
    b = Sim3D.load(snap)
    assert b.steps() == 10 and (b.nx, b.ny, b.nz) == (nx, ny, nz)
    b.step(10)
    for fld in ("f", "g", "F"):
        assert np.array_equal(a.get(fld), b.get(fld)), fld


def test_3d_version_1_snapshot_still_loads(cuda, tmp_path):
    """A version 1 file (FP32 state, the configuration without its storage
    field) restores and continues bit for bit: written here by taking a
    version 2 file apart (magic, version, configuration, then the rest)."""
    import ctypes

    from ip_cu_lbm_b200 import _lib
    from ip_cu_lbm_b200.sim3d import Sim3D

    nx, ny, nz = 24, 16, 10
    S0 = np.linspace(0.2, 0.8, nx * ny * nz)
    a = Sim3D(nx, ny, nz, tau=0.58, taus=0.53, rho_sal=1e-3, g_bouss=1e-4, s0=S0)
    a.step(10)
    v2 = tmp_path / "v2.ipcu3"
    a.save(v2)
    raw = v2.read_bytes()
    cfg = ctypes.sizeof(_lib.Sim3DConfig)
    storage_at = _lib.Sim3DConfig.storage.offset
    assert int.from_bytes(raw[8:12], "little") == 2
    v1 = raw[:8] + (1).to_bytes(4, "little") + raw[12:12 + storage_at] + raw[12 + cfg:]
    (tmp_path / "v1.ipcu3").write_bytes(v1)
    a.step(10)
    b = Sim3D.load(tmp_path / "v1.ipcu3")
    assert b.storage == "f32" and b.steps() == 10
    b.step(10)
    for fld in ("f", "g", "F"):
        assert np.array_equal(a.get(fld), b.get(fld)), fld
    a.close()
    b.close()
