"""Host-side sizing of served requests (no GPU): the admission budget counts
the device bytes a request will hold, for 3-D requests the per-cell state
of ipcu_sim3d_bytes_per_cell (232 B FP32, 148 B with 16-bit storage: two
buffers of f, g, the FP32 force planes and the 16-bit reference planes)
plus a sphere's force density and update scratch."""
from ip_cu_lbm_b200.serving import request_bytes, stratified_box_request


def test_3d_request_bytes_follow_the_storage():
    nx, ny, nz = 32, 24, 40
    cells = nx * ny * nz
    f32 = stratified_box_request(0, nx, ny, nz, 10, sphere=False)
    f16 = stratified_box_request(1, nx, ny, nz, 10, sphere=False, storage="f16")
    bf16 = stratified_box_request(2, nx, ny, nz, 10, sphere=False, storage="bf16")
    assert request_bytes(f32) == 2 * 4 * (19 + 7 + 3) * cells == 232 * cells
    assert request_bytes(f16) == request_bytes(bf16) == 2 * (2 * (19 + 7 + 5) + 4 * 3) * cells == 148 * cells
    with_sphere = stratified_box_request(3, nx, ny, nz, 10)
    assert request_bytes(with_sphere) == 232 * cells + 12 * cells + (4 << 20)
    assert f16.kwargs["storage"] == "f16" and "storage" not in f32.kwargs
