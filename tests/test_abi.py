"""The C-ABI libraries load and export every entry point include/*.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT
from ip_cu_lbm_b200 import _abi, _lib

HEADERS = [os.path.join(ROOT, "include", h) for h in ("ipcu.h", "ipcu_sim.h", "ipcu_sim3d.h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        # macro-generated per-precision entries: ipcu_<name>_##S(
        for m in re.finditer(r"\bipcu_(\w+?)_##S\s*\(", src):
            names.add(f"ipcu_{m.group(1)}_f32")
            names.add(f"ipcu_{m.group(1)}_f64")
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(ipcu_\w+)\s*\(", src, flags=re.M):
            if "##" not in m.group(0):
                names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_reference_api():
    names = set(declared_symbols())
    for k in _abi.LEGACY:
        assert f"ipcu_{k}_f32" in names and f"ipcu_{k}_f64" in names, k
    for k in _abi.FLOAT_ONLY:
        assert f"ipcu_{k}_f32" in names, k
    assert "ipcu_IP_process_f32" in names and "ipcu_sim_step" in names


def test_libipcu_exports_every_declared_symbol():
    L = _lib.lib()
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing


def test_libipcu_host_helpers_without_gpu():
    L = _lib.lib()
    assert L.ipcu_version() >= 100
    assert L.ipcu_status_string(-4) == b"output capacity too small"


def test_oracle_exports_every_reference_kernel():
    from oracle import oracle as _o

    L = ctypes.CDLL(_o.ORACLE_SO)
    for k in _abi.LEGACY:
        for p in ("f32", "f64"):
            assert hasattr(L, f"oracle_{k}_{p}"), k
    assert hasattr(L, "oracle_IP_process_f32") and hasattr(L, "oracle_IB_directForcing_f32")


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libipcu_ref.so")),
                    reason="reference build (oracle/_ref) not present")
def test_reference_harness_exports():
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libipcu_ref.so"))
    for k in _abi.LEGACY:
        precs = ("f32",) if k in _abi.REF_FLOAT_ONLY else ("f32", "f64")
        for p in precs:
            assert hasattr(L, f"ref_{k}_{p}"), k


# the ctypes mirrors of the header's structs, field by field
MIRRORS = [("ipcu_sim_config", "SimConfig"), ("ipcu_ib_body2d", "IBBody2D"), ("ipcu_ib_sphere3d", "IBSphere3D"),
           ("ipcu_sim3d_axes", "Sim3DAxes"), ("ipcu_sim3d_config", "Sim3DConfig")]


def test_ctypes_mirrors_match_the_header_layout(tmp_path):
    """Size and every field offset of each mirrored struct, as the C
    compiler lays them out from include/ipcu.h (gcc on the host)."""
    import shutil
    import subprocess

    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no host C compiler")
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "ipcu.h"', "int main(void) {"]
    for cname, pyname in MIRRORS:
        cls = getattr(_lib, pyname)
        lines.append(f'  printf("{pyname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{pyname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln.strip():
            name, field, val = ln.split()
            got[(name, field)] = int(val)
    for _, pyname in MIRRORS:
        cls = getattr(_lib, pyname)
        assert got[(pyname, "size")] == ctypes.sizeof(cls), pyname
        for fname, _ in cls._fields_:
            assert got[(pyname, fname)] == getattr(cls, fname).offset, (pyname, fname)

