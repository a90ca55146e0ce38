"""The C ABI without a GPU: the library loads, exports every entry point include/*.h declares, and a C11 caller
compiles against the header. Compute calls are not made here (no device); they must fail with a status, not crash."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include"))) if f.endswith(".h")]


def declared_functions():
    names = []
    for h in HEADERS:
        text = open(h).read()
        names += re.findall(r"ZTC_API\s+[\w\s\*]+?\b(zap_tex_cuda_\w+)\s*\(", text)
    return sorted(set(names))


def test_built_library_is_current():
    """The in-tree library must be rebuilt after any source change (zap_b200.build())."""
    import zap_b200
    lib = zap_b200._lib.LIB_PATH
    if not os.path.exists(lib):
        zap_b200.build()
    csrc = os.path.join(ROOT, "zap_b200", "csrc")
    sources = [os.path.join(csrc, f) for f in os.listdir(csrc) if f.endswith((".cu", ".cuh", ".h"))] + HEADERS
    newer = [os.path.basename(s) for s in sources if os.path.getmtime(s) > os.path.getmtime(lib)]
    assert not newer, f"rebuild zap_b200 (make -C zap_b200/csrc): {newer} changed after the library was built"


def test_header_declares_entry_points():
    names = declared_functions()
    assert "zap_tex_cuda_bc_encode" in names and "zap_tex_cuda_bc6h_encode" in names and "zap_tex_cuda_astc_encode" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    import zap_b200
    lib = zap_b200.load()
    out = subprocess.run(["nm", "-D", "--defined-only", zap_b200._lib.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (zap_tex_cuda_\w+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        getattr(lib, n)  # resolvable through ctypes too


def test_python_binding_covers_the_header():
    import zap_b200._lib as L
    assert sorted(L.exported_names()) == declared_functions()


def test_c11_caller_compiles_and_links(tmp_path):
    import zap_b200
    src = tmp_path / "caller.c"
    src.write_text(
        '#include "zap_tex_cuda.h"\n#include <stdio.h>\n#include <string.h>\n'
        "int main(void) {\n"
        "  uint8_t rgba[16 * 4], out[16];\n  memset(rgba, 128, sizeof rgba);\n"
        "  int st = zap_tex_cuda_bc_encode(NULL, rgba, 4, 4, 16, ZTC_BC7, 0.0f, out);\n"
        '  printf("%d %zu %d %s\\n", st, zap_tex_cuda_bc_size(5, 3, ZTC_BC1), zap_tex_cuda_mip_levels(256, 128),\n'
        "         zap_tex_cuda_status_string(st));\n  return 0;\n}\n")
    exe = tmp_path / "caller"
    lib = zap_b200._lib.LIB_PATH
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    lib, "-Wl,-rpath," + os.path.dirname(lib)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    st, size, levels = r.stdout.split()[:3]
    assert size == "16" and levels == "9"
    import torch
    if not torch.cuda.is_available():
        assert st == "-6"  # no usable device: a status, never a CPU fallback


def test_host_api_rejects_bad_arguments_without_device():
    import numpy as np
    import zap_b200
    lib = zap_b200.load()
    img = np.zeros((8, 8, 4), np.uint8)
    out = np.zeros(64, np.uint8)
    assert lib.zap_tex_cuda_bc_encode(None, img.ctypes.data, 0, 8, 32, 0, 0.0, out.ctypes.data) == -1
    assert lib.zap_tex_cuda_bc_encode(None, None, 8, 8, 32, 0, 0.0, out.ctypes.data) == -1
    assert lib.zap_tex_cuda_bc_encode(None, img.ctypes.data, 8, 8, 32, 7, 0.0, out.ctypes.data) == -2  # no such format
    assert lib.zap_tex_cuda_bc_encode(None, img.ctypes.data, 8, 8, 32, 0, float("nan"), out.ctypes.data) == -1
    assert zap_b200.bc_size(0, 4, 0) == 0 and zap_b200.mip_levels(5, 3) == 3 and zap_b200.block_bytes(4) == 16


@pytest.mark.parametrize("w,h", [(1, 1), (256, 128), (5, 3), (4096, 1)])
def test_mip_levels_matches_oracle(oracle, w, h):
    import zap_b200
    assert zap_b200.mip_levels(w, h) == oracle.mip_levels(w, h)
