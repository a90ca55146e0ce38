"""Host code under AddressSanitizer and UndefinedBehaviorSanitizer, no GPU needed.

- The C ABI's host paths (tests/host_emu/abi_driver.c) against the library built with its host code instrumented
  (make -C zap_b200/csrc sanitize -> libzap_tex_cuda_san.so): size helpers, container headers, status strings, the
  trace record, the test hooks, every entry point's argument checks, and the no-device statuses. Leak detection on.
- The kernels' per-block logic compiled for the host (tests/host_emu/emu.cu) with the same instrumentation, run by
  tests/host_emu/emu_driver.c over images written here, its output checked against the oracle.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle_lib
from oracle_lib import BC1, BC3, BC4, BC5, BC7

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU_DIR = os.path.join(ROOT, "tests", "host_emu")
BUILD = os.path.join(ROOT, "_build", "host_san")
SAN_FLAGS = ["-fsanitize=address", "-fsanitize=undefined", "-fno-omit-frame-pointer", "-fno-sanitize-recover=undefined"]
ENV = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:protect_shadow_gap=0:abort_on_error=0",
           UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")

pytestmark = pytest.mark.skipif(shutil.which("nvcc") is None or shutil.which("gcc") is None, reason="nvcc and gcc needed")


def _clean(r):
    text = r.stdout + r.stderr
    assert "AddressSanitizer" not in text and "LeakSanitizer" not in text and "runtime error" not in text, text[-4000:]
    assert r.returncode == 0, text[-4000:]


def test_abi_host_paths_under_sanitizers():
    import torch
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "zap_b200", "csrc"), "-j", str(min(8, os.cpu_count() or 1)), "sanitize"],
                   check=True, capture_output=True)
    lib = os.path.join(ROOT, "zap_b200", "lib", "libzap_tex_cuda_san.so")
    os.makedirs(BUILD, exist_ok=True)
    exe = os.path.join(BUILD, "abi_driver")
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", *SAN_FLAGS, "-I", os.path.join(ROOT, "include"),
                    os.path.join(EMU_DIR, "abi_driver.c"), "-o", exe, lib, "-Wl,-rpath," + os.path.dirname(lib), "-lm"], check=True)
    r = subprocess.run([exe] + (["gpu"] if torch.cuda.is_available() else []), capture_output=True, text=True, env=ENV, timeout=300)
    _clean(r)
    assert r.stdout.strip() == "ok"


def _images():
    rng = np.random.default_rng(21)
    noise = rng.integers(0, 256, (29, 37, 4), dtype=np.uint8)
    opaque = noise.copy()
    opaque[..., 3] = 255
    y, x = np.mgrid[0:40, 0:52]
    smooth = np.stack([x * 4, y * 5, (x + y) * 2, 255 - x], -1).clip(0, 255).astype(np.uint8)
    hdr = (2.0 ** rng.uniform(-12, 10, (21, 23, 4))).astype(np.float32)
    hdr[::4, ::3, 1] *= -1
    return [noise, opaque, smooth, np.ones((1, 1, 4), np.uint8) * 77], [hdr]


def test_block_logic_under_sanitizers(oracle, tmp_path):
    os.makedirs(BUILD, exist_ok=True)
    emu = os.path.join(BUILD, "libztc_emu_san.so")
    deps = [os.path.join(EMU_DIR, "emu.cu")] + [os.path.join(ROOT, "zap_b200", "csrc", f) for f in os.listdir(os.path.join(ROOT, "zap_b200", "csrc"))
                                                if f.endswith((".cu", ".cuh", ".h"))]
    if not os.path.exists(emu) or os.path.getmtime(emu) < max(os.path.getmtime(p) for p in deps):
        subprocess.run(["nvcc", "-O1", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-fmad=false", "-diag-suppress", "20091",
                        "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-fPIC", *sum((["-Xcompiler", f] for f in SAN_FLAGS), []),
                        "-shared", "-o", emu, os.path.join(EMU_DIR, "emu.cu")], check=True, capture_output=True)
    exe = os.path.join(BUILD, "emu_driver")
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", *SAN_FLAGS, os.path.join(EMU_DIR, "emu_driver.c"), "-o", exe, emu,
                    "-Wl,-rpath," + BUILD], check=True)
    u8, f32 = _images()
    src = tmp_path / "in.bin"
    with open(src, "wb") as f:
        for img in u8:
            f.write(np.array([img.shape[1], img.shape[0], 0], np.int32).tobytes() + np.ascontiguousarray(img).tobytes())
        for img in f32:
            f.write(np.array([img.shape[1], img.shape[0], 1], np.int32).tobytes() + np.ascontiguousarray(img).tobytes())
    dst = tmp_path / "out.bin"
    r = subprocess.run([exe, str(src), str(dst)], capture_output=True, text=True, env=ENV, timeout=600)
    _clean(r)
    got = np.fromfile(dst, np.uint8)
    off = 0

    def take(n):
        nonlocal off
        off += n
        return got[off - n:off]
    for img in u8:
        h, w = img.shape[:2]
        nb = ((w + 3) // 4) * ((h + 3) // 4)
        for fmt in (BC1, BC3, BC4, BC5, BC7):
            blocks = take(oracle_lib.bc_size(w, h, fmt))
            want = oracle.bc_encode(img, fmt)
            if fmt == BC7:  # mode-6 blocks exactly; the rest go to the second phase, which is device-only
                easy = take(nb) == 0
                assert np.array_equal(blocks.reshape(-1, 16)[easy], want.reshape(-1, 16)[easy]), (w, h)
            else:
                assert np.array_equal(blocks, want), (fmt, w, h)
        blocks, easy = take(nb * 16), take(nb) == 0
        assert np.array_equal(blocks.reshape(-1, 16)[easy], oracle.astc_encode(img).reshape(-1, 16)[easy]), (w, h)
        for srgb in (0, 1):
            mip = oracle.mip_next(img, srgb)
            assert np.array_equal(take(mip.size), mip.reshape(-1)), (w, h, srgb)
    for img in f32:
        h, w = img.shape[:2]
        assert np.array_equal(take(oracle_lib.bc_size(w, h, BC7)), oracle.bc6h_encode(img))
    assert off == got.size
