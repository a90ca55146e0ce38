"""The kernels' per-block logic, compiled for the host (tests/host_emu/emu.cu), against the oracle - no GPU needed.

This catches logic and float-order mistakes in the device code on the CPU. The GPU parity tests remain the
authority: they run the real kernels on the device.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle_lib
from oracle_lib import BC1, BC3, BC4, BC5, BC7

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "host_emu", "emu.cu")
OUT = os.path.join(ROOT, "_build", "host_emu", "libztc_emu.so")
DEPS = [SRC] + [os.path.join(ROOT, "zap_b200", "csrc", f) for f in os.listdir(os.path.join(ROOT, "zap_b200", "csrc"))
                if f.endswith((".cu", ".cuh", ".h"))]


@pytest.fixture(scope="module")
def emu():
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not available")
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(p) for p in DEPS):
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        subprocess.run(["nvcc", "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-fmad=false",
                        "-diag-suppress", "20091", "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-fPIC", "-shared",
                        "-o", OUT, SRC], check=True, capture_output=True)
    lib = C.CDLL(OUT)
    vp, i, sz = C.c_void_p, C.c_int, C.c_size_t
    lib.emu_bc_encode.argtypes = [vp, i, i, sz, i, vp, vp]
    lib.emu_bc6h_encode.argtypes = [vp, i, i, sz, vp]
    lib.emu_astc_encode.argtypes = [vp, i, i, sz, vp, vp]
    lib.emu_mip_next.argtypes = [vp, i, i, sz, i, vp, sz]
    lib.emu_div255_mismatches.argtypes = [C.c_uint64, C.c_uint64]
    lib.emu_div255_mismatches.restype = C.c_uint64
    lib.emu_bc6_nearest_mismatches.argtypes = [C.c_uint64, C.c_uint64]
    lib.emu_bc6_nearest_mismatches.restype = C.c_uint64
    lib.emu_div_small_mismatches.argtypes = [i]
    lib.emu_div_small_mismatches.restype = C.c_uint64
    lib.emu_srgb_search_mismatches.argtypes = [C.c_uint64, C.c_uint64]
    lib.emu_srgb_search_mismatches.restype = C.c_uint64
    lib.emu_lerp4_mismatches.argtypes = []
    lib.emu_lerp4_mismatches.restype = C.c_uint64
    return lib


def _images():
    import zap_b200.synth as S
    rng = np.random.default_rng(5)
    noise = rng.integers(0, 256, (33, 45, 4), dtype=np.uint8)
    opaque = noise.copy()
    opaque[..., 3] = 255
    return [S.colour_texture(96, 72, seed=1).numpy(), S.colour_texture(61, 37, seed=2, alpha="noise").numpy(), noise, opaque]


def _blocks(a, bs):
    return a.reshape(-1, bs)


def test_bcn_block_logic(emu, oracle):
    for img in _images():
        h, w = img.shape[:2]
        for fmt in (BC1, BC3, BC4, BC5):
            out = np.zeros(oracle_lib.bc_size(w, h, fmt), np.uint8)
            emu.emu_bc_encode(img.ctypes.data, w, h, w * 4, fmt, out.ctypes.data, None)
            assert np.array_equal(out, oracle.bc_encode(img, fmt)), (fmt, w, h)


def test_bc7_mode6_block_logic(emu, oracle):
    for img in _images():
        h, w = img.shape[:2]
        out = np.zeros(oracle_lib.bc_size(w, h, BC7), np.uint8)
        hard = np.zeros(out.size // 16, np.uint8)
        emu.emu_bc_encode(img.ctypes.data, w, h, w * 4, BC7, out.ctypes.data, hard.ctypes.data)
        ref = oracle.bc_encode(img, BC7)
        easy = hard == 0
        assert np.array_equal(_blocks(out, 16)[easy], _blocks(ref, 16)[easy])


def test_bc6h_block_logic(emu, oracle, golden):
    import zap_b200.synth as S
    imgs = [golden["himg/" + k[5:]] for k in golden if k.startswith("himg/")]
    half = S.hdr_texture(40, 24, seed=2).numpy()
    rgba = np.ones((24, 40, 4), np.float32)
    rgba[..., :3] = half.astype(np.float32)
    imgs.append(rgba)
    for img in imgs:
        img = np.ascontiguousarray(img, np.float32)
        h, w = img.shape[:2]
        out = np.zeros(oracle_lib.bc_size(w, h, BC7), np.uint8)
        emu.emu_bc6h_encode(img.ctypes.data, w, h, w * 4, out.ctypes.data)
        ref = oracle.bc6h_encode(img)
        bad = np.nonzero(np.any(_blocks(out, 16) != _blocks(ref, 16), axis=1))[0]
        assert bad.size == 0, (w, h, bad[:8])


def test_astc_single_partition_block_logic(emu, oracle):
    for img in _images():
        h, w = img.shape[:2]
        out = np.zeros(oracle_lib.bc_size(w, h, BC7), np.uint8)
        hard = np.zeros(out.size // 16, np.uint8)
        emu.emu_astc_encode(img.ctypes.data, w, h, w * 4, out.ctypes.data, hard.ctypes.data)
        ref = oracle.astc_encode(img)
        easy = hard == 0
        assert np.array_equal(_blocks(out, 16)[easy], _blocks(ref, 16)[easy]), (w, h)


def test_mip_block_logic(emu, oracle):
    for img in _images():
        h, w = img.shape[:2]
        for srgb in (0, 1):
            nw, nh = max(1, w // 2), max(1, h // 2)
            out = np.zeros((nh, nw, 4), np.uint8)
            emu.emu_mip_next(img.ctypes.data, w, h, w * 4, srgb, out.ctypes.data, nw * 4)
            assert np.array_equal(out, oracle.mip_next(img, srgb))


def test_bc6h_block_logic_extreme_values(emu, oracle):
    """Negative, NaN, +inf, tiny (half-subnormal) and huge (clamped) floats in one image."""
    rng = np.random.default_rng(4)
    wild = (2.0 ** rng.uniform(-30, 20, (37, 29, 4))).astype(np.float32)
    wild[::3, ::2, 1] *= -1
    wild[5, 5, 0] = np.inf
    wild[6, 6, 2] = np.nan
    h, w = wild.shape[:2]
    out = np.zeros(oracle_lib.bc_size(w, h, BC7), np.uint8)
    emu.emu_bc6h_encode(wild.ctypes.data, w, h, w * 4, out.ctypes.data)
    assert np.array_equal(out, oracle.bc6h_encode(wild))


def test_div255_equals_division_for_every_float(emu):
    """The quantisers divide by 255 with Markstein's FMA correction instead of a division; that must give the
    correctly rounded quotient, bit for bit, for all 2^32 bit patterns (non-finite ones and -0 skipped)."""
    from concurrent.futures import ThreadPoolExecutor
    chunks = 64
    step = (1 << 32) // chunks
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        bad = sum(ex.map(lambda k: emu.emu_div255_mismatches(k * step, (k + 1) * step), range(chunks)))
    assert bad == 0


def test_bc6h_nearest_endpoint_for_every_float(emu):
    """BC6H's nearest 10-bit endpoint clamps its guess before truncating it without a conversion; it must pick the
    reference's endpoint for all 2^32 bit patterns of the pre-finish value, NaN, infinities and negatives included."""
    from concurrent.futures import ThreadPoolExecutor
    chunks = 64
    step = (1 << 32) // chunks
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        bad = sum(ex.map(lambda k: emu.emu_bc6_nearest_mismatches(k * step, (k + 1) * step), range(chunks)))
    assert bad == 0


def test_small_divisor_division_equals_ieee_on_its_domain(emu):
    """The partition scores and subset means divide integer-valued floats below 2^24 by counts 1..16, and the BC6H
    texel load divides 64 h (h a half's bits) by 31, with the same FMA correction; every such pair must give the IEEE
    quotient bit for bit."""
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        bad = sum(ex.map(emu.emu_div_small_mismatches, list(range(1, 17)) + [31]))
    assert bad == 0


def test_srgb_bucket_search_equals_binary_search(emu):
    """The mip generator maps a linear value back to sRGB by scanning from a per-bucket start instead of the
    reference's binary search; both must give the same code for every float in [0, 1] (the averages the generator
    forms lie there) and for the negative, above-one and infinite values around it."""
    from concurrent.futures import ThreadPoolExecutor
    top = 0x3F800001  # bit patterns 0 .. 1.0f
    chunks = 64
    step = (top + chunks - 1) // chunks
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        bad = sum(ex.map(lambda k: emu.emu_srgb_search_mismatches(k * step, min(top, (k + 1) * step)), range(chunks)))
    bad += emu.emu_srgb_search_mismatches(0x3F800001, 0x3F800001 + (1 << 20))  # just above 1
    bad += emu.emu_srgb_search_mismatches(0x7F800000, 0x7F800001)  # +inf
    bad += emu.emu_srgb_search_mismatches(0x80000000, 0x80000000 + (1 << 20))  # -0 and small negatives
    assert bad == 0


def test_packed_lerp_equals_lerp64(emu):
    """The encoders build BC7 palettes with two channels per 32-bit word (one multiply-add for R and B, one for G
    and A); every endpoint pair and weight must give lerp64's bytes, including negative slopes that borrow across
    the fields."""
    assert emu.emu_lerp4_mismatches() == 0
