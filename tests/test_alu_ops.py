"""The op-counting build of the oracle (oracle/count_ops.py, the ALU roofline's numerator), on the CPU.

Counting must not change the restatement's output, the count must match a closed form where one exists (BC4: 9
endpoint candidates x 16 texels x 8 entries x 4 ops per block without a solid block), and the committed table must
name the kernels bench.py looks up.
"""
import ctypes as C
import json
import os
import subprocess

import numpy as np

import oracle_lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _ops_lib():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ops"], check=True, stdout=subprocess.DEVNULL)
    lib = C.CDLL(os.path.join(ROOT, "oracle", "liboracle_ops.so"))
    lib.zo_bc_encode.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_size_t, C.c_int, C.c_float, C.c_void_p]
    lib.zo_ops_take.argtypes = [C.POINTER(C.c_uint64)]
    return lib


def _encode(lib, img, fmt):
    h, w = img.shape[:2]
    out = np.zeros(oracle_lib.bc_size(w, h, fmt), np.uint8)
    ops = (C.c_uint64 * 2)()
    lib.zo_ops_take(ops)
    lib.zo_bc_encode(img.ctypes.data, w, h, w * 4, fmt, 0.0, out.ctypes.data)
    lib.zo_ops_take(ops)
    return out, int(ops[0]), int(ops[1])


def test_counting_build_matches_the_oracle(oracle):
    import zap_b200.synth as S
    lib = _ops_lib()
    img = np.ascontiguousarray(S.colour_texture(64, 48, seed=3, alpha="noise").numpy())
    for fmt in (oracle_lib.BC1, oracle_lib.BC3, oracle_lib.BC4, oracle_lib.BC5, oracle_lib.BC7):
        out, ops, m6 = _encode(lib, img, fmt)
        assert np.array_equal(out, oracle.bc_encode(img, fmt)), fmt
        assert ops > 0
        assert (m6 > 0) == (fmt == oracle_lib.BC7) and m6 <= ops
        assert _encode(lib, img, fmt)[1:] == (ops, m6)  # deterministic


def test_bc4_count_has_closed_form():
    rng = np.random.default_rng(0)
    img = rng.integers(0, 256, (32, 32, 4), dtype=np.uint8)
    img[::4, ::4, 0] = 0
    img[1::4, 1::4, 0] = 255  # every block spans 0..255: no solid block
    _, ops, _ = _encode(_ops_lib(), img, oracle_lib.BC4)
    assert ops == 64 * 9 * 16 * 8 * 4


def test_committed_table_names_the_bench_kernels():
    with open(os.path.join(ROOT, "profiles", "alu_ops.json")) as f:
        table = json.load(f)
    assert set(table["bc7"]["ops_per_texture"]) == {"bc7_mode6", "bc7_modes51"}
    assert set(table["bc1"]["ops_per_texture"]) == {"bc1_encode"}
    assert table["bc7"]["ops_per_texture"]["bc7_mode6"] > table["bc7"]["ops_per_texture"]["bc7_modes51"] > 0
