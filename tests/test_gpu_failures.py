"""Failure paths on the device, made on the host: allocation failures and the bounds-check build.

- zap_tex_cuda_debug_fail_allocations makes chosen device / pinned allocations of the library fail. Every entry point
  that allocates must then return ZTC_ERR_NO_MEMORY (and write nothing it should not), and the next call, with the
  hook cleared, must succeed with the reference's bytes. The batch planner is failed at each of its allocations in
  turn and must release what it had taken each time.
- The bounds-check build (libzap_tex_cuda_checks.so, -DZTC_CHECKS) runs small odd-size cases of every encoder in a
  child process, and every device entry point on a texture past that build's 4096 blocks per launch (so the encode
  runs as several launches); its output must equal the oracle's and its device check word must stay 0.
No kernel faults, traps or waits in any of these: the failures are made by the host.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle_lib

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NO_MEMORY = -4


def _expect_no_memory(cuda_lib, call, skip=0):
    lib = cuda_lib.load()
    assert lib.zap_tex_cuda_debug_fail_allocations(skip, 1) == 0
    try:
        with pytest.raises(cuda_lib.ZapTexError) as e:
            call()
        assert e.value.status == NO_MEMORY, str(e.value)
    finally:
        lib.zap_tex_cuda_debug_fail_allocations(0, 0)


def test_entry_points_report_no_memory_and_recover(cuda_lib):
    import torch

    import zap_b200.synth as S
    ref = oracle_lib.best()
    lib = cuda_lib.load()
    img = S.colour_texture(72, 52, seed=31, alpha="noise").numpy()
    dev = torch.from_numpy(img).cuda()
    ctx = C.c_void_p()
    assert lib.zap_tex_cuda_create(0, C.byref(ctx)) == 0  # a fresh context: its first call grows its staging buffers
    try:
        cases = [
            ("host BC7 encode", lambda: cuda_lib.bc_encode(img, cuda_lib.BC7, ctx=ctx), lambda o: np.array_equal(o, ref.bc_encode(img, 4))),
            ("device BC7 encode (work list)", lambda: cuda_lib.bc_encode_dev(dev, cuda_lib.BC7).cpu().numpy(),
             lambda o: np.array_equal(o, ref.bc_encode(img, 4))),
            ("device ASTC encode (work list)", lambda: cuda_lib.astc_encode_dev(dev).cpu().numpy(),
             lambda o: np.array_equal(o, ref.astc_encode(img))),
            ("device BC7 rate-distortion (decoded bases)", lambda: cuda_lib.bc_encode_rdo_dev(dev, cuda_lib.BC7, 30.0).cpu().numpy(),
             lambda o: np.array_equal(o, ref.bc_encode(img, 4, rdo=30.0))),
            ("host decode", lambda: cuda_lib.bc_decode(ref.bc_encode(img, 0), 72, 52, cuda_lib.BC1),
             lambda o: np.array_equal(o, ref.bc_decode(ref.bc_encode(img, 0), 72, 52, 0))),
            ("CLI file", lambda: cuda_lib.tex_file(img, cuda_lib.BC1, mips=True, srgb=True),
             lambda o: np.array_equal(o, oracle_lib.port().tex_file(img, 0, 0.0, 1, 1))),
        ]
        for name, call, ok in cases:
            _expect_no_memory(cuda_lib, call)
            torch.cuda.synchronize()
            assert ok(call()), name  # the library works again once allocations succeed
        big = S.colour_texture(300, 200, seed=32).numpy()  # a larger image grows the context's buffers again
        _expect_no_memory(cuda_lib, lambda: cuda_lib.bc_encode(big, cuda_lib.BC1, ctx=ctx))
        _expect_no_memory(cuda_lib, lambda: cuda_lib.bc_encode(big, cuda_lib.BC1, ctx=ctx), skip=1)
        assert np.array_equal(cuda_lib.bc_encode(big, cuda_lib.BC1, ctx=ctx), ref.bc_encode(big, 0))
    finally:
        lib.zap_tex_cuda_destroy(ctx)


def test_batch_planner_fails_cleanly_at_every_allocation(cuda_lib):
    import torch

    import zap_b200.synth as S
    texs = [S.colour_texture(w, h, seed=40 + k, device="cuda") for k, (w, h) in enumerate([(64, 32), (17, 9), (128, 128)])]
    fmts = [4, 0, 1]
    free0 = torch.cuda.mem_get_info()[0]
    failures = 0
    for skip in range(64):
        lib = cuda_lib.load()
        lib.zap_tex_cuda_debug_fail_allocations(skip, 1)
        try:
            b = cuda_lib.Batch(texs, fmts, autotune=skip % 2 == 1)
        except cuda_lib.ZapTexError as e:
            assert e.status == NO_MEMORY, str(e)
            failures += 1
            continue
        finally:
            lib.zap_tex_cuda_debug_fail_allocations(0, 0)
        b.run()
        b.run_plain()
        torch.cuda.synchronize()
        b.close()
        break
    assert failures >= 8  # the planner's allocations each failed once, then one batch was built and ran
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] >= free0 - (64 << 20)  # failed plans released what they had allocated


CHECKS_SCRIPT = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
import zap_b200, zap_b200.synth as S, oracle_lib, ctypes as C
ref = oracle_lib.best()
lib = zap_b200.load()
assert lib._name.endswith("libzap_tex_cuda_checks.so"), lib._name
rng = np.random.default_rng(9)
imgs = [S.colour_texture(53, 37, seed=1, alpha="noise").numpy(), rng.integers(0, 256, (21, 30, 4), dtype=np.uint8),
        S.colour_texture(1, 1, seed=2).numpy(), S.colour_texture(130, 66, seed=3).numpy()]
for img in imgs:
    for fmt in range(5):
        assert np.array_equal(zap_b200.bc_encode(img, fmt), ref.bc_encode(img, fmt)), fmt
    assert np.array_equal(zap_b200.astc_encode(img), ref.astc_encode(img))
hdr = np.ones((19, 27, 4), np.float32)
hdr[..., :3] = S.hdr_texture(27, 19, seed=4).numpy().astype(np.float32)
assert np.array_equal(zap_b200.bc6h_encode(hdr), ref.bc6h_encode(hdr))
# device entry points on 75 x 66 blocks: more than the build's 4096 blocks per launch, so each encode runs as two
# launches of whole block rows
big = S.colour_texture(300, 261, seed=5, alpha="noise")
bg = big.cuda()
for fmt in range(5):
    assert np.array_equal(zap_b200.bc_encode_dev(bg, fmt).cpu().numpy(), ref.bc_encode(big.numpy(), fmt)), ("dev", fmt)
assert np.array_equal(zap_b200.astc_encode_dev(bg).cpu().numpy(), ref.astc_encode(big.numpy()))
half = S.hdr_texture(300, 261, seed=6)
f32 = np.ones((261, 300, 4), np.float32)
f32[..., :3] = half.numpy().astype(np.float32)
assert np.array_equal(zap_b200.bc6h_encode_dev(half.cuda()).cpu().numpy(), ref.bc6h_encode(f32))
texs = [torch.from_numpy(i).cuda() for i in imgs]
b = zap_b200.Batch(texs, [4, 0, 1, 4], plan=("tiles_2d", "tile_x2"))
b.run(); torch.cuda.synchronize(); b.close()
word = C.c_uint(123)
assert lib.zap_tex_cuda_debug_checks(C.byref(word)) == 0, lib.zap_tex_cuda_last_error()
print("check word", hex(word.value))
assert word.value == 0
"""


def test_bounds_check_build_runs_clean():
    lib = os.path.join(ROOT, "zap_b200", "lib", "libzap_tex_cuda_checks.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "zap_b200", "csrc"), "-j", "8", "checks"], check=True)
    env = dict(os.environ, ZAP_TEX_CUDA_LIB=lib)
    r = subprocess.run([sys.executable, "-c", CHECKS_SCRIPT, ROOT], capture_output=True, text=True, env=env, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "check word 0x0" in r.stdout
