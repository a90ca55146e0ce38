"""The allocation-free BC7 entry point (zap_tex_cuda_bc7_encode_noalloc_dev), through the C ABI.

Some callers cannot allocate device memory while they encode - real-time frame loops where an allocation would
stall, engines with a fixed up-front GPU budget, plug-in hosts that only hand over their own buffers. This entry
point keeps its BC7 work list in a static device array instead of allocating one. Its output must be byte-for-byte
the output of the allocating entry point, also on consecutive calls that share that array (the list must start
empty every time), and oversize textures must be refused before anything runs. At exactly its limit (4096 x 4096
texels, 1048576 blocks) of uniform noise, where every block goes on the list, its bytes must be the reference
encoder's.

The file name sorts last so that a run stopping at the first failure has run every other test already.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle_lib

pytestmark = pytest.mark.gpu


def _call(lib, tex, out, stream):
    h, w = tex.shape[0], tex.shape[1]
    return lib.zap_tex_cuda_bc7_encode_noalloc_dev(C.c_void_p(tex.data_ptr()), w, h, tex.stride(0), C.c_void_p(out.data_ptr()),
                                                   C.c_void_p(stream.cuda_stream))


def test_noalloc_bc7_matches_allocating_entry_point(cuda_lib):
    import torch

    import zap_b200.synth as S
    lib = cuda_lib.load()
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(3)
    noise = torch.from_numpy(rng.integers(0, 256, (360, 200, 4), dtype=np.uint8)).cuda()
    inputs = [S.colour_texture(1024, 512, seed=1, alpha="noise", device="cuda"),  # mostly mode 6, some listed blocks
              noise,                                                              # every block on the work list
              S.colour_texture(301, 197, seed=2, alpha="opaque", device="cuda")]  # odd size, fewer blocks than before
    for tex in inputs:  # consecutive calls reuse the static work list
        expect = cuda_lib.bc_encode_dev(tex, cuda_lib.BC7)
        got = torch.full_like(expect, 0xAB)
        assert _call(lib, tex, got, stream) == 0, lib.zap_tex_cuda_last_error()
        torch.cuda.synchronize()
        assert torch.equal(got, expect)


def test_noalloc_bc7_at_its_block_limit(cuda_lib):
    import torch

    import zap_b200.synth as S
    lib = cuda_lib.load()
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(11)
    host = rng.integers(0, 256, (4096, 4096, 4), dtype=np.uint8)  # 1048576 blocks, every one past mode 6
    host[:2048, :, 3] = 255                                         # opaque top half: mode 1 runs there too
    noise = torch.from_numpy(host).cuda()
    got = torch.full((4096 * 4096,), 0xAB, dtype=torch.uint8, device="cuda")
    assert _call(lib, noise, got, stream) == 0, lib.zap_tex_cuda_last_error()
    torch.cuda.synchronize()
    want = oracle_lib.best().bc_encode(host, oracle_lib.BC7, threads=os.cpu_count() or 1)
    assert np.array_equal(got.cpu().numpy(), want)
    # the next call after a full list: smooth content at the same size, few listed blocks, same bytes as the
    # allocating entry point
    smooth = S.colour_texture(4096, 4096, seed=5, alpha="noise", device="cuda")
    got.fill_(0xAB)
    assert _call(lib, smooth, got, stream) == 0, lib.zap_tex_cuda_last_error()
    torch.cuda.synchronize()
    assert torch.equal(got, cuda_lib.bc_encode_dev(smooth, cuda_lib.BC7))


def test_noalloc_rejects_textures_beyond_its_limit(cuda_lib):
    import torch
    lib = cuda_lib.load()
    stream = torch.cuda.current_stream()
    tex = torch.zeros((4100, 4096, 4), dtype=torch.uint8, device="cuda")  # 1025 x 1024 blocks > 1048576
    out = torch.zeros(16, dtype=torch.uint8, device="cuda")
    assert _call(lib, tex, out, stream) == -1
    assert b"1048576" in lib.zap_tex_cuda_last_error()
    small = torch.zeros((8, 8, 4), dtype=torch.uint8, device="cuda")
    out = torch.zeros(64, dtype=torch.uint8, device="cuda")
    assert _call(lib, small, out, stream) == 0  # still usable after the refusal
    torch.cuda.synchronize()
