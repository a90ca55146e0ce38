"""Full-size and very large inputs on the device, byte for byte.

- The benchmark configurations at their full sizes (2048x2048): BC7 RGBA8, BC4 from R8, BC5 from RG8, BC6H from
  RGB16F, ASTC 4x4, BC1, against the reference encoder (all host threads when the reference library is built).
- The exact textures the benchmark times, generated the way it generates them: BC1 of the 512x512 seed-0 texture
  (the reference's plain BC1 case, which must be byte-identical), the headline BC7 texture, and the first texture
  of every secondary figure's ring.
- A 32768x16400 RGBA8 image (2.1 GB, past 32-bit byte offsets; odd last block row) encoded to BC1 and BC7 through
  the device API. At rdo 0 each block depends only on its own 16 texels (edge texels replicated), so the texels of
  any block, cut out as a 4x4 image (smaller at the right and bottom edges), encode to that block's bytes: sampled
  blocks, every corner and edge block included, are checked against the oracle that way.
"""
import os

import numpy as np
import pytest

import oracle_lib
from oracle_lib import BC1, BC4, BC5, BC7

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 1


def test_full_size_configs_match_reference(cuda_lib):
    import torch

    import zap_b200.synth as S
    ref = oracle_lib.best()
    dev = torch.device("cuda", 0)
    rgba = S.colour_texture(2048, 2048, seed=301, alpha="noise", device=dev)
    host = rgba.cpu().numpy()
    for fmt in (BC7, BC1):
        got = cuda_lib.bc_encode_dev(rgba, fmt).cpu().numpy()
        assert np.array_equal(got, ref.bc_encode(host, fmt, threads=THREADS)), fmt
    got = cuda_lib.astc_encode_dev(rgba).cpu().numpy()
    assert np.array_equal(got, ref.astc_encode(host, threads=THREADS))
    # narrow inputs: the reference reads them widened to RGBA8 (missing channels 0, alpha 255)
    r8 = rgba[..., :1].contiguous()
    wide = np.zeros((2048, 2048, 4), np.uint8)
    wide[..., 0] = host[..., 0]
    wide[..., 3] = 255
    assert np.array_equal(cuda_lib.bc_encode_dev(r8, BC4).cpu().numpy(), ref.bc_encode(wide, BC4, threads=THREADS))
    rg8 = S.normal_map(2048, 2048, seed=302, device=dev)
    wide[..., :2] = rg8.cpu().numpy()
    assert np.array_equal(cuda_lib.bc_encode_dev(rg8, BC5).cpu().numpy(), ref.bc_encode(wide, BC5, threads=THREADS))
    half = S.hdr_texture(2048, 2048, seed=303, device=dev)
    f32 = np.ones((2048, 2048, 4), np.float32)
    f32[..., :3] = half.cpu().numpy().astype(np.float32)
    assert np.array_equal(cuda_lib.bc6h_encode_dev(half).cpu().numpy(), ref.bc6h_encode(f32, threads=THREADS))


def test_benchmark_textures_match_reference(cuda_lib):
    import torch

    import zap_b200.synth as S
    ref = oracle_lib.best()
    dev = torch.device("cuda", 0)
    # plain BC1 (default quality, rdo 0) of one 512x512 RGBA8 texture from seed 0, alpha 255: byte-identical
    c0 = S.colour_texture(512, 512, seed=0, device=dev)
    assert bool((c0[..., 3] == 255).all())
    got = cuda_lib.bc_encode_dev(c0, BC1).cpu().numpy()
    assert np.array_equal(got, ref.bc_encode(c0.cpu().numpy(), BC1))
    # the headline texture (BC7, noise alpha, seed 100) and each secondary figure's first ring texture (seed 0)
    c1 = S.colour_texture(2048, 2048, seed=100, alpha="noise", device=dev)
    assert np.array_equal(cuda_lib.bc_encode_dev(c1, BC7).cpu().numpy(), ref.bc_encode(c1.cpu().numpy(), BC7, threads=THREADS))
    opaque = S.colour_texture(2048, 2048, seed=0, device=dev)
    host = opaque.cpu().numpy()
    assert np.array_equal(cuda_lib.bc_encode_dev(opaque, BC1).cpu().numpy(), ref.bc_encode(host, BC1, threads=THREADS))
    wide = np.zeros_like(host)
    wide[..., 0], wide[..., 3] = host[..., 0], 255
    assert np.array_equal(cuda_lib.bc_encode_dev(opaque[..., :1].contiguous(), BC4).cpu().numpy(),
                          ref.bc_encode(wide, BC4, threads=THREADS))
    # BC7 on the opaque texture: few blocks leave mode 6 (at most one per CTA of the modes-5/1 launch)
    assert np.array_equal(cuda_lib.bc_encode_dev(opaque, BC7).cpu().numpy(), ref.bc_encode(host, BC7, threads=THREADS))
    # BC7 on an atlas of 1024 textures of 64x64 in a seeded order: a quarter of the blocks leave mode 6, several
    # rounds per CTA of the modes-5/1 launch
    tiles = torch.stack([S.colour_texture(64, 64, seed=30000 + k, device=dev) for k in range(1024)])
    perm = torch.randperm(1024, generator=torch.Generator().manual_seed(0)).to(dev)
    atlas = tiles[perm].view(32, 32, 64, 64, 4).permute(0, 2, 1, 3, 4).reshape(2048, 2048, 4).contiguous()
    assert np.array_equal(cuda_lib.bc_encode_dev(atlas, BC7).cpu().numpy(), ref.bc_encode(atlas.cpu().numpy(), BC7, threads=THREADS))


def _huge_image(w, h, device):
    """A w x h RGBA8 image tiled from one 2048x2048 texture, every tile shifted by its own offset."""
    import torch

    import zap_b200.synth as S
    tile = S.colour_texture(2048, 2048, seed=304, alpha="noise", device=device)
    img = torch.empty((h, w, 4), dtype=torch.uint8, device=device)
    for ty in range(0, h, 2048):
        for tx in range(0, w, 2048):
            hh, ww = min(2048, h - ty), min(2048, w - tx)
            k = (ty // 2048) * 31 + (tx // 2048) * 7
            img[ty:ty + hh, tx:tx + ww] = tile[:hh, :ww] + torch.tensor([k & 255, (3 * k) & 255, 0, 0], dtype=torch.uint8, device=device)
    return img


def test_huge_image_sampled_blocks(cuda_lib):
    import torch
    ref = oracle_lib.port()
    dev = torch.device("cuda", 0)
    w, h = 32768, 16400 + 3  # 2.15 GB of texels; the last block row holds 3 texel rows
    img = _huge_image(w, h, dev)
    bw, bh = (w + 3) // 4, (h + 3) // 4
    rng = np.random.default_rng(305)
    picks = {(0, 0), (bw - 1, 0), (0, bh - 1), (bw - 1, bh - 1)}
    picks |= {(int(x), bh - 1) for x in rng.integers(0, bw, 64)} | {(bw - 1, int(y)) for y in rng.integers(0, bh, 64)}
    picks |= {(int(x), int(y)) for x, y in zip(rng.integers(0, bw, 600), rng.integers(0, bh, 600))}
    picks = sorted(picks)
    crops = {(x, y): img[4 * y:min(h, 4 * y + 4), 4 * x:min(w, 4 * x + 4)].cpu().numpy() for x, y in picks}
    for fmt in (BC1, BC7):
        bs = 8 if fmt == BC1 else 16
        out = cuda_lib.bc_encode_dev(img, fmt)
        torch.cuda.synchronize()
        assert out.numel() == bw * bh * bs
        idx = torch.tensor([y * bw + x for x, y in picks], dtype=torch.int64, device=dev)
        got = out.view(-1, bs)[idx].cpu().numpy()
        for k, (x, y) in enumerate(picks):
            want = ref.bc_encode(crops[(x, y)], fmt)
            assert np.array_equal(got[k], want), (fmt, x, y)
        del out
    del img
    torch.cuda.empty_cache()
