"""Device decoders against the reference's decoders, the palette-decode adjoint against FP64 gradients, and the
gradient refinement (never worse than the encoder, valid blocks)."""
import numpy as np
import pytest

import oracle_lib
from oracle_lib import BC1, BC7

pytestmark = pytest.mark.gpu


def _tex(seed, w, h, alpha="opaque"):
    import zap_b200.synth as S
    return S.colour_texture(w, h, seed=seed, alpha=alpha, device="cuda")


def test_device_decoders_match_reference(cuda_lib, golden):
    import torch
    ref = oracle_lib.best()
    rng = np.random.default_rng(8)
    noise = rng.integers(0, 256, (37, 53, 4), dtype=np.uint8)
    for name, img in [("noise", noise)] + [(k[4:], golden[k]) for k in golden if k.startswith("img/")][:8]:
        h, w = img.shape[:2]
        for fmt in range(5):
            bc = ref.bc_encode(img, fmt)
            got = cuda_lib.bc_decode_dev(torch.from_numpy(bc).cuda(), w, h, fmt).cpu().numpy()
            assert np.array_equal(got, ref.bc_decode(bc, w, h, fmt)), (name, fmt)
    for k in [k for k in golden if k.startswith("himg/")]:
        img = golden[k]
        h, w = img.shape[:2]
        bc = golden["bc6h/" + k[5:]]
        got = cuda_lib.bc6h_decode_dev(torch.from_numpy(bc).cuda(), w, h).cpu().numpy().view(np.uint16)
        assert np.array_equal(got, ref.bc6h_decode(bc, w, h)), k


def _weights_fp64(blocks, fmt):
    """Per-texel weight of endpoint 0 from the stored indices, in float64 (numpy restatement of the layouts)."""
    b = blocks.reshape(-1, 8 if fmt == BC1 else 16).astype(np.uint64)
    n = b.shape[0]
    a = np.zeros((n, 16))
    if fmt == BC1:
        c0 = b[:, 0] | (b[:, 1] << 8)
        c1 = b[:, 2] | (b[:, 3] << 8)
        idx = b[:, 4] | (b[:, 5] << 8) | (b[:, 6] << 16) | (b[:, 7] << 24)
        table = np.array([1.0, 0.0, 2.0 / 3.0, 1.0 / 3.0])
        for i in range(16):
            k = ((idx >> np.uint64(2 * i)) & np.uint64(3)).astype(int)
            k = np.where(c0 <= c1, np.where(k == 1, 1, 0), k)
            a[:, i] = table[k]
        return a, 3
    bits = np.unpackbits(blocks.reshape(-1, 16), axis=1, bitorder="little").astype(int)
    w4 = np.array([(64 * j + 7) // 15 for j in range(16)])
    for i in range(16):
        pos, nb = (65, 3) if i == 0 else (68 + 4 * (i - 1), 4)
        idx = sum(bits[:, pos + k] << k for k in range(nb))
        a[:, i] = 1.0 - w4[idx] / 64.0
    return a, 4


def test_palette_adjoint_against_fp64_and_finite_differences(cuda_lib):
    import torch

    class PaletteDecode(torch.autograd.Function):  # test harness only: forward / backward through the C ABI
        @staticmethod
        def forward(ctx, endpoints, blocks, fmt):
            ctx.blocks, ctx.fmt = blocks, fmt
            return cuda_lib.palette_decode_dev(blocks, fmt, endpoints)

        @staticmethod
        def backward(ctx, g):
            return cuda_lib.palette_adjoint_dev(ctx.blocks, ctx.fmt, g), None, None

    for fmt in (BC1, BC7):
        tex = _tex(3, 64, 48, "opaque")
        blocks = cuda_lib.bc_encode_dev(tex, fmt)
        x = tex.view(12, 4, 16, 4, 4).permute(0, 2, 1, 3, 4).reshape(-1, 16, 4).double()  # block-major texels
        e0 = cuda_lib.block_endpoints_dev(blocks, fmt) + torch.randn(x.shape[0], 2, 4, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
        e = e0.clone().requires_grad_(True)
        dec = PaletteDecode.apply(e, blocks, fmt)
        a, nc = _weights_fp64(blocks.cpu().numpy(), fmt)
        if fmt == BC7:
            mode6 = (blocks.view(-1, 16)[:, 0] & 0x7F).cpu().numpy() == 0x40
            assert mode6.mean() > 0.5
        else:
            mode6 = np.ones(a.shape[0], bool)
        cmask = torch.zeros(4, dtype=torch.float64, device="cuda")
        cmask[:nc] = 1
        loss = (((dec.double() - x) * cmask) ** 2).sum()
        loss.backward()
        g_cuda = e.grad.double().cpu().numpy()
        # FP64 analytic gradient of the same loss
        e64 = e0.double().cpu().numpy()
        A = a[:, :, None]
        d64 = A * e64[:, None, 0, :] + (1 - A) * e64[:, None, 1, :]
        r = (d64 - x.cpu().numpy()) * cmask.cpu().numpy()
        g64 = np.stack([(2 * r * A).sum(1), (2 * r * (1 - A)).sum(1)], 1)
        g64[~mode6] = 0
        scale = np.abs(g64).max()
        assert np.max(np.abs(g_cuda - g64)) / scale <= 1e-4, fmt
        # central finite differences (h = 1e-3) of the FP64 loss, on a sample of endpoint components
        rng = np.random.default_rng(2)
        for _ in range(24):
            blk = int(rng.integers(0, a.shape[0]))
            if not mode6[blk]:
                continue
            k, c = int(rng.integers(0, 2)), int(rng.integers(0, nc))

            def loss64(ev):
                dd = A[blk] * ev[0] + (1 - A[blk]) * ev[1]
                return float((((dd - x[blk].cpu().numpy()) * cmask.cpu().numpy()) ** 2).sum())
            ep, em = e64[blk].copy(), e64[blk].copy()
            ep[k, c] += 1e-3
            em[k, c] -= 1e-3
            fd = (loss64(ep) - loss64(em)) / 2e-3
            assert abs(g_cuda[blk, k, c] - fd) <= 1e-4 * max(1.0, abs(fd), scale * 1e-2), (fmt, blk, k, c, g_cuda[blk, k, c], fd)


@pytest.mark.parametrize("fmt", [BC1, BC7])
def test_refinement_never_worse_and_valid(cuda_lib, fmt):
    import torch
    ref = oracle_lib.best()
    tex = _tex(11, 256, 128, "opaque")
    blocks = cuda_lib.bc_encode_dev(tex, fmt)
    original = blocks.clone()
    s0, s1 = cuda_lib.refine_dev(tex, fmt, blocks, steps=8, lr=1.0)
    torch.cuda.synchronize()
    s0, s1 = s0.cpu().numpy().astype(np.int64), s1.cpu().numpy().astype(np.int64)
    assert np.all(s1 <= s0)
    img = tex.cpu().numpy()
    bs = 8 if fmt == BC1 else 16

    def block_sse(bc):
        dec = ref.bc_decode(bc, 256, 128, fmt).astype(np.int64)
        chans = 3 if fmt == BC1 else 4
        d = ((dec - img.astype(np.int64))[..., :chans] ** 2).sum(-1)
        return d.reshape(32, 4, 64, 4).sum((1, 3)).reshape(-1)
    before, after = block_sse(original.cpu().numpy()), block_sse(blocks.cpu().numpy())
    assert np.array_equal(before, s0) and np.array_equal(after, s1)  # the kernel's numbers are the decoder's
    changed = np.any(blocks.cpu().numpy().reshape(-1, bs) != original.cpu().numpy().reshape(-1, bs), axis=1)
    assert np.all(after[changed] < before[changed]) and np.array_equal(after[~changed], before[~changed])
    assert after.sum() <= before.sum()
