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


def _mixed_bc7_texture():
    """128x128 atlas of 32x32 textures, opaque and noise alpha alternating: its BC7 blocks are about 39 % mode 1,
    46 % mode 5 (every rotation) and 15 % mode 6."""
    import torch

    import zap_b200.synth as S
    tiles = [S.colour_texture(32, 32, seed=k, alpha="noise" if k % 2 else "opaque") for k in range(16)]
    return torch.cat([torch.cat(tiles[r * 4:(r + 1) * 4], 1) for r in range(4)], 0).contiguous().cuda()


def _linear_model_fp64(blocks, fmt, oracle):
    """The linear decode of every block in float64, from the oracle's own parse of the stored bits: per block and
    texel, the endpoint-0 weight in decoded channel order, the rows of the two endpoints it mixes, the stored channel,
    and where the value is a constant instead (BC7 alpha without bits: 255; BC1 alpha: not decoded, 0)."""
    b = blocks.reshape(-1, 8 if fmt == BC1 else 16)
    n = b.shape[0]
    A = np.zeros((n, 16, 4))
    R0 = np.zeros((n, 16, 4), int)
    SC = np.tile(np.arange(4), (n, 16, 1))
    fixed = np.full((n, 16, 4), np.nan)
    if fmt == BC1:
        bb = b.astype(np.uint64)
        c0 = bb[:, 0] | (bb[:, 1] << 8)
        c1 = bb[:, 2] | (bb[:, 3] << 8)
        idx = bb[:, 4] | (bb[:, 5] << 8) | (bb[:, 6] << 16) | (bb[:, 7] << 24)
        four, three = np.array([1.0, 0.0, 2.0 / 3.0, 1.0 / 3.0]), np.array([1.0, 0.0, 0.5, 0.0])
        for i in range(16):  # the decoder's rule (zap_tex.h:1508-1517): 3 colours and black when c0 <= c1
            k = ((idx >> np.uint64(2 * i)) & np.uint64(3)).astype(int)
            A[:, i, :] = np.where(c0 > c1, four[k], three[k])[:, None]
            fixed[(c0 <= c1) & (k == 3), i, :3] = 0.0
        fixed[:, :, 3] = 0.0
        return A, R0, SC, fixed
    for k in range(n):
        f = oracle.bc7_fields(b[k])
        if f["mode"] == 8:
            fixed[k] = 0.0
            continue
        rot = f["rot"]
        for c in range(4):
            sc = c if rot == 0 else (rot - 1 if c == 3 else 3 if c == rot - 1 else c)
            SC[k, :, c] = sc
            wts = np.array(f["aw"] if sc == 3 else f["cw"], float)
            A[k, :, c] = 1.0 - wts / 64.0
            R0[k, :, c] = 2 * np.array(f["subset"])
            if sc == 3 and not f["ab"]:
                fixed[k, :, c] = 255.0
    return A, R0, SC, fixed


def _decode_fp64(E, A, R0, SC, fixed):
    n = E.shape[0]
    bi = np.arange(n)[:, None, None]
    d = A * E[bi, R0, SC] + (1 - A) * E[bi, R0 + 1, SC]
    return np.where(np.isnan(fixed), d, fixed)


def _grad_fp64(E, A, R0, SC, fixed, r):
    """d(sum r . decoded)/dE in float64 (r: upstream gradient on the decoded texels)."""
    G = np.zeros_like(E)
    live = np.isnan(fixed)
    n = E.shape[0]
    bi = np.broadcast_to(np.arange(n)[:, None, None], A.shape)
    np.add.at(G, (bi[live], R0[live], SC[live]), (A * r)[live])
    np.add.at(G, (bi[live], R0[live] + 1, SC[live]), ((1 - A) * r)[live])
    return G


def test_palette_adjoint_against_fp64_and_finite_differences(cuda_lib, oracle):
    import torch

    class PaletteDecode(torch.autograd.Function):  # test harness only: forward / backward through the C ABI
        @staticmethod
        def forward(ctx, endpoints, blocks, fmt):
            ctx.blocks, ctx.fmt = blocks, fmt
            return cuda_lib.palette_decode_dev(blocks, fmt, endpoints)

        @staticmethod
        def backward(ctx, g):
            return cuda_lib.palette_adjoint_dev(ctx.blocks, ctx.fmt, g), None, None

    for fmt, tex in ((BC1, _tex(3, 64, 48, "opaque")), (BC7, _tex(3, 64, 48, "noise")), (BC7, _mixed_bc7_texture())):
        h, w = tex.shape[:2]
        blocks = cuda_lib.bc_encode_dev(tex, fmt)
        x = tex.view(h // 4, 4, w // 4, 4, 4).permute(0, 2, 1, 3, 4).reshape(-1, 16, 4).double()  # block-major texels
        rows = cuda_lib.endpoint_rows(fmt)
        noise = torch.randn(x.shape[0], rows, 4, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
        e0 = cuda_lib.block_endpoints_dev(blocks, fmt) + noise
        e = e0.clone().requires_grad_(True)
        dec = PaletteDecode.apply(e, blocks, fmt)
        model = _linear_model_fp64(blocks.cpu().numpy(), fmt, oracle)
        if fmt == BC7:
            modes = np.array([oracle.bc7_fields(b)["mode"] for b in blocks.cpu().numpy().reshape(-1, 16)])
            if h == 128:  # the mixed texture: every mode the encoder writes, each a large share
                for m, share in ((1, 0.2), (5, 0.2), (6, 0.1)):
                    assert np.mean(modes == m) >= share, (m, np.mean(modes == m))
        nc = 3 if fmt == BC1 else 4
        cmask = torch.zeros(4, dtype=torch.float64, device="cuda")
        cmask[:nc] = 1
        loss = (((dec.double() - x) * cmask) ** 2).sum()
        loss.backward()
        g_cuda = e.grad.double().cpu().numpy()
        # FP64 decode and analytic gradient of the same loss
        e64 = e0.double().cpu().numpy()
        d64 = _decode_fp64(e64, *model)
        assert np.max(np.abs(dec.detach().double().cpu().numpy() - d64)) <= 1e-3, fmt
        r = 2 * (d64 - x.cpu().numpy()) * cmask.cpu().numpy()
        g64 = _grad_fp64(e64, *model, r)
        scale = np.abs(g64).max()
        assert np.max(np.abs(g_cuda - g64)) / scale <= 1e-4, fmt
        # central finite differences (h = 1e-3) of the FP64 loss, on a sample of endpoint components
        rng = np.random.default_rng(2)
        xs = x.cpu().numpy()
        cm = cmask.cpu().numpy()
        live = [(b, k, c) for b in range(e64.shape[0]) for k in range(rows) for c in range(nc) if g64[b, k, c] != 0]
        for j in rng.choice(len(live), 48, replace=False):
            blk, k, c = live[j]
            one = tuple(m[blk:blk + 1] for m in model)

            def loss64(ev):
                return float((((_decode_fp64(ev[None], *one)[0] - xs[blk]) * cm) ** 2).sum())
            ep, em = e64[blk].copy(), e64[blk].copy()
            ep[k, c] += 1e-3
            em[k, c] -= 1e-3
            fd = (loss64(ep) - loss64(em)) / 2e-3
            assert abs(g_cuda[blk, k, c] - fd) <= 1e-4 * max(1.0, abs(fd), scale * 1e-2), (fmt, blk, k, c, g_cuda[blk, k, c], fd)


def test_palette_decode_at_stored_endpoints_rounds_to_the_decoder(cuda_lib):
    """Every BC7 mode (arbitrary blocks, the reserved mode too) and BC1 (4-colour, 3-colour and black texels): the
    linear decode at the blocks' own endpoints is the integer decoder's output before its rounding, so within 0.5
    of it (and 0 on BC1's black texels)."""
    import torch
    rng = np.random.default_rng(17)
    bc = rng.integers(0, 256, (9 * 256, 16), dtype=np.uint8)
    for m in range(9):
        rows = bc[m::9]
        rows[:, 0] = 0 if m == 8 else ((rows[:, 0] >> (m + 1)) << (m + 1)) | (1 << m)
    for fmt, blocks, w, h in ((BC7, bc.reshape(-1), 4 * 64, 4 * 36), (BC1, bc.reshape(-1)[:8 * 64 * 36], 4 * 64, 4 * 36)):
        blk = torch.from_numpy(np.ascontiguousarray(blocks)).cuda()
        lin = cuda_lib.palette_decode_dev(blk, fmt, cuda_lib.block_endpoints_dev(blk, fmt)).cpu().numpy()
        img = cuda_lib.bc_decode_dev(blk, w, h, fmt).cpu().numpy().astype(np.float64)
        img = img.reshape(h // 4, 4, w // 4, 4, 4).transpose(0, 2, 1, 3, 4).reshape(-1, 16, 4)
        nc = 3 if fmt == BC1 else 4
        assert np.max(np.abs(lin[..., :nc] - img[..., :nc])) <= 0.5 + 1e-3, fmt


@pytest.mark.parametrize("fmt,content", [(BC1, "opaque"), (BC7, "opaque"), (BC7, "mixed")])
def test_refinement_never_worse_and_valid(cuda_lib, oracle, fmt, content):
    import torch
    ref = oracle_lib.best()
    tex = _tex(11, 256, 128, "opaque") if content == "opaque" else _mixed_bc7_texture().repeat(1, 2, 1).contiguous()
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
    if content == "mixed":  # refinement reaches every mode the encoder writes, and keeps each block's mode
        old_modes = np.array([oracle.bc7_fields(b)["mode"] for b in original.cpu().numpy().reshape(-1, 16)])
        new_modes = np.array([oracle.bc7_fields(b)["mode"] for b in blocks.cpu().numpy().reshape(-1, 16)])
        assert np.array_equal(old_modes, new_modes)
        for m in (1, 5, 6):
            assert changed[old_modes == m].any(), m
