"""GPU parity: the CUDA path against the reference's golden bytes and against the oracle, through the C ABI.

Bar: byte-identical output (BC1/BC3/BC4/BC5 and, on these inputs, BC7/BC6H/ASTC and the mips as well).
"""
import numpy as np
import pytest

import oracle_lib
from oracle_lib import BC1, BC3, BC4, BC5, BC7, chmask, psnr

pytestmark = pytest.mark.gpu


def _names(golden, prefix):
    return sorted(k[len(prefix):] for k in golden if k.startswith(prefix))


def test_golden_bcn_all_formats(cuda_lib, golden):
    for name in _names(golden, "img/"):
        img = golden["img/" + name]
        for fmt in range(5):
            got = cuda_lib.bc_encode(img, fmt)
            exp = golden[f"bc{fmt}/{name}"]
            assert np.array_equal(got, exp), (name, fmt, int(np.sum(got != exp)))


def test_golden_astc(cuda_lib, golden):
    for name in _names(golden, "img/"):
        got = cuda_lib.astc_encode(golden["img/" + name])
        assert np.array_equal(got, golden["astc/" + name]), name


def test_golden_bc6h(cuda_lib, golden):
    for name in _names(golden, "himg/"):
        got = cuda_lib.bc6h_encode(golden["himg/" + name])
        assert np.array_equal(got, golden["bc6h/" + name]), name


def test_golden_mips(cuda_lib, golden):
    for name in _names(golden, "img/"):
        img = golden["img/" + name]
        assert np.array_equal(cuda_lib.mip_next(img, 0), golden["mip0/" + name]), name
        assert np.array_equal(cuda_lib.mip_next(img, 1), golden["mip1/" + name]), name
    for name in _names(golden, "himg/"):
        got = cuda_lib.mip_next_f(golden["himg/" + name])
        assert np.array_equal(got.view(np.uint32), golden["mipf/" + name].view(np.uint32)), name


def _content(seed, w, h, alpha):
    import zap_b200.synth as S
    return S.colour_texture(w, h, seed=seed, alpha=alpha).numpy()


@pytest.mark.parametrize("w,h,alpha", [(256, 192, "opaque"), (256, 256, "noise"), (131, 77, "noise"), (67, 45, "opaque")])
def test_synthetic_vs_oracle(cuda_lib, w, h, alpha):
    ref = oracle_lib.best()
    img = _content(w * 7 + h, w, h, alpha)
    for fmt in (BC1, BC3, BC4, BC5, BC7):
        got, exp = cuda_lib.bc_encode(img, fmt), ref.bc_encode(img, fmt)
        assert np.array_equal(got, exp), (fmt, w, h, alpha, int(np.sum(got != exp)))
    got, exp = cuda_lib.astc_encode(img), ref.astc_encode(img)
    assert np.array_equal(got, exp), ("astc", w, h, alpha, int(np.sum(got != exp)))
    for srgb in (0, 1):
        assert np.array_equal(cuda_lib.mip_next(img, srgb), ref.mip_next(img, srgb))


def test_noise_images_vs_oracle(cuda_lib):
    """Uniform noise: every block is 'hard' (BC7 modes 5 and 1, ASTC two-partition search, long BC1 climbs)."""
    ref = oracle_lib.best()
    rng = np.random.default_rng(77)
    for alpha in (False, True):
        img = rng.integers(0, 256, (96, 80, 4), dtype=np.uint8)
        if not alpha:
            img[..., 3] = 255
        for fmt in (BC1, BC3, BC4, BC5, BC7):
            assert np.array_equal(cuda_lib.bc_encode(img, fmt), ref.bc_encode(img, fmt)), (fmt, alpha)
        assert np.array_equal(cuda_lib.astc_encode(img), ref.astc_encode(img)), alpha


def test_hdr_vs_oracle(cuda_lib):
    import zap_b200.synth as S
    ref = oracle_lib.best()
    half = S.hdr_texture(132, 68, seed=3).numpy()
    rgba = np.ones(half.shape[:2] + (4,), np.float32)
    rgba[..., :3] = half.astype(np.float32)
    assert np.array_equal(cuda_lib.bc6h_encode(rgba), ref.bc6h_encode(rgba))
    rng = np.random.default_rng(4)
    wild = (2.0 ** rng.uniform(-30, 20, (37, 29, 4))).astype(np.float32)
    wild[::3, ::2, 1] *= -1
    wild[5, 5, 0] = np.inf
    wild[6, 6, 2] = np.nan
    assert np.array_equal(cuda_lib.bc6h_encode(wild), ref.bc6h_encode(wild))


def test_device_api_narrow_inputs(cuda_lib):
    """R8 -> BC4, RG8 -> BC5, RGB16F -> BC6H equal the reference on the same texels widened to its input types."""
    import torch
    import zap_b200.synth as S
    ref = oracle_lib.best()
    col = S.colour_texture(200, 120, seed=9)
    nm = S.normal_map(200, 120, seed=9)
    dev = torch.device("cuda")
    r8 = col[..., :1].contiguous()
    got = cuda_lib.bc_encode_dev(r8.to(dev), BC4).cpu().numpy()
    wide = np.zeros((120, 200, 4), np.uint8)
    wide[..., 0] = r8[..., 0].numpy()
    wide[..., 3] = 255
    assert np.array_equal(got, ref.bc_encode(wide, BC4))
    got = cuda_lib.bc_encode_dev(nm.to(dev), BC5).cpu().numpy()
    wide = np.zeros((120, 200, 4), np.uint8)
    wide[..., :2] = nm.numpy()
    wide[..., 3] = 255
    assert np.array_equal(got, ref.bc_encode(wide, BC5))
    half = S.hdr_texture(64, 36, seed=1)
    got = cuda_lib.bc6h_encode_dev(half.to(dev)).cpu().numpy()
    rgba = np.ones((36, 64, 4), np.float32)
    rgba[..., :3] = half.numpy().astype(np.float32)
    assert np.array_equal(got, ref.bc6h_encode(rgba))
    t = torch.from_numpy(_content(5, 128, 64, "noise")).to(dev)
    for fmt in (BC1, BC7):
        assert np.array_equal(cuda_lib.bc_encode_dev(t, fmt).cpu().numpy(), ref.bc_encode(t.cpu().numpy(), fmt))


def test_unaligned_pitch_and_views(cuda_lib):
    """Row pitch not a multiple of 16 (scalar gather path) and a cropped view of a larger image."""
    ref = oracle_lib.best()
    big = _content(21, 103, 61, "noise")
    view = big[3:50, 5:90]  # non-contiguous rows, pitch 103*4
    for fmt in (BC1, BC3, BC7):
        assert np.array_equal(cuda_lib.bc_encode(view, fmt), ref.bc_encode(np.ascontiguousarray(view), fmt))
    assert np.array_equal(cuda_lib.mip_next(view, 1), ref.mip_next(np.ascontiguousarray(view), 1))


def test_large_image_band_pipeline(cuda_lib):
    """A host call large enough to be split into several bands over two streams."""
    ref = oracle_lib.best()
    img = _content(1, 1024, 1100, "opaque")
    got = cuda_lib.bc_encode(img, BC1)
    assert np.array_equal(got, ref.bc_encode(img, BC1, threads=8))


def test_mip_chain_matches_iterated_mips(cuda_lib):
    import torch
    ref = oracle_lib.best()
    img = _content(2, 100, 37, "noise")
    levels = cuda_lib.mip_chain_dev(torch.from_numpy(img).cuda(), srgb=1)
    cur = img
    assert len(levels) == ref.mip_levels(100, 37) - 1
    for lv in levels:
        cur = ref.mip_next(cur, 1)
        assert np.array_equal(lv.cpu().numpy(), cur)


def test_selftest_asserts_on_gpu_output(cuda_lib, golden):
    """tex_bench.c's quality asserts (rdo 0), applied to the GPU encoder's output."""
    ref = oracle_lib.best()
    img = golden["img/selftest67x45"]
    q = {}
    for fmt in range(5):
        dec = ref.bc_decode(cuda_lib.bc_encode(img, fmt), 67, 45, fmt)
        q[fmt] = psnr(img, dec, chmask(fmt))
        assert q[fmt] > 32
    assert q[BC7] > q[BC3]
    m5 = cuda_lib.bc_encode(golden["img/mode5_64x64"], BC7)
    assert np.sum((m5[0::16] & 0x3F) == 0x20) > 0
    one = np.array([[[10, 200, 30, 255]]], np.uint8)
    for fmt in range(5):
        dec = ref.bc_decode(cuda_lib.bc_encode(one, fmt), 1, 1, fmt)
        assert all(abs(int(dec[0, 0, c]) - int(one[0, 0, c])) <= 4 for c in range(4) if (chmask(fmt) >> c) & 1)


def test_errors_are_reported(cuda_lib):
    img = np.zeros((8, 8, 4), np.uint8)
    with pytest.raises(cuda_lib.ZapTexError) as e:
        cuda_lib.bc_encode(img, BC1, rdo=float("nan"))
    assert e.value.status == -1
    with pytest.raises(cuda_lib.ZapTexError) as e:
        cuda_lib.bc_encode(img, 9)
    assert e.value.status == -2
    lib = cuda_lib.load()
    out = np.zeros(64, np.uint8)
    assert lib.zap_tex_cuda_bc_encode(None, img.ctypes.data, 0, 8, 32, BC1, 0.0, out.ctypes.data) == -1
    assert lib.zap_tex_cuda_bc_encode(None, img.ctypes.data, 8, 8, 16, BC1, 0.0, out.ctypes.data) == -1
    assert lib.zap_tex_cuda_bc_encode(None, None, 8, 8, 32, BC1, 0.0, out.ctypes.data) == -1
    # the library still works after rejected calls
    assert np.array_equal(cuda_lib.bc_encode(img, BC1), oracle_lib.best().bc_encode(img, BC1))


def test_trace_counts_launches(cuda_lib):
    img = _content(3, 64, 64, "opaque")
    cuda_lib.trace(True)
    cuda_lib.bc_encode(img, BC7)
    rep = cuda_lib.trace_report()
    cuda_lib.trace(False)
    assert rep["bc7_mode6"][0] == 1 and rep["bc7_modes51"][0] == 1
    assert rep["bc7_mode6"][2] == 256 and 0 <= rep["bc7_modes51"][2] <= 256
