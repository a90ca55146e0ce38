"""Pin the oracle restatement (oracle/zt_oracle.c) before trusting it.

1. Byte-identical to the reference's own output on the committed golden fixtures (tests/golden, made by running
   the reference itself).
2. The known answers of the reference's self-test (tex_bench.c), re-run against the restatement.
3. Byte-identical to the live reference library on fresh seeded inputs, where that library is built.
"""
import numpy as np
import pytest

import oracle_lib
from oracle_lib import BC1, BC3, BC4, BC5, BC7, chmask, psnr


def _names(golden, prefix):
    return sorted(k[len(prefix):] for k in golden if k.startswith(prefix))


def test_golden_bcn(oracle, golden):
    for name in _names(golden, "img/"):
        img = golden["img/" + name]
        for fmt in range(5):
            got = oracle.bc_encode(img, fmt)
            assert np.array_equal(got, golden[f"bc{fmt}/{name}"]), (name, fmt)


def test_golden_astc(oracle, golden):
    for name in _names(golden, "img/"):
        assert np.array_equal(oracle.astc_encode(golden["img/" + name]), golden["astc/" + name]), name


def test_golden_bc6h_and_float_mips(oracle, golden):
    for name in _names(golden, "himg/"):
        img = golden["himg/" + name]
        assert np.array_equal(oracle.bc6h_encode(img), golden["bc6h/" + name]), name
        assert np.array_equal(oracle.mip_next_f(img).view(np.uint32), golden["mipf/" + name].view(np.uint32)), name


def test_golden_mips(oracle, golden):
    for name in _names(golden, "img/"):
        img = golden["img/" + name]
        assert np.array_equal(oracle.mip_next(img, 0), golden["mip0/" + name]), name
        assert np.array_equal(oracle.mip_next(img, 1), golden["mip1/" + name]), name


def test_srgb_tables_match_reference_constants(oracle, golden):
    lin, thr = oracle.srgb_tables()
    assert np.array_equal(lin.view(np.uint32), golden["srgb_lin"].view(np.uint32))
    assert np.array_equal(thr.view(np.uint32), golden["srgb_thr"].view(np.uint32))


# ---------------------------------------------------------------- tex_bench.c known answers
def test_half_float_known_answers(oracle):
    """tex_bench.c:47-48."""
    for h in range(0, 0x7BFF + 1, 7):
        assert oracle.f2h(oracle.h2f(h)) == h
    assert oracle.f2h(oracle.h2f(0x7BFF)) == 0x7BFF
    assert oracle.f2h(-1.0) == 0 and oracle.f2h(1e9) == 0x7BFF
    assert oracle.f2h(1.0) == 0x3C00 and oracle.f2h(1.0 + 1.0 / 4096) == 0x3C00


def test_mip_known_answers(oracle):
    """tex_bench.c:87-100."""
    assert oracle.mip_levels(1, 1) == 1 and oracle.mip_levels(256, 128) == 9 and oracle.mip_levels(5, 3) == 3
    bw = np.array([[[0, 0, 0, 255], [255, 255, 255, 255]], [[0, 0, 0, 255], [255, 255, 255, 255]]], np.uint8)
    m = oracle.mip_next(bw, 0)
    assert m[0, 0, 0] == 128 and m[0, 0, 3] == 255
    m = oracle.mip_next(bw, 1)
    assert m[0, 0, 0] == 188 and m[0, 0, 1] == 188 and m[0, 0, 3] == 255
    for v in range(256):
        assert oracle.mip_next(np.full((2, 2, 4), v, np.uint8), 1)[0, 0, 0] == v
    odd = np.full((3, 5, 4), 77, np.uint8)
    m2 = oracle.mip_next(odd, 1)
    assert m2.shape == (1, 2, 4) and m2[0, 0, 0] == 77 and m2[0, 1, 3] == 77
    fl = np.array([1, 2, 3, 4, 3, 2, 1, 0, 5, 5, 5, 5, 7, 7, 7, 7], np.float32).reshape(2, 2, 4)
    fo = oracle.mip_next_f(fl)
    assert fo[0, 0, 0] == 4 and fo[0, 0, 3] == 4


def test_astc_ise_roundtrip(oracle):
    """tex_bench.c:104-117: every range kind, n = 1..16."""
    import ctypes
    rng = np.random.default_rng(1)
    levels = [2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64, 80, 96, 128, 160, 192, 256]
    for ri, lv in enumerate(levels):
        for n in range(1, 17):
            v = rng.integers(0, lv, 16).astype(np.int32)
            got = np.zeros(16, np.int32)
            assert oracle._ise_roundtrip(ri, n, v.ctypes.data, got.ctypes.data) >= 0, (ri, n)
    del ctypes


def test_astc_partition_checksum(oracle):
    """tex_bench.c:118-121: FNV-1a over the 1024 two-partition patterns."""
    h = 2166136261
    for sd in range(1024):
        for i in range(16):
            h ^= oracle.astc_partition(sd, i & 3, i >> 2, 2)
            h = (h * 16777619) & 0xFFFFFFFF
    assert h == 0x5D5FC459


def test_astc_void_extent(oracle):
    """tex_bench.c:123-125."""
    ve = np.array([0xFC, 0xFD, 0xFF, 0xFF, 0xFF, 0xFF, 0xFF, 0xFF, 0x00, 0x40, 0x00, 0x80, 0x00, 0xC0, 0xFF, 0xFF], np.uint8)
    vo = oracle.astc_decode(ve, 4, 4)
    assert tuple(vo[0, 0]) == (0x40, 0x80, 0xC0, 0xFF)


def test_selftest_quality_floors(oracle, golden):
    """tex_bench.c:155-177 at rdo 0: PSNR floors, BC7 beats BC3, BC1 never transparent, 1x1 within 4."""
    img = golden["img/selftest67x45"]
    h, w = img.shape[:2]
    q = {}
    for fmt in range(5):
        dec = oracle.bc_decode(oracle.bc_encode(img, fmt), w, h, fmt)
        q[fmt] = psnr(img, dec, chmask(fmt))
        assert q[fmt] > 32, (fmt, q[fmt])
        if fmt == BC1:
            assert np.all(dec[..., 3] == 255)
    assert q[BC7] > q[BC3]
    one = np.array([[[10, 200, 30, 255]]], np.uint8)
    for fmt in range(5):
        dec = oracle.bc_decode(oracle.bc_encode(one, fmt), 1, 1, fmt)
        for c in range(4):
            if (chmask(fmt) >> c) & 1:
                assert abs(int(dec[0, 0, c]) - int(one[0, 0, c])) <= 4


def test_selftest_bc7_mode5_and_hdr(oracle, golden):
    """tex_bench.c:51-84: mode 5 chosen on independent alpha; BC6H mean relative error < 0.08."""
    img = golden["img/mode5_64x64"]
    bc = oracle.bc_encode(img, BC7)
    assert np.sum((bc[0::16] & 0x3F) == 0x20) > 0
    assert psnr(img, oracle.bc_decode(bc, 64, 64, BC7), 15) > 30
    hdr = golden["himg/hdr37x21"]
    dec = oracle.bc6h_decode(oracle.bc6h_encode(hdr), 37, 21)
    df = np.vectorize(oracle.h2f)(dec[..., :3]).astype(np.float64)
    a = hdr[..., :3].astype(np.float64)
    assert np.mean(np.abs(a - df) / (a + 0.01)) < 0.08 and dec[0, 0, 3] == 0x3C00


def test_selftest_astc_quality(oracle, golden):
    """tex_bench.c:127-141."""
    for k, floor in ((0, 41), (1, 26)):
        img = golden[f"img/astc64x48_k{k}"]
        assert psnr(img, oracle.astc_decode(oracle.astc_encode(img), 64, 48), 15) > floor


# ---------------------------------------------------------------- live reference
@pytest.mark.parametrize("seed", [11, 12])
def test_port_matches_reference_live(oracle, reference, seed):
    rng = np.random.default_rng(seed)
    for _ in range(4):
        w, h = int(rng.integers(1, 90)), int(rng.integers(1, 90))
        img = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
        img[: h // 2] = np.sort(img[: h // 2], axis=1)  # smooth half, noisy half
        if rng.random() < 0.5:
            img[..., 3] = 255
        for fmt in (BC1, BC3, BC4, BC5, BC7):
            assert np.array_equal(oracle.bc_encode(img, fmt), reference.bc_encode(img, fmt)), (fmt, w, h)
        assert np.array_equal(oracle.astc_encode(img), reference.astc_encode(img)), (w, h)
        hdr = (2.0 ** rng.uniform(-12, 14, (h, w, 4))).astype(np.float32)
        assert np.array_equal(oracle.bc6h_encode(hdr), reference.bc6h_encode(hdr)), (w, h)


def test_reference_band_parallel_matches_single_call(reference):
    """The all-cores CPU baseline (8-block-row bands, viewer.cpp:455-471) gives the single-call bytes at rdo 0."""
    rng = np.random.default_rng(5)
    img = rng.integers(0, 256, (75, 61, 4), dtype=np.uint8)
    for fmt in (BC1, BC7):
        assert np.array_equal(reference.bc_encode(img, fmt, threads=4), reference.bc_encode(img, fmt))
    assert np.array_equal(reference.astc_encode(img, threads=3), reference.astc_encode(img))
    assert oracle_lib.bc_size(61, 75, BC7) == reference.bc_encode(img, BC7).size


# ---------------------------------------------------------------- split / merge (zap_tex.h:1549-1571)
def test_split_merge_identity(oracle):
    """tex_bench.c:166-168: merge(split(x)) == x, for every format, whole blocks and stray tail bytes."""
    rng = np.random.default_rng(8)
    for fmt in (BC1, BC3, BC4, BC5, BC7):
        for n in (0, 5, 8, 16, 17, 8 * 37 + 3, 16 * 41, 16 * 41 + 9):
            x = rng.integers(0, 256, n, dtype=np.uint8)
            s = oracle.bc_split(x, fmt)
            assert np.array_equal(oracle.bc_merge(s, fmt), x), (fmt, n)
            bs = oracle_lib.block_bytes(fmt)
            if n >= 2 * bs:  # plane 0 starts with field 0 of blocks 0, 1, ...
                f0 = {BC1: 4, BC3: 2, BC4: 2, BC5: 2, BC7: 8}[fmt]
                assert np.array_equal(s[:f0], x[:f0]) and np.array_equal(s[f0:2 * f0], x[bs:bs + f0]), (fmt, n)


def test_split_merge_match_reference_live(oracle, reference):
    rng = np.random.default_rng(9)
    for fmt in (BC1, BC3, BC4, BC5, BC7):
        for n in (3, 16 * 53, 16 * 53 + 11):
            x = rng.integers(0, 256, n, dtype=np.uint8)
            assert np.array_equal(oracle.bc_split(x, fmt), reference.bc_split(x, fmt)), (fmt, n)
            assert np.array_equal(oracle.bc_merge(x, fmt), reference.bc_merge(x, fmt)), (fmt, n)


def _astc_block_mix(rng, n):
    """Random 16-byte ASTC blocks with void-extent blocks and the reference encoder's own mode words mixed in."""
    blocks = rng.integers(0, 256, (n, 16), dtype=np.uint8)
    blocks[::7, 0] = 0xFC  # void extent: low 9 mode bits 0x1FC
    blocks[::7, 1] = (blocks[::7, 1] & 0xFE) | 0x01
    modes = [0x242, 0x443, 0x642, 0x253, 0x653, 0x243]  # 4x4 grids of several weight ranges, as the encoder writes them
    for k, m in enumerate(modes):
        rows = blocks[3 + k::11]
        rows[:, 0] = m & 0xFF
        rows[:, 1] = (rows[:, 1] & 0xF8) | (m >> 8)
    return blocks


def test_astc_decode_matches_reference_live(oracle, reference):
    """The port's decoder on arbitrary blocks (void extent, supported modes, everything it must reject)."""
    rng = np.random.default_rng(14)
    bc = _astc_block_mix(rng, 24 * 20).reshape(-1)
    assert np.array_equal(oracle.astc_decode(bc, 95, 77), reference.astc_decode(bc, 95, 77))


def test_bc7_decode_all_modes_matches_reference_live(oracle, reference):
    """The port's BC7 decoder on arbitrary blocks: every mode (each block's lowest set bit of byte 0 picks it), every
    partition, rotation and index selector, and the reserved mode."""
    rng = np.random.default_rng(15)
    bc = rng.integers(0, 256, (9 * 512, 16), dtype=np.uint8)
    for m in range(9):  # mode m: bits below m clear, bit m set (m = 8: byte 0 zero, the reserved mode)
        rows = bc[m::9]
        rows[:, 0] = 0 if m == 8 else ((rows[:, 0] >> (m + 1)) << (m + 1)) | (1 << m)
    w, h = 4 * 64, 4 * (9 * 512 // 64)
    assert np.array_equal(oracle.bc_decode(bc.reshape(-1), w, h, BC7), reference.bc_decode(bc.reshape(-1), w, h, BC7))


def test_bc7_fields_rebuild_the_decoder_output(oracle):
    """zo_bc7_fields (the linear form the adjoint tests use) gives back the decoder's texels on every mode."""
    rng = np.random.default_rng(16)
    bc = rng.integers(0, 256, (8 * 64, 16), dtype=np.uint8)
    for m in range(8):
        rows = bc[m::8]
        rows[:, 0] = ((rows[:, 0] >> (m + 1)) << (m + 1)) | (1 << m)
    dec = oracle.bc_decode(bc.reshape(-1), 4 * 8, 4 * 64, BC7).reshape(64, 4, 8, 4, 4).transpose(0, 2, 1, 3, 4).reshape(-1, 16, 4)
    for k in range(bc.shape[0]):
        f = oracle.bc7_fields(bc[k])
        assert f["mode"] == k % 8
        ep, s = f["ep"], f["subset"]
        for i in range(16):
            px = [((64 - f["cw"][i]) * ep[2 * s[i]][c] + f["cw"][i] * ep[2 * s[i] + 1][c] + 32) >> 6 for c in range(3)]
            px.append(((64 - f["aw"][i]) * ep[2 * s[i]][3] + f["aw"][i] * ep[2 * s[i] + 1][3] + 32) >> 6)
            if f["rot"]:
                px[3], px[f["rot"] - 1] = px[f["rot"] - 1], px[3]
            assert px == list(dec[k, i]), (k, i)


# ---------------------------------------------------------------- rate-distortion mode (zap_tex.h:223-306, :786-815)
@pytest.mark.parametrize("rdo", [10.0, 30.0, 300.0])
def test_rdo_port_matches_reference_live(oracle, reference, rdo):
    import zap_b200.synth as S
    rng = np.random.default_rng(int(rdo))
    imgs = [S.colour_texture(64, 48, seed=3, alpha="noise").numpy(), S.colour_texture(37, 29, seed=4).numpy(),
            rng.integers(0, 256, (21, 27, 4), dtype=np.uint8)]
    for img in imgs:
        for fmt in (BC1, BC3, BC4, BC5, BC7):
            assert np.array_equal(oracle.bc_encode(img, fmt, rdo=rdo), reference.bc_encode(img, fmt, rdo=rdo)), (fmt, rdo, img.shape)


def test_rdo_nonpositive_lambda_is_the_plain_encode(oracle):
    img = np.random.default_rng(2).integers(0, 256, (20, 24, 4), dtype=np.uint8)
    for fmt in (BC1, BC7):
        assert np.array_equal(oracle.bc_encode(img, fmt, rdo=-5.0), oracle.bc_encode(img, fmt))


def test_container_files_match_reference_cli(oracle, golden_containers):
    """The restated `zap tex` (zap.c:309-355) against the files the reference CLI wrote: DDS with and without the DX10
    extension, sRGB codes, BC4/BC5 never sRGB, full mip chains down to 1x1, rdo per level, the one-level .astc file."""
    assert len(golden_containers) == 17
    for key, (img, (fmt, rdo, mips, srgb), want) in golden_containers.items():
        got = oracle.tex_file(img, int(fmt), rdo, int(mips), int(srgb))
        assert np.array_equal(got, want), key
        h, w = img.shape[:2]
        if int(fmt) == 6:
            assert np.array_equal(oracle.astc_header(w, h), want[:16]), key
        else:
            hdr = oracle.dds_header(w, h, int(fmt), int(mips), int(srgb))
            assert hdr.size in (128, 148) and np.array_equal(hdr, want[:hdr.size]), key


def test_dds_header_fields(oracle):
    """Field values of zap.c:344-349 for one case per branch, read back as little-endian words."""
    def words(hdr):
        return np.frombuffer(hdr.tobytes(), "<u4")
    h = oracle.dds_header(4096, 2048, 4, 1, 1)
    wd = words(h)
    assert h.size == 148 and bytes(h[:4]) == b"DDS " and wd[1] == 124
    assert wd[3] == 2048 and wd[4] == 4096 and wd[5] == 4096 * 2048 and wd[7] == 13
    assert wd[2] == 0x1 | 0x2 | 0x4 | 0x1000 | 0x80000 | 0x20000 and wd[27] == 0x401008
    assert bytes(h[84:88]) == b"DX10" and wd[32] == 99 and wd[33] == 3 and wd[35] == 1
    h = oracle.dds_header(5, 3, 2, 0, 1)  # BC4: sRGB ignored, no DX10 extension
    wd = words(h)
    assert h.size == 128 and bytes(h[84:88]) == b"BC4U" and wd[7] == 1 and wd[2] == 0x81007 and wd[27] == 0x1000
    assert oracle.dds_header(8, 8, 0, 0, 1).size == 148 and words(oracle.dds_header(8, 8, 0, 0, 1))[32] == 72
    a = oracle.astc_header(0x123456, 0x10203)
    assert list(a) == [0x13, 0xAB, 0xA1, 0x5C, 4, 4, 1, 0x56, 0x34, 0x12, 0x03, 0x02, 0x01, 1, 0, 0]
