"""Device ASTC 4x4 decoder (zap_astc_decode, zap_tex.h:1344-1356) and the host-memory decoder drop-ins, against
the oracle, byte for byte: blocks from the encoder, the committed golden ASTC blocks, and arbitrary blocks that
exercise the void-extent path and every rejection (which decodes to magenta, as in the reference)."""
import numpy as np
import pytest

from oracle_lib import BC1, BC3, BC4, BC5, BC7
from test_oracle import _astc_block_mix

pytestmark = pytest.mark.gpu


def test_astc_decode_dev_matches_oracle(cuda_lib, oracle, golden):
    import torch

    import zap_b200.synth as S
    rng = np.random.default_rng(41)
    cases = []
    for name in sorted(k[4:] for k in golden if k.startswith("img/")):
        img = golden["img/" + name]
        cases.append((golden["astc/" + name], img.shape[1], img.shape[0]))
    img = S.colour_texture(203, 131, seed=42, alpha="noise").numpy()
    cases.append((cuda_lib.astc_encode(img), 203, 131))
    cases.append((_astc_block_mix(rng, 40 * 30).reshape(-1), 160, 119))
    decoded_any = 0
    for bc, w, h in cases:
        d = torch.from_numpy(np.ascontiguousarray(bc)).cuda()
        got = cuda_lib.astc_decode_dev(d, w, h)
        torch.cuda.synchronize()
        want = oracle.astc_decode(bc, w, h)
        assert np.array_equal(got.cpu().numpy(), want), (w, h)
        assert np.array_equal(cuda_lib.astc_decode(bc, w, h), want), (w, h)
        decoded_any += int((want.reshape(-1, 4) != [255, 0, 255, 255]).any(axis=1).sum())
    assert decoded_any > 0


def test_host_decoders_match_oracle(cuda_lib, oracle):
    import zap_b200.synth as S
    img = S.colour_texture(90, 70, seed=43, alpha="noise").numpy()
    for fmt in (BC1, BC3, BC4, BC5, BC7):
        bc = oracle.bc_encode(img, fmt)
        assert np.array_equal(cuda_lib.bc_decode(bc, 90, 70, fmt), oracle.bc_decode(bc, 90, 70, fmt)), fmt
    hdr = np.ones((37, 45, 4), np.float32)
    hdr[..., :3] = S.hdr_texture(45, 37, seed=44).numpy().astype(np.float32)
    bc = oracle.bc6h_encode(hdr)
    assert np.array_equal(cuda_lib.bc6h_decode(bc, 45, 37), oracle.bc6h_decode(bc, 45, 37))


def test_device_entry_points_reject_misaligned_pointers(cuda_lib):
    """Vector loads / stores need aligned device pointers; a misaligned one is an argument error, never a launch."""
    import torch
    d = torch.zeros(4096 + 16, dtype=torch.uint8, device="cuda")
    img = torch.zeros((16, 16, 4), dtype=torch.uint8, device="cuda")
    hdr = torch.zeros((16, 16, 4), dtype=torch.float32, device="cuda")
    calls = (lambda: cuda_lib.astc_decode_dev(d[1:], 16, 16), lambda: cuda_lib.bc_decode_dev(d[4:], 16, 16, BC7),
             lambda: cuda_lib.bc6h_decode_dev(d[8:], 16, 16), lambda: cuda_lib.bc_encode_dev(img, BC7, out=d[8:]),
             lambda: cuda_lib.bc_encode_dev(img, BC1, out=d[4:]),
             lambda: cuda_lib.bc6h_encode_dev(hdr, out=d[4:4100]))
    for k, call in enumerate(calls):
        with pytest.raises(cuda_lib.ZapTexError) as e:
            call()
        assert e.value.status == -1, k  # ZTC_ERR_INVALID_ARG, before any launch
    torch.cuda.synchronize()  # the device is untouched
