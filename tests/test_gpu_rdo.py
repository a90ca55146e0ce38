"""Rate-distortion mode (zap_bc_encode with rdo > 0, zap_tex.h:223-306, :786-815) on the device, byte for byte.

One chain per call: the host drop-in and the device entry against the oracle's single call. Banded chains: each
band of block rows against one oracle call on that band's rows, as callers that encode in bands run the reference.
Edge cases: odd sizes (partial blocks, one block row, one block column), lambda <= 0 (the plain encode), and the
non-finite lambdas the entry points reject.
"""
import numpy as np
import pytest

import oracle_lib
from oracle_lib import BC1, BC3, BC4, BC5, BC7

pytestmark = pytest.mark.gpu
FORMATS = (BC1, BC3, BC4, BC5, BC7)


def _images():
    import zap_b200.synth as S
    rng = np.random.default_rng(51)
    return [S.colour_texture(96, 72, seed=52, alpha="noise").numpy(), S.colour_texture(61, 37, seed=53).numpy(),
            rng.integers(0, 256, (9, 70, 4), dtype=np.uint8), S.colour_texture(3, 45, seed=54).numpy()]


@pytest.mark.parametrize("rdo", [10.0, 100.0])
def test_rdo_one_chain_matches_oracle(cuda_lib, oracle, reference, rdo):
    import torch
    for img in _images():
        t = torch.from_numpy(np.ascontiguousarray(img)).cuda()
        for fmt in FORMATS:
            want = oracle.bc_encode(img, fmt, rdo=rdo)
            assert np.array_equal(want, reference.bc_encode(img, fmt, rdo=rdo))
            assert np.array_equal(cuda_lib.bc_encode(img, fmt, rdo=rdo), want), (fmt, rdo, img.shape)
            dev = cuda_lib.bc_encode_rdo_dev(t, fmt, rdo)
            torch.cuda.synchronize()
            assert np.array_equal(dev.cpu().numpy(), want), (fmt, rdo, img.shape)


def test_rdo_bands_match_one_oracle_call_per_band(cuda_lib, oracle):
    import torch

    import zap_b200.synth as S
    img = S.colour_texture(128, 100, seed=55, alpha="noise").numpy()
    t = torch.from_numpy(np.ascontiguousarray(img)).cuda()
    h = img.shape[0]
    for fmt in FORMATS:
        for band_rows in (8, 3):
            got = cuda_lib.bc_encode_rdo_dev(t, fmt, 30.0, band_rows=band_rows)
            torch.cuda.synchronize()
            want = np.concatenate([oracle.bc_encode(img[y0:min(h, y0 + 4 * band_rows)], fmt, rdo=30.0)
                                   for y0 in range(0, h, 4 * band_rows)])
            assert np.array_equal(got.cpu().numpy(), want), (fmt, band_rows)


def test_rdo_lambda_rules(cuda_lib, oracle):
    import torch
    img = np.random.default_rng(56).integers(0, 256, (24, 20, 4), dtype=np.uint8)
    t = torch.from_numpy(img).cuda()
    for fmt in (BC1, BC7):
        plain = oracle.bc_encode(img, fmt)
        assert np.array_equal(cuda_lib.bc_encode(img, fmt, rdo=-3.0), plain)
        assert np.array_equal(cuda_lib.bc_encode_rdo_dev(t, fmt, 0.0).cpu().numpy(), plain)
        for bad in (float("nan"), float("inf")):
            with pytest.raises(cuda_lib.ZapTexError) as e:
                cuda_lib.bc_encode(img, fmt, rdo=bad)
            assert e.value.status == -1
    assert oracle_lib.bc_size(20, 24, BC7) == 16 * 30
