"""Split / merge (zap_tex.h:1549-1571) on the device, and encoding straight into the split form, against the oracle.

Byte-exact: the host drop-ins (zap_tex_cuda_bc_split / _merge), the device-memory variants (aligned and unaligned
buffers, stray tail bytes) and zap_tex_cuda_bc_encode_split_dev, whose output must equal the oracle's
bc_split(bc_encode(image)).
"""
import numpy as np
import pytest

import oracle_lib
from oracle_lib import BC1, BC3, BC4, BC5, BC7

pytestmark = pytest.mark.gpu
FORMATS = (BC1, BC3, BC4, BC5, BC7)


def test_host_split_merge_match_oracle(cuda_lib, oracle):
    rng = np.random.default_rng(21)
    for fmt in FORMATS:
        for n in (0, 7, 16, 16 * 1000, 16 * 1000 + 5, 8 * 4099 + 3):
            x = rng.integers(0, 256, n, dtype=np.uint8)
            s = cuda_lib.bc_split(x, fmt)
            assert np.array_equal(s, oracle.bc_split(x, fmt)), (fmt, n)
            assert np.array_equal(cuda_lib.bc_merge(s, fmt), x), (fmt, n)


def test_device_split_merge_aligned_and_unaligned(cuda_lib, oracle):
    import torch
    rng = np.random.default_rng(22)
    for fmt in FORMATS:
        for off in (0, 1, 3):  # offset views exercise the byte-wise path
            n = 16 * 777 + 9
            x = rng.integers(0, 256, n + off, dtype=np.uint8)
            d = torch.from_numpy(x).cuda()[off:]
            s = cuda_lib.bc_split_dev(d, fmt)
            torch.cuda.synchronize()
            assert np.array_equal(s.cpu().numpy(), oracle.bc_split(x[off:], fmt)), (fmt, off)
            m = cuda_lib.bc_merge_dev(s, fmt)
            torch.cuda.synchronize()
            assert np.array_equal(m.cpu().numpy(), x[off:]), (fmt, off)


def test_encode_split_matches_encode_then_split(cuda_lib, oracle):
    import torch

    import zap_b200.synth as S
    imgs = [S.colour_texture(256, 192, seed=31, alpha="noise").numpy(), S.colour_texture(61, 37, seed=32).numpy(),
            np.random.default_rng(33).integers(0, 256, (45, 33, 4), dtype=np.uint8)]
    for img in imgs:
        h, w = img.shape[:2]
        t = torch.from_numpy(np.ascontiguousarray(img)).cuda()
        for fmt in FORMATS:
            got = cuda_lib.bc_encode_split_dev(t, fmt)
            torch.cuda.synchronize()
            want = oracle.bc_split(oracle.bc_encode(img, fmt), fmt)
            assert np.array_equal(got.cpu().numpy(), want), (fmt, w, h)
            blocks = cuda_lib.bc_merge_dev(got, fmt)
            ref = cuda_lib.bc_encode_dev(t, fmt)
            torch.cuda.synchronize()
            assert torch.equal(blocks, ref), (fmt, w, h)


def test_split_rejects_overlap_and_formats(cuda_lib):
    import torch
    x = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    with pytest.raises(cuda_lib.ZapTexError) as e:
        cuda_lib.bc_split_dev(x, BC7, out=x)  # in place: the reference needs distinct buffers
    assert e.value.status == -1  # ZTC_ERR_INVALID_ARG
    with pytest.raises(cuda_lib.ZapTexError) as e:
        cuda_lib.bc_split_dev(x, 5)  # BC6H has no split form
    assert e.value.status == -2  # ZTC_ERR_UNSUPPORTED
    assert oracle_lib.block_bytes(BC7) == 16
