"""Whole texture files as the CLI's `zap tex` writes them (zap.c:309-355), with the mip chain and every level's blocks
computed on the device: byte for byte against the files the reference CLI wrote, and against the restated CLI on
larger, odd-sized images (full chains down to 1x1, sRGB, rdo per level, .astc)."""
import numpy as np
import pytest

import oracle_lib

pytestmark = pytest.mark.gpu


def test_tex_files_match_reference_cli(cuda_lib, golden_containers):
    for key, (img, (fmt, rdo, mips, srgb), want) in golden_containers.items():
        got = cuda_lib.tex_file(img, int(fmt), rdo, int(mips), int(srgb))
        assert np.array_equal(got, want), key


@pytest.mark.parametrize("fmt,rdo,mips,srgb", [(0, 0.0, 1, 1), (1, 0.0, 1, 1), (2, 0.0, 1, 1), (3, 0.0, 1, 0),
                                               (4, 0.0, 1, 1), (4, 25.0, 1, 0), (0, 60.0, 1, 0), (6, 0.0, 1, 0)])
def test_tex_files_match_oracle(cuda_lib, oracle, fmt, rdo, mips, srgb):
    import zap_b200.synth as S
    for w, h, seed in ((173, 90, 61), (256, 33, 62)):
        img = S.colour_texture(w, h, seed=seed, alpha="noise").numpy()
        want = oracle.tex_file(img, fmt, rdo, mips, srgb)
        got = cuda_lib.tex_file(img, fmt, rdo, mips, srgb)
        assert got.size == want.size and np.array_equal(got, want), (fmt, rdo, mips, srgb, w, h)


def test_tex_file_strided_source(cuda_lib, oracle):
    """A source with row padding gives the file of the tightly packed image."""
    rng = np.random.default_rng(63)
    padded = rng.integers(0, 256, (45, 80, 4), dtype=np.uint8)
    img = padded[:, :67]
    want = oracle.tex_file(np.ascontiguousarray(img), oracle_lib.BC7, 0.0, 1, 1)
    got = cuda_lib.tex_file(img, oracle_lib.BC7, 0.0, 1, 1)
    assert np.array_equal(got, want)
