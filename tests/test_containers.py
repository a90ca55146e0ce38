"""The CLI's texture containers (zap.c:309-355) through the C ABI, host side: the DDS and .astc header writers touch no
device, so they run here against the files the reference CLI wrote and against the restated headers."""
import numpy as np

import zap_b200


def test_headers_match_reference_cli_files(golden_containers):
    for key, (img, (fmt, rdo, mips, srgb), want) in golden_containers.items():
        h, w = img.shape[:2]
        if int(fmt) == 6:
            assert np.array_equal(zap_b200.astc_header(w, h), want[:16]), key
        else:
            hdr = zap_b200.dds_header(w, h, int(fmt), int(mips), int(srgb))
            assert np.array_equal(hdr, want[:hdr.size]), key
        # the declared file size is the reference's file size
        assert zap_b200.load().zap_tex_cuda_tex_file_bytes(w, h, int(fmt), int(mips), int(srgb)) == want.size, key


def test_headers_match_oracle_over_sizes_and_flags(oracle):
    lib = zap_b200.load()
    for w, h in ((1, 1), (3, 7), (4096, 2048), (65535, 3), (1 << 24, 1 << 24), (1000, 1)):
        for fmt in range(5):
            for mips in (0, 1):
                for srgb in (0, 1, 7):
                    assert np.array_equal(zap_b200.dds_header(w, h, fmt, mips, srgb), oracle.dds_header(w, h, fmt, mips, srgb)), \
                        (w, h, fmt, mips, srgb)
                    want = oracle.dds_header(w, h, fmt, mips, srgb).size + sum(
                        zap_b200.bc_size(max(1, w >> l), max(1, h >> l), fmt) for l in range(zap_b200.mip_levels(w, h) if mips else 1))
                    assert lib.zap_tex_cuda_tex_file_bytes(w, h, fmt, mips, srgb) == want
        assert np.array_equal(zap_b200.astc_header(w, h), oracle.astc_header(w, h))


def test_header_argument_errors():
    lib = zap_b200.load()
    buf = np.zeros(148, np.uint8)
    assert lib.zap_tex_cuda_dds_header(0, 4, 0, 0, 0, buf.ctypes.data, None) == -1
    assert lib.zap_tex_cuda_dds_header(4, 4, 5, 0, 0, buf.ctypes.data, None) == -2  # BC6H has no DDS path in the CLI
    assert lib.zap_tex_cuda_dds_header(4, 4, 0, 0, 0, None, None) == -1
    assert lib.zap_tex_cuda_astc_header(4, 0, buf.ctypes.data) == -1
    assert lib.zap_tex_cuda_tex_file_bytes(4, 4, 5, 0, 0) == 0 and lib.zap_tex_cuda_tex_file_bytes(0, 4, 0, 0, 0) == 0
    img = np.zeros((4, 4, 4), np.uint8)
    out = np.zeros(64, np.uint8)
    # out_cap below the file size is rejected before any device work
    assert lib.zap_tex_cuda_tex_file(None, img.ctypes.data, 4, 4, 16, 0, 0.0, 0, 0, out.ctypes.data, 10) == -1
