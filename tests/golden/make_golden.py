"""Generate tests/golden/golden_tex.npz by running the REFERENCE encoder itself (oracle/_ref/libzapref.so).

Run from the repo root where the reference tree exists:  python tests/golden/make_golden.py
The fixture stores every input next to the reference's output, so tests never need the generator or the
reference at run time. Inputs:
  - the reference self-test's own images (tex_bench.c): the 67x45 BCn image (srand(3), glibc rand), the 64x64
    independent-alpha BC7 image, the two 64x48 ASTC images and the 37x21 HDR gradient;
  - seeded odd-size images (1x1 .. 45x33) with smooth gradients, hard edges and noise, opaque and with alpha.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import oracle_lib  # noqa: E402


def selftest_bcn_image():
    """tex_bench.c:147-154 (uses the C library's rand(), seeded with 3)."""
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(3)
    W, H = 67, 45
    img = np.zeros((H, W, 4), np.uint8)
    for y in range(H):
        for x in range(W):
            img[y, x] = (x * 255 // W, y * 255 // H, ((x + y) * 2 + libc.rand() % 8) & 255, 255 if x < 30 else (x * y) & 255)
    return img


def selftest_mode5_image():
    """tex_bench.c:76 (alpha varies independently of colour)."""
    i = np.arange(64 * 64)
    img = np.zeros((64 * 64, 4), np.uint8)
    img[:, 0] = (i % 64 * 4) & 255
    img[:, 1] = (i // 64 * 4) & 255
    img[:, 2] = 90
    img[:, 3] = ((255 - i % 64 * 4) ^ (i // 64 * 4)) & 255
    return img.reshape(64, 64, 4)


def selftest_astc_image(k):
    """tex_bench.c:129-134."""
    W, H = 64, 48
    img = np.zeros((H, W, 4), np.uint8)
    for y in range(H):
        for x in range(W):
            edge = (x + 2 * y) % 13 < 6
            img[y, x] = (220 if edge else 30 + x, 40 if edge else 200 - y, (x * 3) & 255, ((x * 5 + y * 3) & 255) if k else 255)
    return img


def selftest_hdr_image():
    """tex_bench.c:54-57."""
    W, H = 37, 21
    img = np.zeros((H, W, 4), np.float32)
    for y in range(H):
        for x in range(W):
            img[y, x, 0] = np.float32(0.05) * np.float32(1 << (x // 6))
            img[y, x, 1] = np.float32(0.5) + np.float32(y) * np.float32(0.25)
            img[y, x, 2] = np.float32(10000.0) if (x == 20 and y == 10) else np.float32(0.01) * np.float32(x + 1)
            img[y, x, 3] = 1
    return img


def seeded_image(seed, w, h, alpha):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    img = np.zeros((h, w, 4))
    for c in range(4):
        img[..., c] = rng.uniform(40, 200) + rng.uniform(-3, 3) * x + rng.uniform(-3, 3) * y
    for _ in range(3):
        x0, y0 = rng.integers(0, max(1, w), 2)
        img[y0:y0 + rng.integers(1, 12), x0:x0 + rng.integers(1, 12), :3] = rng.integers(0, 256, 3)
    img += rng.normal(0, 6, img.shape)
    if not alpha:
        img[..., 3] = 255
    elif alpha == 2:
        img[..., 3] = np.where(rng.random((h, w)) < 0.3, 0, img[..., 3])
    return np.clip(img, 0, 255).astype(np.uint8)


def seeded_hdr(seed, w, h):
    rng = np.random.default_rng(seed)
    lum = 2.0 ** rng.uniform(-8, 8, (h, w))
    hue = rng.uniform(0.2, 1.0, (h, w, 3))
    img = np.ones((h, w, 4), np.float32)
    img[..., :3] = (lum[..., None] * hue).astype(np.float32)
    img[0, 0, 0] = -1.0  # negative clamps to 0
    return img


def main():
    ref = oracle_lib.reference()
    if ref is None:
        sys.exit("oracle/_ref/libzapref.so is required (run make -C oracle ref where the reference tree exists)")
    out = {}
    images = {
        "selftest67x45": selftest_bcn_image(),
        "mode5_64x64": selftest_mode5_image(),
        "astc64x48_k0": selftest_astc_image(0),
        "astc64x48_k1": selftest_astc_image(1),
    }
    sizes = [(1, 1), (2, 1), (3, 2), (5, 3), (4, 4), (13, 7), (32, 32), (45, 33)]
    for n, (w, h) in enumerate(sizes):
        for alpha in (0, 1, 2):
            images[f"seed{n}_{w}x{h}_a{alpha}"] = seeded_image(1000 + 10 * n + alpha, w, h, alpha)
    for name, img in images.items():
        out["img/" + name] = img
        for fmt in range(5):
            out[f"bc{fmt}/{name}"] = ref.bc_encode(img, fmt)
        out["astc/" + name] = ref.astc_encode(img)
        out["mip0/" + name] = ref.mip_next(img, 0)
        out["mip1/" + name] = ref.mip_next(img, 1)
    hdr = {"hdr37x21": selftest_hdr_image()}
    for n, (w, h) in enumerate([(1, 1), (5, 3), (16, 16), (23, 9)]):
        hdr[f"hdrseed{n}_{w}x{h}"] = seeded_hdr(2000 + n, w, h)
    for name, img in hdr.items():
        out["himg/" + name] = img
        out["bc6h/" + name] = ref.bc6h_encode(img)
        out["mipf/" + name] = ref.mip_next_f(img)
    lin, thr = ref.srgb_tables()
    out["srgb_lin"] = lin
    out["srgb_thr"] = thr
    path = os.path.join(HERE, "golden_tex.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
