"""Generate tests/golden/golden_containers.npz by running the REFERENCE CLI itself (oracle/_ref/zap, built from zap.c).

Run from the repo root where the reference tree exists:  make -C oracle ref && python tests/golden/make_containers.py
Each case runs `zap tex -f <fmt> [-r rdo] [-m] [-S] w h in.rgba out` (zap.c:309-355) on a seeded RGBA8 image and stores
the file it wrote, byte for byte, next to the input and the arguments, so tests need neither the reference nor the CLI.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
from make_golden import seeded_image  # noqa: E402

FMT_IDS = {"bc1": 0, "bc3": 1, "bc4": 2, "bc5": 3, "bc7": 4, "astc": 6}

IMAGES = {
    "odd37x21": seeded_image(3001, 37, 21, 1),
    "wide64x40": seeded_image(3002, 64, 40, 2),
    "tiny1x1": seeded_image(3003, 1, 1, 1),
    "opaque16x9": seeded_image(3004, 16, 9, 0),
}

# (image, format, rdo, mips, srgb)
CASES = [
    ("odd37x21", "bc1", 0.0, 0, 0), ("odd37x21", "bc1", 0.0, 1, 0), ("wide64x40", "bc1", 0.0, 1, 1),
    ("odd37x21", "bc3", 0.0, 1, 1), ("wide64x40", "bc4", 0.0, 1, 1), ("odd37x21", "bc5", 0.0, 1, 0),
    ("opaque16x9", "bc7", 0.0, 0, 0), ("wide64x40", "bc7", 0.0, 1, 1), ("odd37x21", "bc7", 20.0, 1, 0),
    ("wide64x40", "bc1", 40.0, 1, 0), ("odd37x21", "bc3", 15.0, 0, 1), ("tiny1x1", "bc1", 0.0, 1, 0),
    ("tiny1x1", "bc7", 0.0, 1, 1), ("odd37x21", "astc", 0.0, 0, 0), ("wide64x40", "astc", 0.0, 1, 1),
    ("tiny1x1", "astc", 0.0, 0, 0), ("opaque16x9", "bc5", 0.0, 0, 1),
]


def main():
    cli = os.path.join(ROOT, "oracle", "_ref", "zap")
    if not os.path.exists(cli):
        sys.exit("oracle/_ref/zap is required (run make -C oracle ref where the reference tree exists)")
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, img in IMAGES.items():
            out["img/" + name] = img
            img.tofile(os.path.join(tmp, name + ".rgba"))
        for n, (name, fmt, rdo, mips, srgb) in enumerate(CASES):
            h, w = IMAGES[name].shape[:2]
            dst = os.path.join(tmp, f"case{n}.{'astc' if fmt == 'astc' else 'dds'}")
            args = [cli, "tex", "-f", fmt] + (["-r", repr(rdo)] if rdo else []) + (["-m"] if mips else []) + \
                   (["-S"] if srgb else []) + [str(w), str(h), os.path.join(tmp, name + ".rgba"), dst]
            subprocess.run(args, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            key = f"case{n:02d}"
            out["file/" + key] = np.fromfile(dst, np.uint8)
            out["args/" + key] = np.array([FMT_IDS[fmt], rdo, mips, srgb], np.float64)
            out["image/" + key] = np.array(name)
    path = os.path.join(HERE, "golden_containers.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(CASES)} files, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
