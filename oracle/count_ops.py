"""Counts the reference algorithm's algorithmic operations per texture for the bench workloads (test infrastructure).

Runs the C restatement built with op counters (make -C oracle ops -> oracle/liboracle_ops.so) over the same
synthetic textures bench.py encodes, and writes profiles/alu_ops.json, which bench.py reads for its ALU roofline.
What is counted (zt_oracle.c, ZO_OPS): every texel-to-palette-entry distance of the encoder's searches at
3C + 1 ops for C channels (differences, squares, accumulations, one comparison), and the 9 additions per texel
of the BC7 mode 1 partition ranking's moment sums. PCA, least-squares and packing work is not counted, so the
figures are a lower bound on the algorithm's arithmetic.

    python oracle/count_ops.py            # a few minutes on one core
"""
import ctypes as C
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

import zap_b200.synth as S  # noqa: E402

W = H = 2048
BC1, BC4, BC5, BC7 = 0, 2, 3, 4


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ops"], check=True)
    lib = C.CDLL(os.path.join(ROOT, "oracle", "liboracle_ops.so"))
    lib.zo_bc_encode.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_size_t, C.c_int, C.c_float, C.c_void_p]
    lib.zo_ops_take.argtypes = [C.POINTER(C.c_uint64)]
    lib.zo_astc_encode.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_size_t, C.c_void_p]
    lib.zo_bc6h_encode.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_size_t, C.c_void_p]
    blocks = (W // 4) * (H // 4)

    def count(img, fmt):
        """fmt 0..4: zap_bc_encode; 6: ASTC 4x4; 5: BC6H (img: RGBA float32)"""
        img = np.ascontiguousarray(img)
        out = np.zeros(blocks * 16, np.uint8)
        ops = (C.c_uint64 * 2)()
        lib.zo_ops_take(ops)  # clear
        if fmt == 6:
            lib.zo_astc_encode(img.ctypes.data, W, H, W * 4, out.ctypes.data)
        elif fmt == 5:
            lib.zo_bc6h_encode(img.ctypes.data, W, H, W * 4, out.ctypes.data)
        else:
            lib.zo_bc_encode(img.ctypes.data, W, H, W * 4, fmt, 0.0, out.ctypes.data)
        lib.zo_ops_take(ops)
        return int(ops[0]), int(ops[1])

    def widen(x):  # R8 / RG8 as the reference reads them: missing channels 0, alpha 255
        img = np.zeros((H, W, 4), np.uint8)
        img[..., :x.shape[2]] = x
        img[..., 3] = 255
        return img

    def spread(v):  # seed-to-seed spread of the count, % of the mean
        return float(100.0 * np.std(v) / np.mean(v))

    t0 = time.time()
    # BC7: the headline ring of bench.py (rank 0): colour_texture(2048, 2048, seed=100 + k, alpha="noise"), k < 10
    tot, m6 = [], []
    for k in range(10):
        a, b = count(S.colour_texture(W, H, seed=100 + k, alpha="noise").numpy(), BC7)
        tot.append(a)
        m6.append(b)
    bc7 = {"textures": "colour_texture(2048, 2048, seed=100 + k, alpha='noise'), k = 0..9 (the bench ring's recipe and seeds)",
           "blocks_per_texture": blocks,
           "ops_per_texture": {"bc7_mode6": float(np.mean(m6)), "bc7_modes51": float(np.mean(tot) - np.mean(m6))},
           "spread_pct": {"bc7_mode6": spread(m6), "bc7_modes51": spread(np.array(tot) - np.array(m6))}}
    # BC1: the ring of bench.py's 2048^2 BC1 figure: colour_texture(2048, 2048, seed=k), k < 10
    ops1 = [count(S.colour_texture(W, H, seed=k).numpy(), BC1)[0] for k in range(10)]
    bc1 = {"textures": "colour_texture(2048, 2048, seed=k), k = 0..9 (the bench's BC1 2048x2048 ring's recipe and seeds)",
           "blocks_per_texture": blocks, "ops_per_texture": {"bc1_encode": float(np.mean(ops1))}, "spread_pct": {"bc1_encode": spread(ops1)}}
    # the other formats' rings (their first 10 or 6 textures): BC4 from R8, BC5 from RG8, ASTC 4x4, BC6H from RGB16F
    o4 = [count(widen(S.colour_texture(W, H, seed=k).numpy()[..., :1]), BC4)[0] for k in range(10)]
    o5 = [count(widen(S.normal_map(W, H, seed=k).numpy()), BC5)[0] for k in range(10)]
    oa = [count(S.colour_texture(W, H, seed=k, alpha="noise").numpy(), 6)[0] for k in range(10)]
    o6 = []
    for k in range(6):
        f = np.ones((H, W, 4), np.float32)
        f[..., :3] = S.hdr_texture(W, H, seed=k).numpy().astype(np.float32)
        o6.append(count(f, 5)[0])
    other = {"textures": "the bench's rings for these figures (recipes and seeds): colour_texture(seed=k)[..., :1] (BC4), "
                         "normal_map(seed=k) (BC5), colour_texture(seed=k, alpha='noise') (ASTC), hdr_texture(seed=k) (BC6H)",
             "blocks_per_texture": blocks,
             "ops_per_texture": {"bc4_encode": float(np.mean(o4)), "bc5_encode": float(np.mean(o5)), "astc_encode": float(np.mean(oa)),
                                 "bc6h_encode": float(np.mean(o6))},
             "spread_pct": {"bc4_encode": spread(o4), "bc5_encode": spread(o5), "astc_encode": spread(oa), "bc6h_encode": spread(o6)}}
    res = {"definition": "palette-search ops of the reference algorithm (3C + 1 per texel-to-entry distance over C "
                         "channels) + 9 per texel of the BC7 mode 1 moment sums; counted by the C restatement "
                         "(oracle/zt_oracle.c built with -DZO_COUNT_OPS); a lower bound on the algorithm's arithmetic",
           "textures_note": "generated on the CPU with the bench's recipes and seeds; bench.py generates its rings on the GPU, "
                            "whose random stream differs, so a count is the mean over textures of the same recipe "
                            "(spread_pct: the seed-to-seed standard deviation, % of the mean)",
           "command": "python oracle/count_ops.py", "bc7": bc7, "bc1": bc1, "other": other}
    path = os.path.join(ROOT, "profiles", "alu_ops.json")
    with open(path, "w") as f:
        json.dump(res, f, indent=1)
        f.write("\n")
    print(json.dumps(res, indent=1), f"\n{time.time() - t0:.1f} s")


if __name__ == "__main__":
    main()
