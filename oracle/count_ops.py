"""Counts the reference algorithm's algorithmic operations per texture for the bench workloads (test infrastructure).

Runs the C restatement built with op counters (make -C oracle ops -> oracle/liboracle_ops.so) over the same
synthetic textures bench.py encodes, and writes profiles/alu_ops.json, which bench.py reads for its ALU roofline.
What is counted (zt_oracle.c, ZO_OPS): every texel-to-palette-entry distance of the encoder's searches at
3C + 1 ops for C channels (differences, squares, accumulations, one comparison), and the 9 additions per texel
of the BC7 mode 1 partition ranking's moment sums. PCA, least-squares and packing work is not counted, so the
figures are a lower bound on the algorithm's arithmetic.

    python oracle/count_ops.py            # about a minute on one core
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
BC1, BC7 = 0, 4


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ops"], check=True)
    lib = C.CDLL(os.path.join(ROOT, "oracle", "liboracle_ops.so"))
    lib.zo_bc_encode.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_size_t, C.c_int, C.c_float, C.c_void_p]
    lib.zo_ops_take.argtypes = [C.POINTER(C.c_uint64)]
    blocks = (W // 4) * (H // 4)

    def count(img, fmt):
        img = np.ascontiguousarray(img)
        out = np.zeros(blocks * (8 if fmt == BC1 else 16), np.uint8)
        ops = (C.c_uint64 * 2)()
        lib.zo_ops_take(ops)  # clear
        lib.zo_bc_encode(img.ctypes.data, W, H, W * 4, fmt, 0.0, out.ctypes.data)
        lib.zo_ops_take(ops)
        return int(ops[0]), int(ops[1])

    t0 = time.time()
    # BC7: the headline ring of bench.py (rank 0): colour_texture(2048, 2048, seed=100 + k, alpha="noise"), k < 10
    tot, m6 = [], []
    for k in range(10):
        a, b = count(S.colour_texture(W, H, seed=100 + k, alpha="noise").numpy(), BC7)
        tot.append(a)
        m6.append(b)
    bc7 = {"textures": "colour_texture(2048, 2048, seed=100 + k, alpha='noise'), k = 0..9 (the bench ring)",
           "blocks_per_texture": blocks,
           "ops_per_texture": {"bc7_mode6": float(np.mean(m6)), "bc7_modes51": float(np.mean(tot) - np.mean(m6))}}
    # BC1: the ring of bench.py's 2048^2 BC1 figure: colour_texture(2048, 2048, seed=k), k < 10
    ops1 = [count(S.colour_texture(W, H, seed=k).numpy(), BC1)[0] for k in range(10)]
    bc1 = {"textures": "colour_texture(2048, 2048, seed=k), k = 0..9 (the bench's BC1 2048x2048 ring)", "blocks_per_texture": blocks,
           "ops_per_texture": {"bc1_encode": float(np.mean(ops1))}}
    res = {"definition": "palette-search ops of the reference algorithm (3C + 1 per texel-to-entry distance over C "
                         "channels) + 9 per texel of the BC7 mode 1 moment sums; counted by the C restatement "
                         "(oracle/zt_oracle.c built with -DZO_COUNT_OPS); a lower bound on the algorithm's arithmetic",
           "command": "python oracle/count_ops.py", "bc7": bc7, "bc1": bc1}
    path = os.path.join(ROOT, "profiles", "alu_ops.json")
    with open(path, "w") as f:
        json.dump(res, f, indent=1)
        f.write("\n")
    print(json.dumps(res, indent=1), f"\n{time.time() - t0:.1f} s")


if __name__ == "__main__":
    main()
