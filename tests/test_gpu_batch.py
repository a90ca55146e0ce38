"""Batched encoder (mixed sizes, full mip chains, mixed formats, one graph launch) against the oracle.

Every level of every texture must equal the reference's bytes: level 0 encoded from the source, level l from the
reference mip generator iterated l times. The graph must re-read its inputs on every replay, and the plain
per-texture path must give the same bytes.
"""
import numpy as np
import pytest

import oracle_lib

pytestmark = pytest.mark.gpu


def _make(seed, w, h, alpha):
    import zap_b200.synth as S
    return S.colour_texture(w, h, seed=seed, alpha=alpha, device="cuda")


def _check_item(batch, i, ref, srgb):
    tex = batch.textures[i].cpu().numpy()
    fmt = batch.formats[i]
    cur = tex
    for lv, view in enumerate(batch.level_views(i)):
        if lv > 0:
            cur = ref.mip_next(cur, srgb and fmt not in (oracle_lib.BC4, oracle_lib.BC5))
        exp = ref.bc_encode(cur, fmt)
        got = view.cpu().numpy()
        assert np.array_equal(got, exp), (i, fmt, tex.shape, lv, int(np.sum(got != exp)))


@pytest.mark.parametrize("autotune,graph,plan", [(False, True, ()), (True, True, ()), (False, False, ()),
                                                 (False, True, ("tiles_2d", "regs_loose", "tile_x4", "cta_64")),
                                                 (False, True, ("tiles_2d", "tile_x2", "cta_256")),
                                                 (False, True, ("regs_loose", "tile_x2"))])
def test_batch_matches_oracle(cuda_lib, autotune, graph, plan):
    """Every launch plan the autotuner can pick (CTA size, register cap, blocks per tile, strip or 2-D tiles) gives the
    reference's bytes."""
    import torch
    ref = oracle_lib.best()
    sizes = [(1, 1), (3, 2), (5, 3), (17, 9), (64, 64), (128, 32), (96, 200), (256, 256), (300, 131), (33, 257), (512, 128), (7, 70)]
    fmts = [0, 1, 2, 3, 4, 4, 0, 4, 1, 4, 0, 3]
    texs = [_make(100 + k, w, h, "noise" if fmts[k] in (1, 4) and k % 2 else "opaque") for k, (w, h) in enumerate(sizes)]
    srgb = [k % 3 != 0 for k in range(len(sizes))]
    levels = [0] * len(sizes)
    levels[4] = 2  # a partial chain
    b = cuda_lib.Batch(texs, fmts, srgb=srgb, levels=levels, autotune=autotune, graph=graph, plan=plan)
    b.run()
    torch.cuda.synchronize()
    for i in range(len(texs)):
        _check_item(b, i, ref, srgb[i])
    info = b.info()
    if autotune:
        for knob in ("cta", "regs", "blocks_per_tile", "shape", "hard_grid", "tuned_ms"):
            assert knob in info, (knob, info)
    if "tiles_2d" in plan:
        assert "shape 2d_" in info
    if "regs_loose" in plan:
        assert "regs loose" in info
    b.close()


def test_batch_workload_recipe_matches_oracle(cuda_lib):
    """The batched workload's own recipe at 256 textures (power-of-two sides 64..512, aspect <= 4:1, full sRGB mip
    chains, 40 % BC1 / 20 % BC3 / 40 % BC7, per-texture seeds; about a quarter of its BC7 blocks take modes 5 / 1),
    autotuned and graph-launched: every level of every texture is the reference's bytes (21.9 Mpix in all)."""
    import os
    from concurrent.futures import ThreadPoolExecutor

    import torch

    import zap_b200.synth as S
    ref = oracle_lib.best()
    sizes = S.batch_sizes(256, seed=0, lo=6, hi=9)
    fmts = S.batch_formats(256, seed=0)
    texs = [S.colour_texture(w, h, seed=10000 + k, device="cuda") for k, (w, h) in enumerate(sizes)]
    b = cuda_lib.Batch(texs, fmts, autotune=True)
    b.run()
    torch.cuda.synchronize()
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as pool:  # the oracle's calls release the GIL
        list(pool.map(lambda i: _check_item(b, i, ref, True), range(len(texs))))
    b.close()


def test_batch_replay_reads_new_inputs_and_plain_path_agrees(cuda_lib):
    import torch
    ref = oracle_lib.best()
    sizes = [(64, 64), (200, 100), (9, 13), (256, 128)]
    fmts = [4, 0, 4, 1]
    texs = [_make(7 + k, w, h, "noise") for k, (w, h) in enumerate(sizes)]
    b = cuda_lib.Batch(texs, fmts)
    b.run()
    torch.cuda.synchronize()
    first = [o.clone() for o in b.outputs]
    for k, (w, h) in enumerate(sizes):  # new content in place: the graph must see it
        b.textures[k].copy_(_make(500 + k, w, h, "opaque"))
    b.run()
    torch.cuda.synchronize()
    for i in range(len(sizes)):
        _check_item(b, i, ref, True)
    graph_out = [o.clone() for o in b.outputs]
    for o in b.outputs:
        o.fill_(0)
    b.run_plain()
    torch.cuda.synchronize()
    for g, o in zip(graph_out, b.outputs):
        assert torch.equal(g, o)
    assert not all(torch.equal(f, g) for f, g in zip(first, graph_out))
    b.close()


def test_batch_rejects_bad_items(cuda_lib):
    import torch
    lib = cuda_lib.load()
    t = torch.zeros((4, 4, 4), dtype=torch.uint8, device="cuda")
    with pytest.raises(cuda_lib.ZapTexError):
        cuda_lib.Batch([t], [6])  # ASTC is not a batch format
    assert lib.zap_tex_cuda_batch_item_bytes(4, 4, 0, 0) == 8 + 8 + 8
