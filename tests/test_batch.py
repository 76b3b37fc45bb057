"""Batched projection (xfp_project_batch_*): each scene of a batch must come out
exactly as a single-scene projection of it; across ranks the scenes shard by
cell count with only the stats gathered."""
import os

import numpy as np
import pytest

from xfluid_b200 import scenes
from xfluid_b200.batch import BatchProjector, project_sharded, shard_scenes


# ------------------------------------------------------------------ host logic
def test_shard_scenes_is_lpt_and_balanced():
    cells = [100, 90, 80, 10, 10, 10, 5]
    parts = shard_scenes(cells, 3)
    assert sorted(q for p in parts for q in p) == list(range(len(cells)))
    loads = [sum(cells[q] for q in p) for p in parts]
    # LPT: 100 -> r0, 90 -> r1, 80 -> r2, then the small ones onto the lightest
    assert parts[0][0] == 0 and parts[1][0] == 1 and parts[2][0] == 2
    assert max(loads) - min(loads) <= max(cells[3:])
    assert shard_scenes(cells, 1) == [list(range(len(cells)))]
    assert shard_scenes([], 2) == [[], []]
    with pytest.raises(ValueError):
        shard_scenes(cells, 0)


def _gloo_worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = [{"mat": np.zeros(d, np.uint8)} for d in [(4, 4, 4), (8, 8, 8), (2, 2, 2), (6, 6, 6), (3, 3, 3)]]
        run = lambda mine: [{"rank": rank, "cells": int(np.prod(s["mat"].shape))} for s in mine]
        stats = project_sharded(sc, None, rank, world, run=run)
        out.put((rank, stats))
    finally:
        dist.destroy_process_group()


def test_sharded_projection_gathers_every_scene_on_every_rank():
    import multiprocessing as mp
    import socket
    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    owners = shard_scenes([64, 512, 8, 216, 27], 2)
    for rank in (0, 1):
        st = res[rank]
        assert [s["cells"] for s in st] == [64, 512, 8, 216, 27]
        for r, mine in enumerate(owners):
            for i in mine:
                assert st[i]["rank"] == r
    assert res[0] == res[1]


# ------------------------------------------------------------------ GPU
def _single(sc, precision, dtype, tile_k):
    from gpu_util import make_ctx, project, set_tol
    ctx = make_ctx(precision, tile_k=tile_k)
    try:
        set_tol(ctx, 1e-6, 400)
        rc, p, u, v, w, st = project(ctx, sc, dtype=dtype)
    finally:
        ctx.close()
    return rc, p, u, v, w, st


def _batch_inputs(scs, dtype):
    items = []
    for sc in scs:
        items.append({"mat": np.ascontiguousarray(sc.mat, np.uint8),
                      "u": np.array(sc.u, dtype), "v": np.array(sc.v, dtype), "w": np.array(sc.w, dtype),
                      "wu": None if sc.wu is None else np.ascontiguousarray(sc.wu, dtype),
                      "wv": None if sc.wv is None else np.ascontiguousarray(sc.wv, dtype),
                      "ww": None if sc.ww is None else np.ascontiguousarray(sc.ww, dtype),
                      "pressure": np.zeros((sc.nk, sc.nj, sc.ni), dtype)})
    return items


def _uneven(dtype):
    scs = scenes.batch_scenes(count=5, seed=11, lo=12, hi=44, dtype=dtype)
    scs.append(scenes.dam_break(20, seed=3, noise=0.3, dims=(20, 17, 23)).astype(dtype))
    return scs


@pytest.mark.gpu
@pytest.mark.parametrize("precision,dtype", [("f64", np.float64), ("f32", np.float32), ("mixed", np.float32)])
def test_batch_equals_single_scene_projections(precision, dtype):
    scs = _uneven(dtype)
    items = _batch_inputs(scs, dtype)
    bp = BatchProjector(precision, tol=1e-6, max_iter=400, tile_k=8)
    try:
        assert bp.project(items)
        stats = bp.stats
    finally:
        bp.close()
    for sc, it, st in zip(scs, items, stats):
        rc, p, u, v, w, s1 = _single(sc, precision, dtype, 8)
        assert rc == 0 and st["status"] == 0
        assert st["iterations"] == s1["iterations"], sc.name
        assert st["tile_k"] == 8
        # same kernels, same per-scene reduction order: identical bits
        assert np.array_equal(it["pressure"], p), sc.name
        assert np.array_equal(it["u"], u) and np.array_equal(it["v"], v) and np.array_equal(it["w"], w), sc.name


@pytest.mark.gpu
def test_batch_autotuned_with_empty_and_thin_scenes_vs_oracle():
    import oracle
    O = oracle.Oracle()
    scs = [scenes.blob_scene(dims=(30, 26, 34), seed=2, dtype=np.float64),
           scenes.Scene(9, 7, 5, np.zeros((5, 7, 9), np.uint8), np.zeros((5, 7, 10)), np.zeros((5, 8, 9)),
                        np.zeros((6, 7, 9)), name="all_air"),
           scenes.blob_scene(dims=(40, 3, 37), seed=4, fractional=False, dtype=np.float64),
           scenes.dam_break(24, seed=1, noise=0.2)]
    items = _batch_inputs(scs, np.float64)
    bp = BatchProjector("f64", tol=1e-8, max_iter=1000, tile_k=0)
    try:
        assert bp.project(items)
        first = bp.stats
        items2 = _batch_inputs(scs, np.float64)
        assert bp.project(items2)            # second call: cached tile height
        second = bp.stats
    finally:
        bp.close()
    assert first[0]["tile_k"] in (8, 16) and second[0]["tile_k"] == first[0]["tile_k"]
    assert first[1]["rows"] == 0 and first[1]["iterations"] == 0
    for sc, it, it2 in zip(scs, items, items2):
        ref = O.project(sc, tol=1e-8, maxit=1000)
        assert ref["ok"]
        d = np.linalg.norm(it["pressure"] - ref["p"]) / max(np.linalg.norm(ref["p"]), 1e-300)
        assert d <= 1e-5, (sc.name, d)
        assert np.array_equal(it["pressure"], it2["pressure"])


@pytest.mark.gpu
def test_batch_device_pointers_match_host():
    import torch
    scs = _uneven(np.float32)[:3]
    host = _batch_inputs(scs, np.float32)
    dev = [{k: (None if a is None else torch.from_numpy(a.copy()).cuda()) for k, a in it.items()} for it in host]
    bp = BatchProjector("mixed", tol=1e-6, max_iter=400, tile_k=8)
    try:
        assert bp.project(host)
        assert bp.project(dev)
    finally:
        bp.close()
    for h, d in zip(host, dev):
        for k in ("pressure", "u", "v", "w"):
            assert np.array_equal(h[k], d[k].cpu().numpy()), k
