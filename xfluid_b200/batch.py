"""Batched projection of many independent scenes (xfp_project_batch_*).

``BatchProjector.project(scenes)`` projects a list of scenes of different
sizes in one library call: every scene is solved exactly as a single
``VariationalPressureSolver.project`` would solve it, but the MIC(0) sweeps of
all scenes share one persistent launch and the PCG iteration is replayed as a
CUDA graph.  xFluid itself projects one grid per call
(FluidSimulator.cpp:501-509); this is an extension beside that drop-in.

Across GPUs the scenes shard with no collective on the data path:
``shard_scenes`` bin-packs them by cell count (longest first onto the least
loaded rank) and ``project_sharded`` runs each rank's share, gathering only
the per-scene stats to every rank.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import Context, XfpScene, XfpStats


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _ptr(a):
    if a is None:
        return None
    if _is_torch(a):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data


class BatchProjector:
    """Owns one context; projects lists of scenes.

    Each scene is a mapping (or object) with ``mat`` (nk,nj,ni) uint8, ``u``,
    ``v``, ``w`` face arrays (updated in place), optional ``wu/wv/ww`` and
    optional ``pressure`` (nk,nj,ni) output.  All arrays of one call are host
    numpy arrays or all CUDA torch tensors, all float32 or all float64.
    ``tile_k=0`` lets the library time both sweep tile heights per batch shape.
    """

    def __init__(self, precision: str = "mixed", tol: float = 1e-6, max_iter: int = 200, tile_k: int = 0,
                 device: int = 0, check_every: int = 8, stream=None):
        o = _lib.default_options()
        o.precision = _lib.PREC[precision]
        o.tol, o.max_iter, o.tile_k, o.device, o.check_every = tol, max_iter, tile_k, device, check_every
        self._stream_given = stream is not None
        if stream is not None:
            o.stream = C.c_void_p(stream)
        self._ctx = Context(o)
        self.stats: list[dict] = []

    def close(self) -> None:
        self._ctx.close()

    def project(self, scenes: Sequence) -> bool:
        """Projects every scene in place; True when all converged."""
        get = (lambda s, k: s.get(k)) if scenes and isinstance(scenes[0], dict) else (lambda s, k: getattr(s, k, None))
        n = len(scenes)
        arr = (XfpScene * n)()
        kinds, dtypes = set(), set()
        for q, sc in enumerate(scenes):
            mat, u = get(sc, "mat"), get(sc, "u")
            nk, nj, ni = mat.shape
            kinds.add(_is_torch(u) and u.is_cuda)
            dtypes.add(str(u.dtype).replace("torch.", ""))
            a = arr[q]
            a.ni, a.nj, a.nk = ni, nj, nk
            a.material = _ptr(mat)
            a.u, a.v, a.w = _ptr(u), _ptr(get(sc, "v")), _ptr(get(sc, "w"))
            a.wu, a.wv, a.ww = (_ptr(get(sc, k)) for k in ("wu", "wv", "ww"))
            a.pressure = _ptr(get(sc, "pressure"))
        if len(kinds) != 1 or len(dtypes) != 1:
            raise ValueError("all arrays of a batch must share placement (host/device) and dtype")
        o = self._ctx.opts
        dev = 1 if kinds.pop() else 0
        if o.device_pointers != dev:
            o.device_pointers = dev
            self._ctx.set_options(o)
        if dev and not self._stream_given:
            # the context's own stream is not ordered after torch's: finish
            # the torch work that produced the tensors first
            _lib.sync_torch(o.device)
        st = (XfpStats * n)()
        fn = self._ctx.lib.xfp_project_batch_f64 if dtypes.pop() == "float64" else self._ctx.lib.xfp_project_batch_f32
        rc = self._ctx.check(fn(self._ctx.ptr, n, arr, st))
        self.stats = [st[q].as_dict() for q in range(n)]
        return rc == _lib.XFP_OK


def shard_scenes(cells: Sequence[int], world: int) -> list[list[int]]:
    """Longest-processing-time bin packing: scene indices per rank, biggest
    scene first onto the rank with the fewest cells so far (ties: lower rank).
    Every rank's list keeps the scenes' original order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for q in sorted(range(len(cells)), key=lambda q: (-cells[q], q)):
        r = min(range(world), key=lambda r: (load[r], r))
        out[r].append(q)
        load[r] += cells[q]
    return [sorted(x) for x in out]


def project_sharded(scenes: Sequence, projector: BatchProjector | None, rank: int, world: int, group=None,
                    run=None) -> list[dict]:
    """Projects this rank's share of ``scenes`` and returns every scene's stats
    (gathered from all ranks with torch.distributed.all_gather_object; no data
    crosses ranks).  ``run`` replaces the projector call (for host-only tests)."""
    import torch.distributed as dist

    get = (lambda s, k: s.get(k)) if scenes and isinstance(scenes[0], dict) else (lambda s, k: getattr(s, k, None))
    cells = [int(np.prod(get(s, "mat").shape)) for s in scenes]
    mine = shard_scenes(cells, world)[rank]
    if run is not None:
        local = run([scenes[q] for q in mine])
    elif mine:
        projector.project([scenes[q] for q in mine])
        local = projector.stats
    else:
        local = []
    gathered: list = [None] * world
    if world > 1:
        dist.all_gather_object(gathered, list(zip(mine, local)), group=group)
    else:
        gathered = [list(zip(mine, local))]
    stats: list = [None] * len(scenes)
    for part in gathered:
        for q, s in part:
            stats[q] = s
    return stats
