"""Batched evaluation of many molecules: one persistent launch, a CUDA graph,
and an autotuner for the tile shape.

    from fastesp_b200.batch import BatchESP
    b = BatchESP(tables, points)          # tables: PairTable per molecule
    values = b.run()                      # list of (n_i,) CUDA float64 tensors

The kernels (csrc/batch.cuh) take (molecule, point block, pair split) work items
from a global queue ordered largest first; every item writes its own row of
partial sums and a reduction adds each molecule's rows in a fixed order, so the
values are deterministic and equal ``table.esp(points)`` to rounding of the
split sums.  The tile shape -- points per thread (point block of 128 or 256
points), work items per resident block (the pair-split granularity) and the
pair tile (bytes per shared-memory stage: 8, 16 or 32 KB, i.e. how many pairs
of a class one bulk copy brings in) -- is picked by timing the candidates on the
batch itself; the choice is cached per device and batch signature for the life
of the process.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from .table import PairTable, _empty_bytes, _to_dev

SHAPES = [(np_, w, st) for np_ in (1, 2) for w in (4, 8, 16, 32)
          for st in (8192, 16384, 32768)]
DEFAULT_SHAPE = (2, 4, 16384)
_TUNED: dict = {}


class _Native:
    """One fe_batch handle with its device descriptor and workspace."""

    def __init__(self, mols, shape, device):
        L = _lib.lib()
        arr = (_lib.FeBatchMol * len(mols))(*mols)
        sh = _lib.FeBatchShape(*shape)
        h = C.c_void_p()
        _lib.check(L.fe_batch_create(arr, len(mols), C.byref(sh), C.byref(h), _lib.stream_ptr()))
        self._h = h
        db, wb, ni = C.c_size_t(), C.c_size_t(), C.c_int()
        _lib.check(L.fe_batch_sizes(h, C.byref(db), C.byref(wb), C.byref(ni)))
        self.n_items = ni.value
        self.desc = _empty_bytes(db.value, device)
        self.ws = _empty_bytes(wb.value, device)
        _lib.check(L.fe_batch_upload(h, _lib.ptr(self.desc), self.desc.numel(), _lib.stream_ptr()))

    def run(self):
        _lib.check(_lib.lib().fe_batch_run(self._h, _lib.ptr(self.desc), _lib.ptr(self.ws),
                                           self.ws.numel(), _lib.stream_ptr()))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().fe_batch_destroy(h)
            except Exception:       # interpreter shutdown
                pass
            self._h = None


class BatchESP:
    """V = nuclear - electron for every (table, points) pair of a batch, FP64.

    ``shape``: (points_per_thread, waves[, stage_bytes]) or None to autotune.  ``graph``:
    capture the launch sequence in a CUDA graph and replay it on ``run``.
    """

    def __init__(self, tables, points, shape=None, graph: bool = True, repeats: int = 3):
        import torch
        if len(tables) != len(points):
            raise ValueError("one point set per table")
        if not tables:
            raise ValueError("empty batch")
        self.device = tables[0].device
        self.tables = list(tables)
        self.points = [_to_dev(p, self.device).reshape(-1, 3).contiguous() for p in points]
        self.out = [torch.empty(int(p.shape[0]), dtype=torch.float64, device=self.device)
                    for p in self.points]
        self._mols = [_lib.FeBatchMol(_lib.ptr(t._buf), _lib.ptr(p), _lib.ptr(o), int(p.shape[0]), 0)
                      for t, p, o in zip(self.tables, self.points, self.out)]
        if shape is None:
            key = (str(self.device), torch.cuda.get_device_name(self.device),
                   tuple((tuple(t.counts), int(p.shape[0])) for t, p in zip(self.tables, self.points)))
            shape = _TUNED.get(key)
            if shape is None:
                shape, self.tuning = self._autotune(repeats)
                _TUNED[key] = shape
            else:
                self.tuning = None
        else:
            self.tuning = None
        self.shape = tuple(shape) if len(shape) == 3 else tuple(shape) + (16384,)
        self._native = _Native(self._mols, self.shape, self.device)
        self._graph = None
        if graph:
            self._capture()

    @property
    def n_items(self) -> int:
        return self._native.n_items

    def _autotune(self, repeats):
        """Time every candidate shape on this batch; return the fastest."""
        import torch
        times = {}
        for shape in SHAPES:
            nat = _Native(self._mols, shape, self.device)
            nat.run()                                    # warm-up
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            best = float("inf")
            for _ in range(repeats):
                ev[0].record()
                nat.run()
                ev[1].record()
                ev[1].synchronize()
                best = min(best, ev[0].elapsed_time(ev[1]))
            times[shape] = best
            del nat
        return min(times, key=times.get), times

    def _capture(self):
        import torch
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self._native.run()                           # warm-up outside the capture
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._native.run()
        self._graph = g

    def run(self):
        """Evaluate the batch; returns the list of per-molecule outputs (device)."""
        if self._graph is not None:
            self._graph.replay()
        else:
            self._native.run()
        return self.out


def separate_launches(tables, points):
    """The same values by one plain fe_esp_fp64 call per molecule (the baseline
    the batched launch is compared with); returns (outputs, run) where ``run()``
    repeats the calls with preallocated buffers."""
    import torch
    dev = tables[0].device
    pts = [_to_dev(p, dev).reshape(-1, 3).contiguous() for p in points]
    outs = [torch.empty(int(p.shape[0]), dtype=torch.float64, device=dev) for p in pts]
    L = _lib.lib()
    ws = _empty_bytes(max(int(L.fe_eval_ws_bytes(int(p.shape[0]))) for p in pts), dev)

    def run():
        s = _lib.stream_ptr()
        for t, p, o in zip(tables, pts, outs):
            _lib.check(L.fe_esp_fp64(_lib.ptr(t._buf), _lib.ptr(p), int(p.shape[0]), _lib.ptr(o),
                                     _lib.ptr(ws), ws.numel(), s))
        return outs

    return outs, run


__all__ = ["BatchESP", "separate_launches", "SHAPES", "DEFAULT_SHAPE", "PairTable"]
