"""Host-side mirror of the reference's HashGrid (src/imbatracer/rangesearch/rangesearch.h).

    grid = HashGrid(device=0)
    grid.build(positions, radius)            # HashGrid::build(begin, end, radius), :25-75
    ids, counts = grid.query(points, k)      # HashGrid::query(pos, out, k), :77-129, batched

Positions and query points are torch CUDA tensors (N,3) float32 (or (N, stride) with the
xyz first). Results are device tensors: ids (Q,k) int32 padded with -1, counts (Q,) int32.
Everything runs in libimbart on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N


class HashGrid:
    def __init__(self, device: int = 0):
        self.lib = N.load()
        self.handle = self.lib.imbart_hashgrid_create(device)
        if not self.handle:
            raise N.ImbartError("imbart_hashgrid_create: " + N.last_error()[1])
        self.device = device

    def build(self, positions, radius: float, cell_factor: float = 2.0, table_size: int = 0, stream=None):
        assert positions.is_cuda and positions.dtype.is_floating_point and positions.is_contiguous()
        st = None if stream is None else stream.cuda_stream
        n, stride = positions.shape[0], positions.shape[1]
        N.check(self.lib.imbart_hashgrid_build(self.handle, N.ptr(positions), stride, n, float(radius),
                                               float(cell_factor), int(table_size), st), "imbart_hashgrid_build")

    def query(self, points, k: int, with_d2: bool = False, stream=None):
        import torch
        assert points.is_cuda and points.is_contiguous() and points.shape[1] == 3
        nq = points.shape[0]
        ids = torch.empty((nq, k), dtype=torch.int32, device=points.device)
        cnt = torch.empty(nq, dtype=torch.int32, device=points.device)
        d2 = torch.empty((nq, k), dtype=torch.float32, device=points.device) if with_d2 else None
        st = None if stream is None else stream.cuda_stream
        N.check(self.lib.imbart_hashgrid_query(self.handle, N.ptr(points), nq, k, N.ptr(ids), N.ptr(cnt),
                                               N.ptr(d2), st), "imbart_hashgrid_query")
        return (ids, cnt, d2) if with_d2 else (ids, cnt)

    def params(self):
        p = np.zeros(10, np.float32)
        n = C.c_int(0)
        t = C.c_int(0)
        N.check(self.lib.imbart_hashgrid_get_params(self.handle, N.ptr(p), C.byref(n), C.byref(t)), "params")
        return {"lo": p[:3].copy(), "hi": p[3:6].copy(), "radius": float(p[6]), "radius_sqr": float(p[7]),
                "cell_size": float(p[8]), "inv_cell_size": float(p[9]), "n": n.value, "table_size": t.value}

    def close(self):
        if self.handle:
            self.lib.imbart_hashgrid_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
