"""Serving: continuous batching of solve requests of several grids over libdtb.so.

``Server(budget_bytes)`` owns the library's serving thread. ``add_grid(BatchedEuler)`` registers
a batched context (its device memory counts against the HBM budget); ``submit(grid, f0, dt,
n_steps)`` queues a solve and returns its id; ``wait(id)`` returns the final f and the
request's timings (seconds since ``start``). Requests of one grid share its operators and are
admitted into free slots as earlier requests finish; grids step concurrently on the device.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional

import numpy as np

from . import _lib
from ._lib import check, dptr
from .batch import BatchedEuler


class Server:
    def __init__(self, hbm_budget_bytes: int = 0, max_chunk_steps: int = 0, chunk_ms: float = 0.0):
        self.L = _lib.load()
        opts = _lib.ServeOpts(hbm_budget_bytes=int(hbm_budget_bytes), max_chunk_steps=int(max_chunk_steps),
                              flags=0, chunk_ms=float(chunk_ms))
        srv = ctypes.c_void_p()
        check(self.L.dtb_serve_create(ctypes.byref(opts), ctypes.byref(srv)))
        self.srv = srv
        self.grids: List[BatchedEuler] = []

    def add_grid(self, batched: BatchedEuler) -> int:
        gid = ctypes.c_int32()
        check(self.L.dtb_serve_add_grid(self.srv, batched.ctx, ctypes.byref(gid)))
        self.grids.append(batched)
        return gid.value

    def start(self) -> None:
        check(self.L.dtb_serve_start(self.srv))

    def submit(self, grid: int, f0, dt: float, n_steps: int) -> int:
        b = self.grids[grid]
        f = np.ascontiguousarray(f0, dtype=np.float64)
        rid = ctypes.c_int64()
        check(self.L.dtb_serve_submit(self.srv, int(grid), dptr(f), float(dt) / b.dt0, int(n_steps),
                                      ctypes.byref(rid)))
        return rid.value

    def wait(self, request_id: int, timeout_s: float = 0.0, with_f: bool = True):
        st = _lib.RequestStats()
        grid_n = None
        out = None
        if with_f:
            # the request's grid is known only after it finishes; size the buffer for the largest grid
            grid_n = max(g.n for g in self.grids)
            out = np.empty(grid_n)
        check(self.L.dtb_serve_wait(self.srv, int(request_id), float(timeout_s), dptr(out) if out is not None else None,
                                    ctypes.byref(st)))
        info = {"t_submit": st.t_submit, "t_admit": st.t_admit, "t_done": st.t_done, "steps": st.steps,
                "cr_max": st.cr_max, "finite": bool(st.finite), "grid": st.grid}
        if out is not None:
            out = out[:self.grids[st.grid].n].copy()
        return out, info

    def cancel(self, request_id: int) -> None:
        """Cancels a queued or running request; wait() then raises DtbError with DTB_ESTATE."""
        check(self.L.dtb_serve_cancel(self.srv, int(request_id)))

    def stats(self) -> dict:
        st = _lib.ServeStats()
        check(self.L.dtb_serve_get_stats(self.srv, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in _lib.ServeStats._fields_}

    def close(self) -> None:
        if getattr(self, "srv", None):
            self.L.dtb_serve_destroy(self.srv)
            self.srv = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
