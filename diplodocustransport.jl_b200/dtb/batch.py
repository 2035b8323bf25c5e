"""Batched independent solves on one grid (mixed precision) over libdtb.so.

``BatchedEuler(PhaseSpace, Injection, BinM, EmiM, FluxM, capacity)`` uploads the shared
operators once (as ``ForwardEulerStruct`` does for a single solve, SteppingStructs.jl:33-100)
and holds ``capacity`` slots. Each admitted slot runs the explicit Euler step of
SteppingMethods.jl:12-107 with its own initial f, dt and step count; ``run(k)`` advances every
slot with steps left by k batched steps. A slot may hold several space cells (PhaseSpace.n_space):
every (cell, slot) pair is then a column of the gain GEMM, with the cell's Vol and BinM.Domain
applied per cell, and the flux coupling the cells. The gain contraction of all slots is a tensor-core
GEMM with G in BF16 hi + lo (three MMAs, FP32 accumulation) and f is updated with an FP64
compensated sum.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import check, dptr
from .stepping import _upload_csc, _upload_gain
from .structs import BinaryMatrices, EmissionMatrices, FluxMatrices, PhaseSpace


class BatchedEuler:
    def __init__(self, PhaseSpace: PhaseSpace, Injection, BinM: BinaryMatrices, EmiM: EmissionMatrices,
                 FluxM: FluxMatrices, capacity: int, *, device: int = 0, stream: Optional[int] = None,
                 graph_steps: int = 16, autotune: bool = True):
        self.L = _lib.load()
        self.PhaseSpace = PhaseSpace
        self.capacity = int(capacity)
        self.dt0 = float(PhaseSpace.dt0)
        self.n = PhaseSpace.n_state
        dims = _lib.Dims()
        sizes = PhaseSpace.species_sizes
        dims.n_species = len(sizes)
        dims.n_space = PhaseSpace.n_space
        for i, s in enumerate(sizes):
            dims.species_size[i] = s
        opts = _lib.Opts(precision=_lib.DTB_MIXED, device=device, stream=stream, index_base=0,
                         graph_steps=graph_steps, dt0=self.dt0, batch=self.capacity,
                         flags=0 if autotune else _lib.DTB_FLAG_NO_AUTOTUNE)
        ctx = ctypes.c_void_p()
        check(self.L.dtb_create(ctypes.byref(dims), ctypes.byref(opts), ctypes.byref(ctx)))
        self.ctx = ctx
        try:
            L = self.L
            _upload_csc(L, ctx, FluxM.X_Flux)
            _upload_csc(L, ctx, FluxM.P_Flux)
            if BinM.M_Bin is not None and sp.issparse(BinM.M_Bin):
                M = sp.csc_matrix(BinM.M_Bin)
                ip = [np.ascontiguousarray(x, dtype=np.int64) for x in (M.indptr, M.indices)]
                nz = np.ascontiguousarray(M.data, dtype=np.float64)
                check(L.dtb_upload_mbin_csc(ctx, PhaseSpace.n_momentum, ip[0].ctypes.data_as(_lib._ip),
                                            ip[1].ctypes.data_as(_lib._ip), dptr(nz)))
            elif BinM.M_Bin is not None:
                M = np.asfortranarray(BinM.M_Bin, dtype=np.float64)
                check(L.dtb_upload_mbin_ref(ctx, M.ctypes.data_as(_lib._dp), PhaseSpace.n_momentum))
            for g in BinM.gains:
                _upload_gain(L, ctx, g)
            for l in BinM.losses:
                A = np.ascontiguousarray(l.L, dtype=np.float64)
                check(L.dtb_add_loss_block(ctx, l.sp, l.other_sp, dptr(A)))
            if BinM.Domain is not None:
                D = np.ascontiguousarray(BinM.Domain, dtype=np.int64)
                check(L.dtb_set_bin_domain(ctx, D.ctypes.data_as(_lib._ip), len(D)))
            if EmiM.M_Emi is not None:
                M = np.asfortranarray(EmiM.M_Emi, dtype=np.float64)
                check(L.dtb_upload_emi_ref(ctx, M.ctypes.data_as(_lib._dp), self.n))
            for b in EmiM.blocks:
                E = np.ascontiguousarray(b.E, dtype=np.float64)
                check(L.dtb_add_emi_block(ctx, b.row0, E.shape[0], b.col0, E.shape[1], dptr(E)))
            Ap = np.ascontiguousarray(FluxM.Ap_Flux, dtype=np.float64)
            Vol = np.ascontiguousarray(FluxM.Vol, dtype=np.float64)
            inj = np.ascontiguousarray(Injection, dtype=np.float64)
            zeros = np.zeros(self.n)
            check(L.dtb_upload_vectors(ctx, dptr(Ap), dptr(Vol), dptr(zeros), dptr(inj)))
            check(L.dtb_commit(ctx))
        except Exception:
            self.close()
            raise

    def admit(self, slot: int, f0, dt: float, n_steps: int) -> None:
        """Start a solve in `slot` with initial state f0, step dt (dt/dt0 is applied) and n_steps steps."""
        f = np.ascontiguousarray(f0, dtype=np.float64)
        check(self.L.dtb_batch_admit(self.ctx, int(slot), dptr(f), float(dt) / self.dt0, int(n_steps)))

    def prepare(self) -> None:
        """Captures and uploads the batched step graphs now (dtb_prepare), so no later run pays for it."""
        check(self.L.dtb_prepare(self.ctx))

    def run(self, nsteps: int) -> None:
        check(self.L.dtb_batch_run(self.ctx, int(nsteps)))

    def get_f(self, slot: int) -> np.ndarray:
        out = np.empty(self.n)
        check(self.L.dtb_batch_get_f(self.ctx, int(slot), dptr(out)))
        return out

    def set_f_all(self, F) -> None:
        """Every slot's f from a (capacity, n) array."""
        A = np.ascontiguousarray(F, dtype=np.float64)
        check(self.L.dtb_batch_set_f_all(self.ctx, dptr(A)))

    def get_f_all(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Every slot's f as a (capacity, n) array."""
        if out is None:
            out = np.empty((self.capacity, self.n))
        check(self.L.dtb_batch_get_f_all(self.ctx, dptr(out)))
        return out

    def run_io(self, F_in, nsteps: int, out: Optional[np.ndarray] = None) -> Optional[np.ndarray]:
        """Every slot's f from F_in (None: keep the device state), nsteps batched steps, every
        slot's f into `out` (allocated when None), with one wait for the whole round trip."""
        A = None if F_in is None else np.ascontiguousarray(F_in, dtype=np.float64)
        if out is None:
            out = np.empty((self.capacity, self.n))
        if not hasattr(self, "_io_ptrs"):
            self._io_ptrs = (_lib.LastPtr(), _lib.LastPtr())
        pin, pout = self._io_ptrs
        check(self.L.dtb_batch_run_io(self.ctx, pin(A), int(nsteps), pout(out)))
        return out

    def moments(self, weights) -> tuple:
        """FP64 number and energy per (slot, species) on the device, or per (slot, cell, species)
        when the slots hold several space cells; weights: one per momentum state."""
        w = np.ascontiguousarray(weights, dtype=np.float64)
        ns = len(self.PhaseSpace.species_sizes)
        nsp = self.PhaseSpace.n_space
        num = np.zeros((self.capacity, nsp, ns))
        en = np.zeros_like(num)
        check(self.L.dtb_batch_moments(self.ctx, dptr(w), dptr(num), dptr(en)))
        if nsp == 1:
            return num[:, 0, :], en[:, 0, :]
        return num, en

    def info(self, slot: int) -> dict:
        done, left = ctypes.c_int64(), ctypes.c_int64()
        cr = ctypes.c_double()
        fin = ctypes.c_int32()
        check(self.L.dtb_batch_slot_info(self.ctx, int(slot), ctypes.byref(done), ctypes.byref(left),
                                         ctypes.byref(cr), ctypes.byref(fin)))
        return {"steps_done": done.value, "steps_left": left.value, "cr_max": cr.value, "finite": bool(fin.value)}

    def release(self, slot: int) -> None:
        check(self.L.dtb_batch_release(self.ctx, int(slot)))

    @property
    def step(self) -> int:
        cap, st = ctypes.c_int32(), ctypes.c_int64()
        check(self.L.dtb_batch_capacity(self.ctx, ctypes.byref(cap), ctypes.byref(st)))
        return st.value

    def set_profiling(self, on: bool) -> None:
        check(self.L.dtb_batch_set_profiling(self.ctx, 1 if on else 0))

    def gemm_plan(self, group: int = 0) -> Optional[dict]:
        """The gain-GEMM plan of one gain group (None past the last group): SM pairs or not,
        column tile width, K splits, measured microseconds of one GEMM (0 if not timed)."""
        pair, bn, ns = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        us = ctypes.c_double()
        rc = self.L.dtb_batch_gemm_plan(self.ctx, group, ctypes.byref(pair), ctypes.byref(bn), ctypes.byref(ns),
                                        ctypes.byref(us))
        if rc == _lib.DTB_ENOTFOUND:
            return None
        check(rc)
        return {"pair": bool(pair.value), "bn": bn.value, "n_splits": ns.value, "tuned_us": us.value}

    def gemm_stats(self) -> dict:
        ms, fl, by = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        lps = ctypes.c_int32()
        check(self.L.dtb_batch_gemm_stats(self.ctx, ctypes.byref(ms), ctypes.byref(fl), ctypes.byref(by),
                                          ctypes.byref(lps)))
        return {"avg_ms": ms.value, "flops_per_step": fl.value, "bytes_per_step": by.value,
                "launches_per_step": lps.value}

    def device_bytes(self) -> int:
        v = ctypes.c_int64()
        check(self.L.dtb_device_bytes(self.ctx, ctypes.byref(v)))
        return v.value

    def close(self) -> None:
        if getattr(self, "ctx", None):
            self.L.dtb_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_tune_cache(path: Optional[str]) -> None:
    """Seeds the process-wide gain-GEMM plans from a cache file and records new measurements in
    it; None forgets the plans chosen so far."""
    check(_lib.load().dtb_set_tune_cache(None if path is None else str(path).encode()))
