"""Python entry to the oracle (test infrastructure only).

Wraps oracle/liborc.so, the plain-C FP64 restatement of DiplodocusTransport.jl's explicit
Euler step, and restates the host-side Solve loop (src/Solver.jl:1-64 together with the
dt truncation of src/SteppingMethods.jl:18-27) in Python floats, which are IEEE doubles
like Julia's Float64, so the step schedule is reproduced exactly.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py use this module,
and only to check results. Parity is pinned against hand-derived known-answer vectors and a
literal transliteration of the Julia lines (tests/golden/); it is unpinned against a run of
the reference itself, which needs Julia.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import List, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

THR_F64 = float(np.float32(1e-10))  # Float64(1f-10): SteppingMethods.jl:99 compares with a Float32 literal

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int64)
_bp = ctypes.POINTER(ctypes.c_uint8)


class GainT(ctypes.Structure):
    _fields_ = [("out_sp", ctypes.c_int32), ("in1_sp", ctypes.c_int32), ("in2_sp", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("G", _dp)]


class LossT(ctypes.Structure):
    _fields_ = [("row_sp", ctypes.c_int32), ("col_sp", ctypes.c_int32), ("L", _dp)]


class EmiT(ctypes.Structure):
    _fields_ = [("row0", ctypes.c_int64), ("nrows", ctypes.c_int64), ("col0", ctypes.c_int64),
                ("ncols", ctypes.c_int64), ("E", _dp)]


def build() -> str:
    """Compile oracle/liborc.so with make (system gcc + OpenMP when available)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liborc.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liborc.so")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(os.path.join(_HERE, "orc.c")):
            build()
        L = ctypes.CDLL(path)
        L.orc_step_ref.restype = ctypes.c_int
        L.orc_step_ref.argtypes = [ctypes.c_int64, ctypes.c_int64, _dp, _dp, _ip, _ip, _dp, ctypes.c_int,
                                   _dp, _dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                   _dp, _dp, _dp, _bp]
        L.orc_step_blocked.restype = ctypes.c_int
        L.orc_step_blocked.argtypes = [ctypes.c_int32, _ip, ctypes.c_int64,
                                       ctypes.c_int, ctypes.POINTER(GainT), ctypes.c_int,
                                       ctypes.POINTER(LossT), ctypes.c_int, ctypes.POINTER(EmiT),
                                       _ip, _ip, _dp, ctypes.c_int, _dp, _dp, _dp, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_int, _dp, _dp, _dp, _bp]
        L.orc_step_symplectic_ref.restype = ctypes.c_int
        L.orc_step_symplectic_ref.argtypes = [ctypes.c_int64, ctypes.c_int64, _dp, _dp,
                                              _ip, _ip, _dp, _ip, _ip, _dp, ctypes.c_int,
                                              _dp, _dp, _dp, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_double, ctypes.c_int, _dp, _dp, _bp]
        L.orc_gain_rows.restype = None
        L.orc_gain_rows.argtypes = [_dp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                    _dp, _dp, _dp]
        L.orc_moments.restype = None
        L.orc_moments.argtypes = [ctypes.c_int32, _ip, _dp, _dp, _dp, _dp]
        L.orc_clamp.restype = ctypes.c_double
        L.orc_clamp.argtypes = [ctypes.c_double, ctypes.c_double]
        L.orc_num_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


def _d(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def _i(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(_ip)


def _csc_arrays(F):
    if F is None or F.nnz == 0:
        n = F.shape[0] if F is not None else 0
        return (np.zeros(n + 1, dtype=np.int64), np.zeros(1, dtype=np.int64), np.zeros(1))
    F = F.tocsc()
    F.sort_indices()
    return (np.ascontiguousarray(F.indptr, dtype=np.int64), np.ascontiguousarray(F.indices, dtype=np.int64),
            np.ascontiguousarray(F.data, dtype=np.float64))


def domain_mask(domain, n_space: int):
    """Bin_Domain (a list of 0-based off_space indices, or None for `nothing`) as one byte per
    cell, or None."""
    if domain is None:
        return None
    m = np.zeros(n_space, dtype=np.uint8)
    for k in domain:
        if 0 <= int(k) < n_space:
            m[int(k)] = 1
    return m


def _b(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(_bp)


class RefOperands:
    """Reference-layout operands: M_Bin (n_mom^2 x n_mom, F-order), M_Emi (n x n, F-order), CSC F;
    ``domain`` is BinM.Domain (0-based off_space indices, or None)."""

    def __init__(self, n_mom: int, n_space: int, M_Bin, M_Emi, F, invAp, Vol, inj, domain=None):
        self.n_mom, self.n_space = n_mom, n_space
        self.dom = domain_mask(domain, n_space)
        if M_Bin is not None and hasattr(M_Bin, "toarray"):  # a scipy sparse M_Bin (Bin_sparse)
            M_Bin = M_Bin.toarray()
        self.M_Bin = None if M_Bin is None else np.asfortranarray(M_Bin, dtype=np.float64)
        self.M_Emi = None if M_Emi is None else np.asfortranarray(M_Emi, dtype=np.float64)
        self.colptr, self.rowval, self.nzval = _csc_arrays(F)
        self.invAp = np.ascontiguousarray(invAp, dtype=np.float64)
        self.Vol = np.ascontiguousarray(Vol, dtype=np.float64)
        self.inj = np.ascontiguousarray(inj, dtype=np.float64)

    def step(self, f: np.ndarray, dt_scale: float, verbose: int = 1, thr: float = THR_F64):
        f = np.array(f, dtype=np.float64, copy=True)
        diag = np.zeros(8)
        df = np.zeros_like(f)
        rc = lib().orc_step_ref(self.n_mom, self.n_space, _d(self.M_Bin), _d(self.M_Emi),
                                _i(self.colptr), _i(self.rowval), _d(self.nzval), 0,
                                _d(self.invAp), _d(self.Vol), _d(self.inj), float(dt_scale), float(thr),
                                int(verbose), _d(f), _d(diag), _d(df), _b(self.dom))
        assert rc == 0
        return f, diag, df


class BlockedOperands:
    """Blocked operands (gain/loss/emission blocks); G, L, E are cast to FP64 once."""

    def __init__(self, sp_size: Sequence[int], n_space: int, gains, losses, emis, F, invAp, Vol, inj,
                 domain=None):
        self.sp_size = np.ascontiguousarray(sp_size, dtype=np.int64)
        self.n_space = n_space
        self.dom = domain_mask(domain, n_space)
        self._keep = []
        self.gains = (GainT * max(1, len(gains)))()
        for i, g in enumerate(gains):
            G = np.ascontiguousarray(np.asarray(g.G), dtype=np.float64)
            self._keep.append(G)
            self.gains[i] = GainT(g.out_sp, g.in1_sp, g.in2_sp, 0, _d(G))
        self.n_gain = len(gains)
        self.losses = (LossT * max(1, len(losses)))()
        for i, l in enumerate(losses):
            L = np.ascontiguousarray(np.asarray(l.L), dtype=np.float64)
            self._keep.append(L)
            self.losses[i] = LossT(l.sp, l.other_sp, _d(L))
        self.n_loss = len(losses)
        self.emis = (EmiT * max(1, len(emis)))()
        for i, e in enumerate(emis):
            E = np.ascontiguousarray(np.asarray(e.E), dtype=np.float64)
            self._keep.append(E)
            self.emis[i] = EmiT(e.row0, E.shape[0], e.col0, E.shape[1], _d(E))
        self.n_emi = len(emis)
        self.colptr, self.rowval, self.nzval = _csc_arrays(F)
        self.invAp = np.ascontiguousarray(invAp, dtype=np.float64)
        self.Vol = np.ascontiguousarray(Vol, dtype=np.float64)
        self.inj = np.ascontiguousarray(inj, dtype=np.float64)

    def step(self, f: np.ndarray, dt_scale: float, verbose: int = 1, thr: float = THR_F64):
        f = np.array(f, dtype=np.float64, copy=True)
        diag = np.zeros(8)
        df = np.zeros_like(f)
        rc = lib().orc_step_blocked(len(self.sp_size), _i(self.sp_size), self.n_space,
                                    self.n_gain, self.gains, self.n_loss, self.losses,
                                    self.n_emi, self.emis, _i(self.colptr), _i(self.rowval),
                                    _d(self.nzval), 0, _d(self.invAp), _d(self.Vol), _d(self.inj),
                                    float(dt_scale), float(thr), int(verbose), _d(f), _d(diag), _d(df),
                                    _b(self.dom))
        assert rc == 0
        return f, diag, df


def blocked_from_workload(w) -> BlockedOperands:
    return BlockedOperands(w.ps.species_sizes, w.ps.n_space, w.binm.gains, w.binm.losses,
                           w.emim.blocks, w.fluxm.F_Flux, 1.0 / np.asarray(w.fluxm.Ap_Flux),
                           w.fluxm.Vol, w.inj, domain=getattr(w.binm, "Domain", None))


def ref_from_workload(w) -> RefOperands:
    from dtb.structs import blocked_to_ref, emission_to_dense
    M_Bin = w.binm.M_Bin if w.binm.M_Bin is not None else (
        blocked_to_ref(w.ps, w.binm) if w.binm.has_interactions else None)
    return RefOperands(w.ps.n_momentum, w.ps.n_space, M_Bin, emission_to_dense(w.ps, w.emim),
                       w.fluxm.F_Flux, 1.0 / np.asarray(w.fluxm.Ap_Flux), w.fluxm.Vol, w.inj,
                       domain=getattr(w.binm, "Domain", None))


def gain_rows(G: np.ndarray, r0: int, r1: int, f1: np.ndarray, f2: np.ndarray) -> np.ndarray:
    """sum_b f1[b] sum_c G[a,b,c] f2[c] for a in [r0, r1) (FP64, OpenMP over rows)."""
    G = np.ascontiguousarray(G, dtype=np.float64)
    no, n1, n2 = G.shape
    out = np.zeros(r1 - r0)
    f1 = np.ascontiguousarray(f1, dtype=np.float64)
    f2 = np.ascontiguousarray(f2, dtype=np.float64)
    lib().orc_gain_rows(_d(G), r0, r1, n1, n2, _d(f1), _d(f2), _d(out))
    return out


def clamp(f: float, thr: float = THR_F64) -> float:
    return lib().orc_clamp(float(f), float(thr))


def num_threads() -> int:
    return int(lib().orc_num_threads())


def solve_schedule(dt_initial: float, t_save: Sequence[float], dt0: float, max_steps: int = 10_000_000
                   ) -> List[Tuple[int, List[float], List[float]]]:
    """Step schedule of Solve (Solver.jl:25-37) with the functor's truncation (SteppingMethods.jl:18-27).

    Returns, per save interval i (2..n_save), the list of dt_scale values and the list of
    (dt) values of the steps taken, in order. ``dt0`` is the step's dt0 in its own
    precision (Float32(dt0) for a Float32 state, SteppingStructs.jl:44). Note the returned
    dt is assigned back (Solver.jl:35), so after a truncated step later steps keep the
    shorter dt.
    """
    out = []
    dt = float(dt_initial)
    for i in range(1, len(t_save)):
        t_start = float(t_save[i - 1])
        t_stop = float(t_save[i])
        scales, dts = [], []
        save = False
        while not save:
            if t_start + dt >= t_stop:
                dt = t_stop - t_start
                save = True
            else:
                save = False
            scales.append(dt / dt0)
            dts.append(dt)
            t_start += dt
            if len(scales) > max_steps:
                raise ValueError("step count explodes: the truncated dt carried over from a save point "
                                 f"(Solver.jl:35) is {dt}")
        out.append((i, scales, dts))
    return out


def solve(ops, f_init: np.ndarray, dt_initial: float, t_save: Sequence[float], dt0: float,
          verbose: int = 1):
    """Solve (Solver.jl:1-64) with an oracle step; returns the list of saved states and the Cr trace."""
    f = np.array(f_init, dtype=np.float64, copy=True)
    saved = [f.copy()]
    crs = []
    for _, scales, _ in solve_schedule(dt_initial, t_save, dt0):
        for s in scales:
            f, diag, _ = ops.step(f, s, verbose)
            crs.append(diag[0])
        saved.append(f.copy())
    return saved, np.array(crs)


def moments(sp_size: Sequence[int], f: np.ndarray, w: np.ndarray):
    """Per-species number sum(f) and energy sum(f * w) of one cell (DistributionMoments.jl:33,145,162)."""
    sp_size = np.ascontiguousarray(sp_size, dtype=np.int64)
    f = np.ascontiguousarray(f, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    num = np.zeros(len(sp_size))
    en = np.zeros(len(sp_size))
    lib().orc_moments(len(sp_size), _i(sp_size), _d(f), _d(w), _d(num), _d(en))
    return num, en
