"""Python mirror of the reference's stepping API over libdtb.so.

``ForwardEulerStruct(PhaseSpace, Initial, Injection, BinM, EmiM, FluxM)`` follows
SteppingStructs.jl:33-100: it uploads the operators once (M_Bin in the reference layout or
as blocks, M_Emi dense or as pieces, F = X_Flux + P_Flux, invAp = 1 ./ Ap_Flux, Vol) and
keeps f on the device. Calling it, ``method(t_start, t_stop, dt, Verbose) -> (dt, save)``,
is the functor of SteppingMethods.jl:12-107. ``Solve`` follows Solver.jl:1-64.

All compute runs in libdtb.so on a CUDA device; there is no CPU path.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import check, dptr, iptr
from .structs import BinaryMatrices, EmissionMatrices, FluxMatrices, PhaseSpace

THR_F64 = float(np.float32(1e-10))


@dataclass
class OutputStruct:
    """StructsAndDictionaries.jl:362-377: saved states and their times."""

    f: List[np.ndarray] = field(default_factory=list)
    t: List[float] = field(default_factory=list)


def _precision_code(Precision) -> int:
    if Precision in (np.float64, float, "Float64", "f64"):
        return _lib.DTB_F64
    if Precision in (np.float32, "Float32", "f32"):
        return _lib.DTB_F32
    raise ValueError("Precision must be Float32 or Float64 (SteppingStructs.jl:38)")


def _upload_csc(L, ctx, M, part=None) -> None:
    """A flux matrix as 0-based CSC: summed into F (part None) or kept as X_Flux / P_Flux."""
    if M is None or M.nnz == 0:
        return
    M = M.tocsc()
    M.sort_indices()
    colptr = np.ascontiguousarray(M.indptr, dtype=np.int64)
    rowval = np.ascontiguousarray(M.indices, dtype=np.int64)
    nzval = np.ascontiguousarray(M.data, dtype=np.float64)
    if part is None:
        check(L.dtb_add_flux_csc(ctx, M.shape[0], iptr(colptr), iptr(rowval), dptr(nzval)))
    else:
        check(L.dtb_add_flux_csc_part(ctx, part, M.shape[0], iptr(colptr), iptr(rowval), dptr(nzval)))


def _upload_gain(L, ctx, g) -> None:
    G = g.G
    if hasattr(G, "is_cuda") and G.is_cuda:  # torch tensor already in device memory
        import torch
        G = G.contiguous()
        dtype = _lib.DTB_DTYPE_F64 if G.dtype == torch.float64 else _lib.DTB_DTYPE_F32
        if G.dtype not in (torch.float64, torch.float32):
            raise TypeError("device gain blocks must be float32 or float64")
        check(L.dtb_add_gain_block(ctx, g.out_sp, g.in1_sp, g.in2_sp, ctypes.c_void_p(G.data_ptr()), dtype, 1))
        return
    A = np.asarray(G)
    if A.dtype == np.float32:
        A = np.ascontiguousarray(A)
        dtype = _lib.DTB_DTYPE_F32
    else:
        A = np.ascontiguousarray(A, dtype=np.float64)
        dtype = _lib.DTB_DTYPE_F64
    check(L.dtb_add_gain_block(ctx, g.out_sp, g.in1_sp, g.in2_sp, ctypes.c_void_p(A.ctypes.data), dtype, 0))


class ForwardEulerStruct:
    """Explicit Euler method on a B200; SteppingStructs.jl:33-100 for the B200 backend."""

    _flags = 0

    def __init__(self, PhaseSpace: PhaseSpace, Initial, Injection, BinM: BinaryMatrices,
                 EmiM: EmissionMatrices, FluxM: FluxMatrices, *, Adaptive: bool = False,
                 Precision=np.float64, device: int = 0, stream: Optional[int] = None,
                 graph_steps: int = 0):
        self.L = _lib.load()
        self.PhaseSpace = PhaseSpace
        self.Precision = Precision
        self.Adaptive = Adaptive
        self.Implicit = False
        prec = _precision_code(Precision)
        self.dt0 = float(np.float32(PhaseSpace.dt0)) if prec == _lib.DTB_F32 else float(PhaseSpace.dt0)
        self.Binary_Interactions = BinM.has_interactions
        self.Emission_Interactions = EmiM.has_interactions
        self.f_init = np.array(Initial, dtype=np.float64, copy=True)
        self.n = PhaseSpace.n_state
        dims = _lib.Dims()
        sizes = PhaseSpace.species_sizes
        dims.n_species = len(sizes)
        dims.n_space = PhaseSpace.n_space
        for i, s in enumerate(sizes):
            dims.species_size[i] = s
        opts = _lib.Opts(precision=prec, device=device, stream=stream, index_base=0,
                         graph_steps=graph_steps, dt0=float(PhaseSpace.dt0), batch=1, flags=self._flags)
        ctx = ctypes.c_void_p()
        check(self.L.dtb_create(ctypes.byref(dims), ctypes.byref(opts), ctypes.byref(ctx)))
        self.ctx = ctx
        try:
            L = self.L
            _upload_csc(L, ctx, FluxM.X_Flux, _lib.DTB_FLUX_X)
            _upload_csc(L, ctx, FluxM.P_Flux, _lib.DTB_FLUX_P)
            if BinM.M_Bin is not None and sp.issparse(BinM.M_Bin):  # Bin_sparse (BuildBinaryMatrices.jl:44-52)
                M = sp.csc_matrix(BinM.M_Bin)
                colptr = np.ascontiguousarray(M.indptr, dtype=np.int64)
                rowval = np.ascontiguousarray(M.indices, dtype=np.int64)
                nzval = np.ascontiguousarray(M.data, dtype=np.float64)
                check(L.dtb_upload_mbin_csc(ctx, PhaseSpace.n_momentum, iptr(colptr), iptr(rowval), dptr(nzval)))
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
            check(L.dtb_upload_vectors(ctx, dptr(Ap), dptr(Vol), dptr(self.f_init), dptr(inj)))
            check(L.dtb_commit(ctx))
        except Exception:
            self.close()
            raise
        self.last_diag = _lib.StepDiag()

    # ---- the functor (SteppingMethods.jl:12-107)
    def __call__(self, t_start: float, t_stop: float, dt: float, Verbose: int = 1):
        dt_out = ctypes.c_double()
        save = ctypes.c_int32()
        d = self.last_diag
        check(self.L.dtb_step(self.ctx, float(t_start), float(t_stop), float(dt), int(Verbose),
                              ctypes.byref(dt_out), ctypes.byref(save), ctypes.byref(d)))
        self._report(d, Verbose, t_start, t_stop, dt_out.value)
        return dt_out.value, bool(save.value)

    def step_io(self, f_in, t_start: float, t_stop: float, dt: float, Verbose: int = 0,
                out: Optional[np.ndarray] = None):
        """The functor with the state in host memory: f_in (None keeps the device state) is
        uploaded, one step runs and the new state is returned in `out` (allocated when None; may
        be f_in itself), all in one library call with one wait (dtb_step_io). Returns
        (f, dt, save)."""
        A = None if f_in is None else np.ascontiguousarray(f_in, dtype=np.float64)
        if out is None:
            out = np.empty(self.n)
        dt_out = ctypes.c_double()
        save = ctypes.c_int32()
        d = self.last_diag
        if not hasattr(self, "_io_ptrs"):
            self._io_ptrs = (_lib.LastPtr(), _lib.LastPtr())
        pin, pout = self._io_ptrs
        check(self.L.dtb_step_io(self.ctx, pin(A), pout(out), float(t_start), float(t_stop), float(dt),
                                 int(Verbose), ctypes.byref(dt_out), ctypes.byref(save), ctypes.byref(d)))
        self._report(d, Verbose, t_start, t_stop, dt_out.value)
        return out, dt_out.value, bool(save.value)

    @staticmethod
    def _report(d, Verbose: int, t_start: float, t_stop: float, dt: float) -> None:
        # SteppingMethods.jl:87-93
        if not d.finite:
            print("non-finite value in df calculation")
        if Verbose == 1 and d.cr > 1.0:
            print(f"Cr = {d.cr}, t={t_start}, dt={dt}, system may be unstable")
        elif Verbose == 2:
            print(f"\rCr = {d.cr}, t={t_start}, dt={dt}")
        elif Verbose == 3:
            print(f"Cr = {d.cr},Cr_Bin = {d.cr_bin}, Cr_Emi = {d.cr_emi}, Cr_Flux = {d.cr_flux}, "
                  f"t={t_start}, t_save ={t_stop}, dt={dt}")

    # ---- state access
    @property
    def f(self) -> np.ndarray:
        out = np.empty(self.n)
        check(self.L.dtb_get_f(self.ctx, dptr(out)))
        return out

    @f.setter
    def f(self, value) -> None:
        v = np.ascontiguousarray(value, dtype=np.float64)
        check(self.L.dtb_set_f(self.ctx, dptr(v)))

    def reset(self) -> None:
        check(self.L.dtb_reset(self.ctx))

    def prepare(self) -> None:
        """Captures and uploads the step graphs now (dtb_prepare), so no later run pays for it."""
        check(self.L.dtb_prepare(self.ctx))

    def run(self, dt_scales: Sequence[float], Verbose: int = 0, diag: bool = False):
        s = np.ascontiguousarray(dt_scales, dtype=np.float64)
        hist = (_lib.StepDiag * len(s))() if diag else None
        check(self.L.dtb_run(self.ctx, dptr(s), len(s), int(Verbose), hist))
        return hist

    def moments(self, weights) -> tuple:
        """Per (cell, species) FP64 number and energy (DistributionMoments.jl:33,145,162)."""
        w = np.ascontiguousarray(weights, dtype=np.float64)
        ns = len(self.PhaseSpace.species_sizes)
        num = np.zeros(self.PhaseSpace.n_space * ns)
        en = np.zeros_like(num)
        check(self.L.dtb_moments(self.ctx, dptr(w), dptr(num), dptr(en)))
        return num.reshape(-1, ns), en.reshape(-1, ns)

    def device_bytes(self) -> int:
        v = ctypes.c_int64()
        check(self.L.dtb_device_bytes(self.ctx, ctypes.byref(v)))
        return v.value

    def sync(self) -> None:
        check(self.L.dtb_sync(self.ctx))

    def close(self) -> None:
        if getattr(self, "ctx", None):
            self.L.dtb_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ForwardSymplecticEulerStruct(ForwardEulerStruct):
    """Forward symplectic (semi-implicit) Euler on a B200: SteppingStructs.jl:104-229 for the B200
    backend, stepping as SteppingMethods.jl:120-243 (momentum fluxes, emission and binary terms
    first, clamped at 1f-10; then the space fluxes on the updated f, clamped at 1f-20). The
    diagnostics report the whole-step Cr (:217-218); the per-term Crs of Verbose == 3 are not
    reduced on the device."""

    _flags = _lib.DTB_FLAG_SYMPLECTIC


def solve_schedule(dt_initial: float, t_save: Sequence[float], dt0: float, precision: int = _lib.DTB_F64):
    """Host-side step schedule of Solve computed by the library (no device needed)."""
    L = _lib.load()
    t = np.ascontiguousarray(t_save, dtype=np.float64)
    per = np.zeros(max(1, len(t) - 1), dtype=np.int64)
    total = ctypes.c_int64()
    check(L.dtb_solve_schedule(float(dt_initial), dptr(t), len(t), float(dt0), precision, iptr(per), None, 0,
                               ctypes.byref(total)))
    scales = np.zeros(max(1, total.value))
    check(L.dtb_solve_schedule(float(dt_initial), dptr(t), len(t), float(dt0), precision, iptr(per), dptr(scales),
                               total.value, ctypes.byref(total)))
    return per[:len(t) - 1], scales[:total.value]


def Solve(method: ForwardEulerStruct, dt_initial: float, t_save: Sequence[float], *, progress: bool = False,
          fileName: Optional[str] = None, fileLocation: Optional[str] = None, Verbose: int = 1,
          stepwise: bool = False, moment_weights=None) -> OutputStruct:
    """Solver.jl:1-64. ``stepwise=True`` calls the functor once per step exactly like the
    reference loop; the default enqueues the whole schedule as CUDA-graph replays with the save
    points copied out behind the stepping (dtb_solve_ex). With ``moment_weights`` (one energy
    weight per momentum state) the output also holds ``number`` and ``energy``, arrays
    (n_save, n_space, n_species) of FP64 moments computed on the device at every save point."""
    t_save = [float(t) for t in t_save]
    n_save = len(t_save)
    out = OutputStruct()
    if stepwise:
        method.reset()
        # Solver.jl:10-14 saves f_init, which the struct holds in its precision (SteppingStructs.jl:24,53)
        single = _precision_code(method.Precision) == _lib.DTB_F32
        out.f.append(method.f_init.astype(np.float32).astype(np.float64) if single else method.f_init.copy())
        out.t.append(t_save[0])
        dt = float(dt_initial)
        for i in range(1, n_save):
            t_start, t_stop = t_save[i - 1], t_save[i]
            save = False
            while not save:
                dt, save = method(t_start, t_stop, dt, Verbose)
                t_start += dt
            out.f.append(method.f)
            out.t.append(t_stop)
        return out
    F = np.zeros((n_save, method.n))
    nsteps = ctypes.c_int64()
    t = np.ascontiguousarray(t_save, dtype=np.float64)
    if moment_weights is None:
        check(method.L.dtb_solve(method.ctx, float(dt_initial), dptr(t), n_save, int(Verbose), dptr(F),
                                 ctypes.byref(nsteps)))
    else:
        ps = method.PhaseSpace
        w = np.ascontiguousarray(moment_weights, dtype=np.float64)
        if w.shape != (ps.n_momentum,):
            raise ValueError("moment_weights must hold one weight per momentum state")
        shape = (n_save, ps.n_space, len(ps.species_sizes))
        num = np.zeros(shape)
        en = np.zeros(shape)
        check(method.L.dtb_solve_ex(method.ctx, float(dt_initial), dptr(t), n_save, int(Verbose), dptr(F), dptr(w),
                                    dptr(num), dptr(en), ctypes.byref(nsteps)))
        out.number, out.energy = num, en
    out.f = [F[i].copy() for i in range(n_save)]
    out.t = list(t_save)
    out.n_steps = nsteps.value
    return out
