"""Generates tests/golden/golden_small.json: known-answer and transliteration vectors.

The reference (DiplodocusTransport.jl) cannot run here (no Julia) and its own test suite is
empty (test/runtests.jl:4-6), so these fixtures come from two independent sources:

1. closed-form known answers derived by hand from the Julia lines (injection only, a 1-D
   upwind flux on a known vector, the clamp table, the Solve step schedule), and
2. a literal pure-Python transliteration of src/SteppingMethods.jl:12-107 with
   update_Big_Bin! (:332-397) on tiny random operators in the reference layout, written
   line by line with Python floats (IEEE doubles like Julia's Float64).

Julia semantics reproduced: `x * b::Bool` is ifelse(b, x, copysign(0, x)); the clamp
literal 1f-10 is a Float32 promoted to Float64; min orders -0.0 below +0.0; NaN maps to Inf
in the CFL reductions.

Run:  python tests/golden/make_golden.py   (rewrites golden_small.json deterministically)
"""
from __future__ import annotations

import json
import math
import os
import random
import struct

HERE = os.path.dirname(os.path.abspath(__file__))


def f32(x: float) -> float:
    return struct.unpack("f", struct.pack("f", x))[0]


THR = f32(1e-10)  # Float64(1f-10)


def mul_bool(x: float, b: bool) -> float:
    return x if b else math.copysign(0.0, x)


def jl_min(a: float, b: float) -> float:
    if a < b:
        return a
    if b < a:
        return b
    return a if math.copysign(1.0, a) < 0 else b


def nan_inf(x: float) -> float:
    return math.inf if math.isnan(x) else x


def div(a: float, b: float) -> float:
    """IEEE division (Python raises on /0)."""
    if b == 0.0:
        if a == 0.0 or math.isnan(a):
            return math.nan
        return math.copysign(math.inf, a) * math.copysign(1.0, b)
    return a / b


def step_literal(N, n_space, M_Bin, M_Emi, colptr, rowval, nzval, invAp, Vol, inj, f, dt_scale, verbose):
    """SteppingMethods.jl:12-107 line by line; matrices column-major flat lists, 0-based CSC."""
    n = N * n_space
    # :31 mul!(df_Flux, F_Flux, f), SparseArrays column order
    df_Flux = [0.0] * n
    for j in range(n):
        for p in range(colptr[j], colptr[j + 1]):
            df_Flux[rowval[p]] += nzval[p] * f[j]
    # :32
    df = [-x for x in df_Flux]
    df_Emi = [0.0] * n
    if M_Emi is not None:  # :35-38
        for k in range(n):
            for r in range(n):
                df_Emi[r] += M_Emi[r + k * n] * f[k]
        df = [a + b for a, b in zip(df, df_Emi)]
    df_Bin = [0.0] * n
    if M_Bin is not None:  # :41-44 -> :360-386
        for cell in range(n_space):
            fv = f[cell * N:(cell + 1) * N]
            S = [0.0] * (N * N)  # :372
            for k in range(N):
                for r in range(N * N):
                    S[r] += M_Bin[r + k * N * N] * fv[k]
            out = [0.0] * N  # :373, S as N x N column-major
            for j in range(N):
                for a in range(N):
                    out[a] += S[a + j * N] * fv[j]
            for a in range(N):  # :380
                df_Bin[cell * N + a] = out[a] * Vol[cell]
        df = [a + b for a, b in zip(df, df_Bin)]
    df = [d * (ia * dt_scale) for d, ia in zip(df, invAp)]  # :46
    sdf = 0.0
    for x in df:
        sdf += x
    diag = {"finite": math.isfinite(sdf), "Cr": 0.0, "Cr_Bin": 0.0, "Cr_Emi": 0.0, "Cr_Flux": 0.0}
    if verbose in (1, 2, 3):
        sf = 0.0
        for x in f:
            sf += x
        if sf != 0.0:
            if verbose == 3:
                if M_Bin is not None:
                    m = math.inf
                    for a, b in zip(df_Bin, f):
                        m = jl_min(m, nan_inf(div(a, b)))
                    diag["Cr_Bin"] = -m
                if M_Emi is not None:
                    m = math.inf
                    for a, b in zip(df_Emi, f):
                        m = jl_min(m, nan_inf(div(a, b)))
                    diag["Cr_Emi"] = -m
                m = math.inf
                for a, b in zip(df_Flux, f):
                    m = jl_min(m, nan_inf(div(-a, b)))
                diag["Cr_Flux"] = -m
            m = math.inf
            for a, b in zip(df, f):
                m = jl_min(m, nan_inf(div(a, b)))
            diag["Cr"] = -m
    newf = []
    for fi, di, ji in zip(f, df, inj):  # :97-101
        v = fi + (di + ji * dt_scale)
        v = mul_bool(v, v >= THR)
        v = mul_bool(v, v != math.inf)
        newf.append(v)
    return newf, diag


def enc(x: float):
    """JSON-safe float: repr string for non-finite values."""
    if math.isfinite(x):
        return x
    return repr(x)


def schedule(dt_initial, t_save, dt0):
    """Solver.jl:25-37 with SteppingMethods.jl:18-27."""
    dt = dt_initial
    out = []
    for i in range(1, len(t_save)):
        t_start, t_stop = t_save[i - 1], t_save[i]
        save = False
        sc = []
        while not save:
            if t_start + dt >= t_stop:
                dt = t_stop - t_start
                save = True
            sc.append(dt / dt0)
            t_start += dt
        out.append(sc)
    return out


def main():
    rnd = random.Random(20261203)
    cases = []
    # ---- transliteration cases: random dense M_Bin (any entries), M_Emi, sparse F
    for ci, (sizes, n_space, verbose) in enumerate((((2, 3), 1, 3), ((3, 2), 2, 3), ((4,), 1, 1))):
        N = sum(sizes)
        n = N * n_space
        M_Bin = [rnd.uniform(-0.02, 0.05) if rnd.random() < 0.6 else 0.0 for _ in range(N * N * N)]
        M_Emi = [rnd.uniform(0.0, 0.03) if rnd.random() < 0.5 else 0.0 for _ in range(n * n)]
        colptr, rowval, nzval = [0], [], []
        for j in range(n):
            rows = sorted(set([j] + [rnd.randrange(n) for _ in range(2)]))
            for r in rows:
                rowval.append(r)
                nzval.append(rnd.uniform(-0.1, 0.2))
            colptr.append(len(rowval))
        invAp = [rnd.uniform(0.8, 1.2) for _ in range(n)]
        Vol = [rnd.uniform(0.5, 1.5) for _ in range(n_space)]
        inj = [rnd.uniform(0.0, 1e-3) for _ in range(n)]
        f = [rnd.uniform(0.01, 1.0) for _ in range(n)]
        f[1] = 5e-11  # below the clamp threshold
        f[-1] = 0.0   # zero state: df/f gives +-Inf or NaN in the CFL reduction
        f0 = list(f)
        dt_scale = 0.75
        steps = []
        for _ in range(3):
            f, d = step_literal(N, n_space, M_Bin, M_Emi, colptr, rowval, nzval, invAp, Vol, inj, f, dt_scale,
                                verbose)
            steps.append({"f": [enc(x) for x in f], "diag": {k: (enc(v) if isinstance(v, float) else v)
                                                              for k, v in d.items()}})
        cases.append({"name": f"literal_{ci}", "sizes": list(sizes), "n_space": n_space, "verbose": verbose,
                      "M_Bin": M_Bin, "M_Emi": M_Emi, "colptr": colptr, "rowval": rowval, "nzval": nzval,
                      "invAp": invAp, "Vol": Vol, "inj": inj, "f0": f0, "dt_scale": dt_scale, "steps": steps})
    # ---- KAT 1: no operators, injection only: f_k = f_0 + k * inj * dt_scale (exact for these values)
    kat_inj = {"f0": [0.5, 0.25, 1.0], "inj": [0.125, 0.0625, 0.0], "dt_scale": 0.5, "steps": 4,
               "expect": [0.5 + 4 * 0.0625, 0.25 + 4 * 0.03125, 1.0]}
    # ---- KAT 2: 1-D upwind flux on 4 cells, velocity 0.25 to the right, closed ends.
    # F (column j loses v f_j, row j+1 gains it): df = -F f; expected by hand.
    f = [1.0, 0.5, 0.25, 0.125]
    v = 0.25
    expect = [f[0] - v * f[0], f[1] + v * f[0] - v * f[1], f[2] + v * f[1] - v * f[2], f[3] + v * f[2]]
    kat_flux = {"colptr": [0, 2, 4, 6, 6], "rowval": [0, 1, 1, 2, 2, 3], "nzval": [v, -v, v, -v, v, -v],
                "f0": f, "dt_scale": 1.0, "expect": expect}
    # ---- KAT 5: clamp table (SteppingMethods.jl:99,101)
    ins = [-1.0, -0.0, 0.0, 5e-11, THR, 1.1e-10, math.nan, math.inf, -math.inf, 1.0]
    outs = []
    for x in ins:
        y = mul_bool(x, x >= THR)
        y = mul_bool(y, y != math.inf)
        outs.append(y)
    kat_clamp = {"in": [enc(x) for x in ins], "out": [enc(x) for x in outs],
                 "signbit": [math.copysign(1.0, x) < 0 for x in outs]}
    # ---- KAT 6: Solve schedule with a dt that does not divide the save interval
    t_save = [0.0, 1.0, 2.5, 2.6]
    sched = schedule(0.4, t_save, 1.0)
    kat_sched = {"dt_initial": 0.4, "t_save": t_save, "dt0": 1.0, "scales": sched,
                 "counts": [len(s) for s in sched]}
    # Float32 dt0 rounding (SteppingStructs.jl:44): dt0 = 0.1 becomes Float32(0.1)
    kat_sched32 = {"dt_initial": 0.05, "t_save": [0.0, 0.2], "dt0": 0.1,
                   "scales": schedule(0.05, [0.0, 0.2], f32(0.1))}
    out = {"cases": cases, "kat_inj": kat_inj, "kat_flux": kat_flux, "kat_clamp": kat_clamp,
           "kat_sched": kat_sched, "kat_sched32": kat_sched32, "thr": THR}
    with open(os.path.join(HERE, "golden_small.json"), "w") as fh:
        json.dump(out, fh, indent=0)


if __name__ == "__main__":
    main()
