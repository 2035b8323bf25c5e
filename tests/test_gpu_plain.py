"""Parity of the plain (single-instance) CUDA path with the oracle, through the C ABI.

Tolerances: relative L-infinity (max|f - f_ref| / max|f_ref|) <= 1e-12 for the FP64 path;
<= 2e-5 for the FP32 path against the FP64 oracle (FP32 operators and state).
"""
import json
import math
import os

import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from dtb import _lib, synth
from dtb.stepping import ForwardEulerStruct, Solve
from dtb.structs import (BinaryMatrices, EmissionMatrices, FluxMatrices, PhaseSpace, blocked_to_ref,
                         emission_to_dense, energy_weights)

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden_small.json")))


def rel_linf(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(np.asarray(b))))


def make_method(w, precision=np.float64, ref_layout=False, **kw):
    binm, emim = w.binm, w.emim
    if ref_layout:
        binm = BinaryMatrices(M_Bin=blocked_to_ref(w.ps, w.binm), Domain=w.binm.Domain)
        emim = EmissionMatrices(M_Emi=emission_to_dense(w.ps, w.emim))
    return ForwardEulerStruct(w.ps, w.f0, w.inj, binm, emim, w.fluxm, Precision=precision, **kw)


@pytest.mark.parametrize("p,u,seed,n_space,randv,emi", [
    (4, 2, 0, 1, False, True), (4, 3, 1, 1, True, True), (6, 2, 2, 2, True, True),
    (5, 3, 3, 1, True, False), (16, 8, 4, 1, False, True), (7, 5, 5, 3, True, True)])
def test_f64_functor_matches_oracle(cuda, p, u, seed, n_space, randv, emi):
    w = synth.small(p_num=p, u_num=u, seed=seed, n_space=n_space, with_emission=emi, randomize_vectors=randv)
    m = make_method(w)
    ops = oracle.blocked_from_workload(w)
    f = w.f0.copy()
    for k in range(25):
        dt_scale = 0.9 if k % 5 else 0.6
        _, _ = m(0.0, 1e9, dt_scale * m.dt0, 3)
        f, diag, _ = ops.step(f, dt_scale, 3)
        d = m.last_diag
        assert bool(d.finite) == bool(diag[4])
        for got, exp in zip((d.cr, d.cr_bin, d.cr_emi, d.cr_flux), diag[:4]):
            assert got == pytest.approx(exp, rel=1e-10, abs=1e-300) or (math.isinf(exp) and got == exp)
    assert rel_linf(m.f, f) <= TOL64
    m.close()


@pytest.mark.parametrize("ci", range(3))
def test_golden_literal_cases(cuda, ci):
    """Arbitrary reference-layout M_Bin (not gain/loss structured), dense M_Emi, random CSC flux."""
    c = GOLD["cases"][ci]
    sizes = c["sizes"]
    N = sum(sizes)
    n = N * c["n_space"]
    ps = PhaseSpace(name_list=[f"s{i}" for i in range(len(sizes))], px_num_list=sizes,
                    py_num_list=[1] * len(sizes), pz_num_list=[1] * len(sizes), x_num=c["n_space"])
    F = sp.csc_matrix((c["nzval"], c["rowval"], c["colptr"]), shape=(n, n))
    fluxm = FluxMatrices(Ap_Flux=1.0 / np.array(c["invAp"]), Am_Flux=np.zeros(n), X_Flux=sp.csc_matrix((n, n)),
                         P_Flux=F, Vol=np.array(c["Vol"]))
    binm = BinaryMatrices(M_Bin=np.array(c["M_Bin"]).reshape((N * N, N), order="F"))
    emim = EmissionMatrices(M_Emi=np.array(c["M_Emi"]).reshape((n, n), order="F"))
    m = ForwardEulerStruct(ps, c["f0"], c["inj"], binm, emim, fluxm)
    for st in c["steps"]:
        m(0.0, 1e9, c["dt_scale"], c["verbose"])
        exp = np.array([float(x) for x in st["f"]])
        assert rel_linf(m.f, exp) <= TOL64
        d = st["diag"]
        for got, key in zip((m.last_diag.cr, m.last_diag.cr_bin, m.last_diag.cr_emi, m.last_diag.cr_flux),
                            ("Cr", "Cr_Bin", "Cr_Emi", "Cr_Flux")):
            e = float(d[key])
            assert (got == e) if math.isinf(e) else got == pytest.approx(e, rel=1e-9, abs=1e-300)
    m.close()


def test_reference_layout_upload_equals_blocked(cuda):
    w = synth.small(p_num=6, u_num=3, seed=11, randomize_vectors=True)
    a = make_method(w)
    b = make_method(w, ref_layout=True)
    sc = np.full(40, 0.8)
    a.run(sc)
    b.run(sc)
    assert rel_linf(a.f, b.f) <= 1e-13
    a.close()
    b.close()


def test_functor_run_and_solve_agree_bitwise(cuda):
    w = synth.small(p_num=8, u_num=4, seed=12, randomize_vectors=True)
    t_save = [0.0, 3.0, 7.5, 8.0]
    m1 = make_method(w, graph_steps=4)
    out_step = Solve(m1, 0.4, t_save, Verbose=0, stepwise=True)
    out_graph = Solve(m1, 0.4, t_save, Verbose=0)
    for a, b in zip(out_step.f, out_graph.f):
        np.testing.assert_array_equal(a, b)
    # oracle Solve on the same schedule
    saved, _ = oracle.solve(oracle.blocked_from_workload(w), w.f0, 0.4, t_save, 1.0, verbose=0)
    for a, b in zip(out_graph.f, saved):
        assert rel_linf(a, b) <= TOL64
    assert out_graph.n_steps == sum(len(s[1]) for s in oracle.solve_schedule(0.4, t_save, 1.0))
    m1.close()


@pytest.mark.parametrize("precision", [np.float64, np.float32])
def test_step_io_equals_set_step_get(cuda, precision):
    """dtb_step_io (upload, step, download with one wait) gives, bit for bit, the state, dt, save
    flag and diagnostics of dtb_set_f + dtb_step + dtb_get_f: with a fresh host state every step,
    with f_out aliasing f_in, with f_in None (the device state is kept), and at a truncated last
    step."""
    import torch
    w = synth.small(p_num=8, u_num=4, seed=33, randomize_vectors=True)
    a = make_method(w, precision=precision)
    b = make_method(w, precision=precision)
    rng = np.random.default_rng(5)
    f_pin = torch.empty(w.ps.n_state, dtype=torch.float64).pin_memory().numpy()
    for k in range(6):
        f_host = np.abs(w.f0 * (1.0 + 0.1 * rng.standard_normal(w.ps.n_state)))
        f_pin[:] = f_host
        t_stop = 5.0 if k < 5 else 0.3  # the last step is truncated at t_stop
        out, dt_a, sv_a = a.step_io(f_pin, 0.0, t_stop, 0.9 * a.dt0, 3, out=f_pin)
        assert out is f_pin
        b.f = f_host
        dt_b, sv_b = b(0.0, t_stop, 0.9 * b.dt0, 3)
        np.testing.assert_array_equal(f_pin, b.f)
        assert (dt_a, sv_a) == (dt_b, sv_b)
        for fld in ("cr", "cr_bin", "cr_emi", "cr_flux", "sum_df", "sum_f", "finite"):
            assert getattr(a.last_diag, fld) == getattr(b.last_diag, fld), fld
    got, _, _ = a.step_io(None, 0.0, 5.0, a.dt0, 0)  # pageable output, device state kept
    b(0.0, 5.0, b.dt0, 0)
    np.testing.assert_array_equal(got, b.f)
    np.testing.assert_array_equal(a.f, b.f)
    a.close()
    b.close()


def test_config0_full_run(cuda):
    """Config 0: N_s = 128, two species, FP64, 1000 steps at fixed dt."""
    w = synth.config0(0)
    m = make_method(w)
    n_steps = 1000
    out = Solve(m, 1.0, [0.0, 500.0, 1000.0], Verbose=1)
    ops = oracle.blocked_from_workload(w)
    saved, crs = oracle.solve(ops, w.f0, 1.0, [0.0, 500.0, 1000.0], 1.0)
    assert out.n_steps == n_steps
    assert rel_linf(out.f[1], saved[1]) <= TOL64
    assert rel_linf(out.f[2], saved[2]) <= TOL64
    assert np.count_nonzero(out.f[2]) == np.count_nonzero(saved[2])  # same clamp decisions
    m.close()


def test_f32_path_against_f64_oracle(cuda):
    w = synth.small(p_num=16, u_num=8, seed=13, randomize_vectors=True)
    m = make_method(w, precision=np.float32)
    ops = oracle.blocked_from_workload(w)
    f = w.f0.copy()
    sc = np.full(100, 0.95)
    m.run(sc)
    for s in sc:
        f, _, _ = ops.step(f, s, 0)
    assert rel_linf(m.f, f) <= TOL32
    m.close()


def test_config1_recipe_full_run_length_f32(cuda):
    """Config 1's recipe (p over 1e-3..1e3, FP32 operators and state, the reference's CUDA
    precision) on a reduced grid (2 x 128 states) over the configuration's 2,000 steps: within
    the FP32 tolerance of the FP64 oracle run of the same inputs."""
    w = synth.two_species(16, 1e-3, 1e3, 8, seed=1)
    m = make_method(w, precision=np.float32)
    ops = oracle.blocked_from_workload(w)
    f = w.f0.copy()
    m.run(np.ones(2000))
    for _ in range(2000):
        f, _, _ = ops.step(f, 1.0, 0)
    assert rel_linf(m.f, f) <= TOL32
    m.close()


def test_clamp_semantics_on_device(cuda):
    """Negative, tiny, NaN and Inf states go through SteppingMethods.jl:97-101 exactly."""
    w = synth.small(p_num=4, u_num=2, seed=14, with_emission=False)
    n = w.ps.n_state
    f0 = w.f0.copy()
    specials = [-1.0, 5e-11, float(np.float32(1e-10)), 1.1e-10, np.inf, 0.0, -0.0]
    f0[:len(specials)] = specials
    w.f0 = f0
    w.binm = BinaryMatrices()
    w.fluxm.P_Flux = sp.csc_matrix((n, n))
    w.inj = np.zeros(n)
    m = make_method(w)
    m(0.0, 1e9, 1.0, 0)
    got = m.f
    exp, _, _ = oracle.ref_from_workload(w).step(f0, 1.0, 0)
    np.testing.assert_array_equal(got, exp)
    np.testing.assert_array_equal(np.signbit(got), np.signbit(exp))
    m.close()


def test_device_moments_match_oracle(cuda):
    w = synth.small(p_num=16, u_num=8, seed=15)
    m = make_method(w)
    m.run(np.full(10, 1.0))
    wts = energy_weights(w.ps)
    num, en = m.moments(wts)
    f = m.f
    onum, oen = oracle.moments(w.ps.species_sizes, f, wts)
    np.testing.assert_allclose(num[0], onum, rtol=1e-14)
    np.testing.assert_allclose(en[0], oen, rtol=1e-14)
    m.close()


def test_config1_full_size_properties(cuda):
    """Config 1 (N_s = 1024, FP32 G of 1024 x 1,048,576 per species) at full size:
    (a) one step matches the FP64 oracle on a sample of rows (gain rows from the same G);
    (b) with a number-conserving loss built from G, species numbers stay constant."""
    import torch
    w = synth.config1(seed=1, gain_on_device=True)
    ns = w.ps.species_sizes[0]
    m = make_method(w, precision=np.float32)
    m(0.0, 1e9, 1.0, 0)
    f1 = m.f
    # FP64 oracle of the same step on sampled rows; all O(N^2) terms in numpy
    f0 = w.f0.astype(np.float32).astype(np.float64)
    F = w.fluxm.F_Flux.astype(np.float32).astype(np.float64)
    flux = F @ f0
    emi = np.zeros_like(f0)
    for b in w.emim.blocks:
        E = np.asarray(b.E, dtype=np.float32).astype(np.float64)
        emi[b.row0:b.row0 + E.shape[0]] += E @ f0[b.col0:b.col0 + E.shape[1]]
    loss = np.zeros_like(f0)
    off = w.ps.momentum_species_offset
    for l in w.binm.losses:
        L = np.asarray(l.L, dtype=np.float32).astype(np.float64)
        loss[off[l.sp]:off[l.sp] + ns] += L @ f0[off[l.other_sp]:off[l.other_sp] + ns]
    rng = np.random.default_rng(0)
    rows = np.sort(rng.choice(2 * ns, 48, replace=False))
    for r in rows:
        sp_out = r // ns
        G = w.binm.gains[sp_out].G
        Grow = G[r - off[sp_out]].double().cpu().numpy()[None]
        gain = oracle.gain_rows(Grow, 0, 1, f0[:ns], f0[ns:])[0]
        df = -flux[r] + emi[r] + (gain - f0[r] * loss[r])
        exp = oracle.clamp(f0[r] + df)
        assert abs(f1[r] - exp) <= TOL32 * np.max(np.abs(f1)), (r, f1[r], exp)
    m.close()
    # (b) conservation with L_e[b, c] = sum_a G_e[a, b, c], L_g[c, b] = sum_a G_g[a, b, c]
    from dtb.structs import LossBlock
    Le = w.binm.gains[0].G.double().sum(0).cpu().numpy()
    Lg = w.binm.gains[1].G.double().sum(0).t().cpu().numpy()
    w.binm.losses = [LossBlock(0, 1, Le), LossBlock(1, 0, Lg)]
    w.emim.blocks = []
    m = make_method(w, precision=np.float32)
    n0 = m.f
    m.run(np.full(50, 1.0))
    n1 = m.f
    for s in range(2):
        sl = slice(s * ns, (s + 1) * ns)
        assert abs(n1[sl].sum() - n0[sl].sum()) / n0[sl].sum() < 1e-5
    m.close()
    del w
    torch.cuda.empty_cache()


@pytest.mark.parametrize("precision,tol", [(np.float64, TOL64), (np.float32, TOL32)])
def test_symplectic_euler_matches_oracle(cuda, precision, tol):
    """ForwardSymplecticEuler (SteppingMethods.jl:120-243) on 3 space cells with a space flux X
    and the momentum flux P kept apart; 30 steps against the FP64 oracle restatement."""
    from dtb.stepping import ForwardSymplecticEulerStruct
    w = synth.small(p_num=6, u_num=3, seed=17, n_space=3, randomize_vectors=True)
    w.fluxm.X_Flux = synth.space_flux(w.ps, np.random.default_rng(5), 1.0)
    m = ForwardSymplecticEulerStruct(w.ps, w.f0, w.inj, w.binm, w.emim, w.fluxm, Precision=precision)
    r = oracle.ref_from_workload(w)
    L = oracle.lib()
    X, P = (oracle._csc_arrays(M) for M in (w.fluxm.X_Flux, w.fluxm.P_Flux))
    f = w.f0.copy()
    d = np.zeros(8)
    thr_m = float(np.float32(1e-10))
    thr_s = float(np.float32(1e-20))
    for k in range(30):
        dt = 0.9 if k % 3 else 0.7
        m(0.0, 1e9, dt, 1)
        rc = L.orc_step_symplectic_ref(r.n_mom, r.n_space, oracle._d(r.M_Bin), oracle._d(r.M_Emi),
                                       oracle._i(X[0]), oracle._i(X[1]), oracle._d(X[2]),
                                       oracle._i(P[0]), oracle._i(P[1]), oracle._d(P[2]), 0,
                                       oracle._d(r.invAp), oracle._d(r.Vol), oracle._d(r.inj), dt,
                                       thr_m, thr_s, 1, oracle._d(f), oracle._d(d), oracle._b(r.dom))
        assert rc == 0
        assert m.last_diag.cr == pytest.approx(d[0], rel=1e-6 if precision == np.float32 else 1e-10)
    assert rel_linf(m.f, f) <= tol
    m.close()


def test_bounded_wait_gives_up_and_context_stays_usable(cuda):
    """A device wait on a barrier nothing completes gives up after its limit and reports
    DTB_ETIMEOUT; the same context then steps normally (no fault, no hang)."""
    w = synth.small(p_num=4, u_num=2, seed=31)
    m = make_method(w)
    rc = m.L.dtb_selftest_bounded_wait(m.ctx, 0.2)
    assert rc == _lib.DTB_ETIMEOUT
    assert b"self-test" in m.L.dtb_last_error()
    m(0.0, 1e9, 1.0, 0)
    f, _, _ = oracle.blocked_from_workload(w).step(w.f0, 1.0, 0)
    assert rel_linf(m.f, f) <= TOL64
    m.close()


@pytest.mark.parametrize("precision,tol,domain", [(np.float64, TOL64, [0, 2]), (np.float32, TOL32, [1]),
                                                  (np.float64, TOL64, []), (np.float64, TOL64, [2, 9, -1])])
def test_bin_domain_matches_oracle(cuda, precision, tol, domain):
    """BinM.Domain on 3 space cells: the gain kernel runs only the listed cells and the row
    kernel adds a zero binary term elsewhere; 25 steps against the FP64 oracle with the same
    domain, diagnostics included."""
    w = synth.small(p_num=6, u_num=3, seed=23, n_space=3, randomize_vectors=True)
    w.binm.Domain = domain
    m = make_method(w, precision=precision)
    ops = oracle.blocked_from_workload(w)
    f = w.f0.copy()
    for k in range(25):
        _, _ = m(0.0, 1e9, 0.9 * m.dt0, 3)
        f, diag, _ = ops.step(f, 0.9, 3, thr=oracle.THR_F64)
        assert bool(m.last_diag.finite) == bool(diag[4])
    assert m.last_diag.cr == pytest.approx(diag[0], rel=1e-6 if precision == np.float32 else 1e-10)
    assert rel_linf(m.f, f) <= tol
    m.close()


def test_bin_domain_reference_layout_and_symplectic(cuda):
    """The domain applies to a reference-layout M_Bin upload and to the symplectic step."""
    from dtb.stepping import ForwardSymplecticEulerStruct
    w = synth.small(p_num=5, u_num=2, seed=29, n_space=3, randomize_vectors=True)
    w.binm.Domain = [1]
    m = make_method(w, ref_layout=True)
    r = oracle.ref_from_workload(w)
    f = w.f0.copy()
    for _ in range(20):
        m(0.0, 1e9, 0.8 * m.dt0, 1)
        f, _, _ = r.step(f, 0.8, 1)
    assert rel_linf(m.f, f) <= TOL64
    m.close()
    w.fluxm.X_Flux = synth.space_flux(w.ps, np.random.default_rng(6), 1.0)
    s = ForwardSymplecticEulerStruct(w.ps, w.f0, w.inj, w.binm, w.emim, w.fluxm, Precision=np.float64)
    r = oracle.ref_from_workload(w)
    X, P = (oracle._csc_arrays(M) for M in (w.fluxm.X_Flux, w.fluxm.P_Flux))
    L = oracle.lib()
    f = w.f0.copy()
    d = np.zeros(8)
    for _ in range(20):
        s(0.0, 1e9, 0.8 * s.dt0, 1)
        rc = L.orc_step_symplectic_ref(r.n_mom, r.n_space, oracle._d(r.M_Bin), oracle._d(r.M_Emi),
                                       oracle._i(X[0]), oracle._i(X[1]), oracle._d(X[2]),
                                       oracle._i(P[0]), oracle._i(P[1]), oracle._d(P[2]), 0,
                                       oracle._d(r.invAp), oracle._d(r.Vol), oracle._d(r.inj), 0.8,
                                       oracle.THR_F64, float(np.float32(1e-20)), 1, oracle._d(f), oracle._d(d),
                                       oracle._b(r.dom))
        assert rc == 0
    assert rel_linf(s.f, f) <= TOL64
    s.close()


def _sparse_mbin(ps, rng, density=0.04, band=2):
    """A sparse reference-layout M_Bin (N^2 x N): banded in (j, k) so that runs of consecutive
    b-rows form, random elsewhere, plus loss-form entries (j == a or k == a)."""
    N = ps.n_momentum
    rows, cols, vals = [], [], []
    for a in range(N):
        for j in range(N):
            if rng.random() < 0.35:
                for k in range(max(0, j - band), min(N, j + band + 1)):
                    rows.append(j * N + a)
                    cols.append(k)
                    vals.append(rng.uniform(0.0, 1e-2))
        for k in rng.choice(N, size=max(1, int(density * N)), replace=False):
            rows.append(a * N + a)  # j == a: loss form
            cols.append(int(k))
            vals.append(-rng.uniform(0.0, 1e-2))
    n_rand = int(density * N * N * N / 10)
    rows += list(rng.integers(0, N * N, n_rand))
    cols += list(rng.integers(0, N, n_rand))
    vals += list(rng.uniform(-1e-3, 1e-2, n_rand))
    return sp.csc_matrix((vals, (rows, cols)), shape=(N * N, N))


@pytest.mark.parametrize("precision,tol", [(np.float64, TOL64), (np.float32, TOL32)])
def test_sparse_mbin_matches_oracle(cuda, precision, tol):
    """Bin_sparse (BuildBinaryMatrices.jl:44-52): a sparse M_Bin uploaded as CSC; the gain
    kernel streams only nonzero b-rows trimmed to their c-spans. 20 steps on 2 cells against
    the FP64 oracle with the dense matrix, and against the dense upload on the GPU."""
    w = synth.small(p_num=6, u_num=3, seed=51, n_space=2, randomize_vectors=True)
    M = _sparse_mbin(w.ps, np.random.default_rng(7))
    w.binm = BinaryMatrices(M_Bin=M)
    m = ForwardEulerStruct(w.ps, w.f0, w.inj, w.binm, w.emim, w.fluxm, Precision=precision)
    d = ForwardEulerStruct(w.ps, w.f0, w.inj, BinaryMatrices(M_Bin=M.toarray()), w.emim, w.fluxm,
                           Precision=precision)
    r = oracle.ref_from_workload(w)
    f = w.f0.copy()
    for _ in range(20):
        m(0.0, 1e9, 0.8 * m.dt0, 1)
        d(0.0, 1e9, 0.8 * d.dt0, 1)
        f, diag, _ = r.step(f, 0.8, 1)
    assert rel_linf(m.f, f) <= tol
    assert rel_linf(m.f, d.f) <= (1e-13 if precision == np.float64 else 1e-5)
    m.close()
    d.close()


def test_sparse_mbin_duplicates_and_empty_columns(cuda):
    """Duplicate (row, column) entries are summed like sparse(I, J, V); empty columns and
    all-zero output rows are fine; the same matrix as a dense upload gives the same step."""
    w = synth.small(p_num=4, u_num=2, seed=52)
    N = w.ps.n_momentum
    rng = np.random.default_rng(9)
    cols = {k: [] for k in range(N)}
    for _ in range(300):
        k = int(rng.integers(0, N // 2)) * 2  # odd columns stay empty
        cols[k].append((int(rng.integers(0, N * N)), float(rng.uniform(0, 1e-2))))
    cols[0] += [(5, 1e-3), (5, 2e-3)]  # an explicit duplicate
    colptr = [0]
    rowval, nzval = [], []
    dense = np.zeros((N * N, N))
    for k in range(N):
        for rr, v in cols[k]:
            rowval.append(rr)
            nzval.append(v)
            dense[rr, k] += v
        colptr.append(len(rowval))
    # the context is built by hand to pass the raw CSC (with duplicates) through the C ABI
    import ctypes
    L = _lib.load()
    dims = _lib.Dims()
    dims.n_species = len(w.ps.species_sizes)
    dims.n_space = 1
    for i, s in enumerate(w.ps.species_sizes):
        dims.species_size[i] = s
    opts = _lib.Opts(precision=_lib.DTB_F64, device=0, stream=None, index_base=0, graph_steps=16,
                     dt0=1.0, batch=1, flags=0)
    ctx = ctypes.c_void_p()
    assert L.dtb_create(ctypes.byref(dims), ctypes.byref(opts), ctypes.byref(ctx)) == 0
    cp_ = np.array(colptr, dtype=np.int64)
    rv = np.array(rowval, dtype=np.int64)
    nz = np.array(nzval, dtype=np.float64)
    assert L.dtb_upload_mbin_csc(ctx, N, cp_.ctypes.data_as(_lib._ip), rv.ctypes.data_as(_lib._ip),
                                 nz.ctypes.data_as(_lib._dp)) == 0
    Ap = np.ones(N)
    Vol = np.ones(1)
    inj = np.zeros(N)
    f0 = np.ascontiguousarray(w.f0, dtype=np.float64)
    assert L.dtb_upload_vectors(ctx, Ap.ctypes.data_as(_lib._dp), Vol.ctypes.data_as(_lib._dp),
                                f0.ctypes.data_as(_lib._dp), inj.ctypes.data_as(_lib._dp)) == 0
    dt_out = ctypes.c_double()
    save = ctypes.c_int32()
    dg = _lib.StepDiag()
    assert L.dtb_step(ctx, 0.0, 1e9, 1.0, 0, ctypes.byref(dt_out), ctypes.byref(save), ctypes.byref(dg)) == 0
    got = np.empty(N)
    assert L.dtb_get_f(ctx, got.ctypes.data_as(_lib._dp)) == 0
    L.dtb_destroy(ctx)
    r = oracle.RefOperands(N, 1, dense, None, sp.csc_matrix((N, N)), Ap, Vol, inj)
    f, _, _ = r.step(f0, 1.0, 0)
    assert rel_linf(got, f) <= TOL64
    # a row index past N^2 is refused
    bad = rv.copy()
    bad[0] = N * N
    ctx2 = ctypes.c_void_p()
    assert L.dtb_create(ctypes.byref(dims), ctypes.byref(opts), ctypes.byref(ctx2)) == 0
    assert L.dtb_upload_mbin_csc(ctx2, N, cp_.ctypes.data_as(_lib._ip), bad.ctypes.data_as(_lib._ip),
                                 nz.ctypes.data_as(_lib._dp)) == _lib.DTB_EINVAL
    L.dtb_destroy(ctx2)


def test_nan_in_state_is_flagged_and_clamped_like_the_reference(cuda):
    """Host-side fault injection on the numeric path: a NaN seeded into f. The step reports a
    non-finite df (SteppingMethods.jl:48-50) and the clamp of :99-101 (x * (x >= thr), Julia's
    strong zero) turns every NaN into 0, exactly as the FP64 oracle does; the next step is finite."""
    w = synth.small(p_num=8, u_num=4, seed=17)
    m = make_method(w)
    f0 = w.f0.copy()
    f0[5] = np.nan
    m.f = f0
    m(0.0, 1e9, 1.0, 1)
    assert m.last_diag.finite == 0
    ops = oracle.blocked_from_workload(w)
    f, _, _ = ops.step(f0, 1.0, 0)
    got = m.f
    # the NaN reaches every row through the gain term, so both give all zeros here
    assert np.all(np.isfinite(got)) and np.array_equal(got == 0, f == 0)
    assert np.max(np.abs(got - f)) <= TOL64 * np.max(np.abs(w.f0))
    m.f = w.f0
    m(0.0, 1e9, 1.0, 1)
    assert m.last_diag.finite == 1
    m.close()


def test_malformed_flux_csc_is_refused_and_the_context_stays_usable(cuda):
    """Host-side fault injection: a flux CSC with a row index out of range, and one whose colptr
    is not monotone, are refused with DTB_EINVAL before anything reaches the device; the same
    context then takes the valid matrices and steps as the oracle."""
    import ctypes
    from dtb.stepping import _upload_gain
    L = _lib.load()
    w = synth.small(p_num=4, u_num=2, seed=19)
    n = w.ps.n_state
    dims = _lib.Dims()
    dims.n_species = 2
    dims.n_space = 1
    for i, s_ in enumerate(w.ps.species_sizes):
        dims.species_size[i] = s_
    opts = _lib.Opts(precision=_lib.DTB_F64, device=0, index_base=0, graph_steps=16, dt0=1.0, batch=1)
    ctx = ctypes.c_void_p()
    _lib.check(L.dtb_create(ctypes.byref(dims), ctypes.byref(opts), ctypes.byref(ctx)))
    colptr = np.arange(n + 1, dtype=np.int64)
    rowval = np.zeros(n, dtype=np.int64)
    rowval[3] = n  # out of range
    vals = np.ones(n)
    ip = lambda a: a.ctypes.data_as(_lib._ip)  # noqa: E731
    assert L.dtb_add_flux_csc(ctx, n, ip(colptr), ip(rowval), _lib.dptr(vals)) == _lib.DTB_EINVAL
    assert b"out of range" in L.dtb_last_error()
    bad = colptr.copy()
    bad[4], bad[5] = bad[5], bad[4]
    rowval[3] = 0
    assert L.dtb_add_flux_csc(ctx, n, ip(bad), ip(rowval), _lib.dptr(vals)) == _lib.DTB_EINVAL
    assert b"monotone" in L.dtb_last_error()
    L.dtb_destroy(ctx)
    # the valid workload on a fresh context of the same library state steps as the oracle
    m = make_method(w)
    m(0.0, 1e9, 1.0, 0)
    ops = oracle.blocked_from_workload(w)
    f, _, _ = ops.step(w.f0.copy(), 1.0, 0)
    assert rel_linf(m.f, f) <= TOL64
    m.close()
