"""The oracle (CPU FP64 restatement) against the golden fixtures and known answers (no GPU)."""
import json
import math
import os

import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from dtb import synth
from dtb.structs import blocked_to_ref

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden_small.json")))


def dec(x):
    return float(x) if not isinstance(x, str) else float(x)


def _case_ops(c):
    N = sum(c["sizes"])
    n = N * c["n_space"]
    M_Bin = np.array(c["M_Bin"]).reshape((N * N, N), order="F")
    M_Emi = np.array(c["M_Emi"]).reshape((n, n), order="F")
    F = sp.csc_matrix((c["nzval"], c["rowval"], c["colptr"]), shape=(n, n))
    return oracle.RefOperands(N, c["n_space"], M_Bin, M_Emi, F, c["invAp"], c["Vol"], c["inj"])


@pytest.mark.parametrize("ci", range(3))
def test_oracle_matches_literal_transliteration(ci):
    c = GOLD["cases"][ci]
    ops = _case_ops(c)
    f = np.array(c["f0"])
    for st in c["steps"]:
        f, diag, _ = ops.step(f, c["dt_scale"], c["verbose"])
        exp = np.array([dec(x) for x in st["f"]])
        np.testing.assert_allclose(f, exp, rtol=1e-14, atol=1e-300)
        d = st["diag"]
        assert bool(diag[4]) == d["finite"]
        for k, key in enumerate(("Cr", "Cr_Bin", "Cr_Emi", "Cr_Flux")):
            e = dec(d[key])
            if math.isinf(e):
                assert diag[k] == e
            else:
                assert diag[k] == pytest.approx(e, rel=1e-12, abs=1e-300)


def test_kat_injection_only():
    k = GOLD["kat_inj"]
    n = len(k["f0"])
    ops = oracle.RefOperands(n, 1, None, None, sp.csc_matrix((n, n)), np.ones(n), [1.0], k["inj"])
    f = np.array(k["f0"])
    for _ in range(k["steps"]):
        f, _, _ = ops.step(f, k["dt_scale"])
    np.testing.assert_array_equal(f, k["expect"])


def test_kat_upwind_flux():
    k = GOLD["kat_flux"]
    n = len(k["f0"])
    F = sp.csc_matrix((k["nzval"], k["rowval"], k["colptr"]), shape=(n, n))
    ops = oracle.RefOperands(n, 1, None, None, F, np.ones(n), [1.0], np.zeros(n))
    f, _, _ = ops.step(np.array(k["f0"]), k["dt_scale"])
    np.testing.assert_allclose(f, k["expect"], rtol=0, atol=1e-16)
    assert f.sum() == pytest.approx(sum(k["f0"]), rel=1e-15)  # upwind flux conserves number


def test_kat_clamp_table():
    k = GOLD["kat_clamp"]
    for x, y, neg in zip(k["in"], k["out"], k["signbit"]):
        got = oracle.clamp(dec(x))
        assert got == dec(y)
        assert math.copysign(1.0, got) < 0 if neg else True


def test_kat_schedule():
    k = GOLD["kat_sched"]
    sched = oracle.solve_schedule(k["dt_initial"], k["t_save"], k["dt0"])
    assert [len(s[1]) for s in sched] == k["counts"] == [3, 8, 1]
    for (_, scales, _), exp in zip(sched, k["scales"]):
        assert scales == exp  # bit-exact host arithmetic
    # the truncated dt carries over into the next interval (Solver.jl:35)
    assert sched[1][1][0] == sched[0][1][-1]
    k = GOLD["kat_sched32"]
    sched = oracle.solve_schedule(k["dt_initial"], k["t_save"], float(np.float32(k["dt0"])))
    assert sched[0][1] == k["scales"][0]


def test_blocked_equals_reference_layout():
    w = synth.small(p_num=4, u_num=3, seed=5, randomize_vectors=True)
    b = oracle.blocked_from_workload(w)
    r = oracle.ref_from_workload(w)
    f, g = w.f0.copy(), w.f0.copy()
    for _ in range(10):
        f, d1, _ = b.step(f, 0.9, 3)
        g, d2, _ = r.step(g, 0.9, 3)
    assert np.max(np.abs(f - g)) / np.max(np.abs(g)) < 1e-14
    np.testing.assert_allclose(d1[:4], d2[:4], rtol=1e-12)


def test_blocked_equals_reference_layout_uneven_species():
    """Species of different sizes (electrons 4 x 3 = 12 states, photons 5 x 2 = 10): the blocked
    operands (gain blocks n_out x n_e x n_g, both loss sides, emission) and the reference-layout
    M_Bin and M_Emi they expand to step alike."""
    w = synth.uneven_two_species(4, 3, 5, 2, seed=9)
    assert w.ps.species_sizes == [12, 10]
    b = oracle.blocked_from_workload(w)
    r = oracle.ref_from_workload(w)
    f, g = w.f0.copy(), w.f0.copy()
    for _ in range(10):
        f, d1, _ = b.step(f, 0.9, 3)
        g, d2, _ = r.step(g, 0.9, 3)
    assert np.max(np.abs(f - g)) / np.max(np.abs(g)) < 1e-14
    np.testing.assert_allclose(d1[:4], d2[:4], rtol=1e-12)


def test_conserving_gain_loss_preserves_number():
    """KAT 3: gain/loss built to conserve number per species (flux and emission off)."""
    w = synth.small(p_num=4, u_num=2, seed=8, with_emission=False)
    ns = w.ps.species_sizes[0]
    Ge = np.asarray(w.binm.gains[0].G)  # out e
    Gg = np.asarray(w.binm.gains[1].G)  # out gamma
    from dtb.structs import LossBlock
    w.binm.losses = [LossBlock(0, 1, Ge.sum(axis=0)), LossBlock(1, 0, Gg.sum(axis=0).T)]
    n = w.ps.n_state
    ops = oracle.BlockedOperands(w.ps.species_sizes, 1, w.binm.gains, w.binm.losses, [], sp.csc_matrix((n, n)),
                                 np.ones(n), [1.0], np.zeros(n))
    f = w.f0.copy()
    n0 = [f[:ns].sum(), f[ns:].sum()]
    for _ in range(50):
        f, _, _ = ops.step(f, 1.0)
    assert f.min() > 0
    assert abs(f[:ns].sum() - n0[0]) / n0[0] < 1e-13
    assert abs(f[ns:].sum() - n0[1]) / n0[1] < 1e-13


def test_blocked_to_ref_index_map():
    """A single gain value lands as val/2 at the two M_Bin positions of BuildBinaryMatrices.jl:194-195."""
    from dtb.structs import BinaryMatrices, GainBlock, LossBlock, PhaseSpace
    ps = PhaseSpace(name_list=["A", "B"], px_num_list=[2, 3], py_num_list=[1, 1], pz_num_list=[1, 1])
    G = np.zeros((2, 2, 3))
    G[1, 0, 2] = 4.0  # a = 1, b = 0 (species A), c = 2 of species B -> global c = 4
    L = np.zeros((2, 3))
    L[0, 1] = 6.0  # a = 0, c = global 3
    M = blocked_to_ref(ps, BinaryMatrices(gains=[GainBlock(0, 0, 1, G)], losses=[LossBlock(0, 1, L)]))
    N = 5
    assert M[0 * N + 1, 4] == 2.0 and M[4 * N + 1, 0] == 2.0
    assert M[0 * N + 0, 3] == -3.0 and M[3 * N + 0, 0] == -3.0
    assert np.count_nonzero(M) == 4


def test_symplectic_reduces_to_euler_without_space_flux():
    """With X = 0 the symplectic step equals the plain step up to the two clamp thresholds."""
    w = synth.small(p_num=4, u_num=2, seed=4)
    r = oracle.ref_from_workload(w)
    f = w.f0.copy()
    d = np.zeros(8)
    n = w.ps.n_state
    L = oracle.lib()
    fs = f.copy()
    zero = np.zeros(n + 1, dtype=np.int64)
    rc = L.orc_step_symplectic_ref(r.n_mom, r.n_space, oracle._d(r.M_Bin), oracle._d(r.M_Emi),
                                   oracle._i(zero), oracle._i(np.zeros(1, dtype=np.int64)), oracle._d(np.zeros(1)),
                                   oracle._i(r.colptr), oracle._i(r.rowval), oracle._d(r.nzval), 0,
                                   oracle._d(r.invAp), oracle._d(r.Vol), oracle._d(r.inj), 1.0,
                                   oracle.THR_F64, float(np.float32(1e-20)), 1, oracle._d(fs), oracle._d(d),
                                   oracle._b(r.dom))
    assert rc == 0
    fe, _, _ = r.step(f, 1.0)
    np.testing.assert_allclose(fs, fe, rtol=1e-14, atol=1e-300)


def test_bin_domain_semantics():
    """BinM.Domain (SteppingMethods.jl:355-369): the binary term acts only in listed cells; a
    domain of every cell equals `nothing`; the blocked and reference layouts agree; a cell
    outside the domain whose f is all zero is still evaluated (an Inf in M_Bin then makes
    df non-finite there while the nonzero cells outside stay untouched)."""
    from dtb.structs import BinaryMatrices
    w = synth.small(p_num=5, u_num=3, seed=21, n_space=3, randomize_vectors=True)
    n_mom = w.ps.n_momentum
    f = w.f0.copy()
    r_all = oracle.ref_from_workload(w)
    w.binm.Domain = [0, 1, 2]
    r_every = oracle.ref_from_workload(w)
    np.testing.assert_array_equal(r_all.step(f, 0.8, 3)[0], r_every.step(f, 0.8, 3)[0])
    w.binm.Domain = [1, 7, -2]  # entries that name no cell match nothing
    r_dom = oracle.ref_from_workload(w)
    b_dom = oracle.blocked_from_workload(w)
    f_dom, d_dom, df_dom = r_dom.step(f, 0.8, 3)
    fb, db, dfb = b_dom.step(f, 0.8, 3)
    np.testing.assert_allclose(dfb, df_dom, rtol=1e-12, atol=1e-300)
    w_nobin = synth.small(p_num=5, u_num=3, seed=21, n_space=3, randomize_vectors=True)
    w_nobin.binm = BinaryMatrices()
    _, _, df_nobin = oracle.ref_from_workload(w_nobin).step(f, 0.8, 3)
    _, _, df_full = r_all.step(f, 0.8, 3)
    cells = lambda v, k: v[k * n_mom:(k + 1) * n_mom]  # noqa: E731
    for k in (0, 2):
        np.testing.assert_array_equal(cells(df_dom, k), cells(df_nobin, k))
    np.testing.assert_array_equal(cells(df_dom, 1), cells(df_full, 1))
    # the all-zero exception
    M = np.array(r_dom.M_Bin)
    M[0, 0] = np.inf
    f0 = f.copy()
    f0[2 * n_mom:] = 0.0
    rz = oracle.RefOperands(n_mom, 3, M, r_dom.M_Emi, w.fluxm.F_Flux, r_dom.invAp, r_dom.Vol, r_dom.inj,
                            domain=[])
    _, dz, dfz = rz.step(f0, 0.8, 1)
    assert dz[4] == 0 and np.isnan(cells(dfz, 2)).any()
    assert np.all(np.isfinite(cells(dfz, 0))) and np.all(np.isfinite(cells(dfz, 1)))
