"""Batched mixed-precision path (tcgen05 gain GEMM, BF16 hi+lo operands) against the FP64 oracle.

Tolerances: the gain term alone within 2e-5 (normwise relative) of the FP64 contraction; whole
runs within relative L-infinity 1e-5 of the FP64 oracle run with the same dt per instance.
"""
import contextlib

import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from dtb import synth
from dtb.batch import BatchedEuler, set_tune_cache
from dtb.structs import BinaryMatrices, EmissionMatrices, LossBlock

pytestmark = pytest.mark.gpu

TOL_GAIN = 2e-5
TOL_RUN = 1e-5


def _plan_key(w, batch):
    """Autotuner key of the two-species workloads' one gain group (e, gamma inputs)."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    n1, n2 = w.ps.species_sizes[0], w.ps.species_sizes[1]
    cols = w.ps.n_space * ((batch + 3) // 4 * 4)
    return f"sm{sms}:M{sum(w.ps.species_sizes)}:N1{n1}:n2{n2}:cols{cols}:cells{w.ps.n_space}"


@contextlib.contextmanager
def forced_plan(tmp_path, w, batch, plan):
    """Commits inside the block use the gain GEMM plan `plan` = (pair, bn, splits) for this
    shape, read from a plan cache file instead of measured (None: the autotuner's choice)."""
    if plan is None:
        yield
        return
    cache = tmp_path / "plans.txt"
    cache.write_text(f"{_plan_key(w, batch)} {plan[0]} {plan[1]} {plan[2]} 0\n")
    set_tune_cache(str(cache))
    try:
        yield
    finally:
        set_tune_cache(None)


def rel_linf(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(np.asarray(b))))


def _gain_only(w):
    n = w.ps.n_state
    w.binm = BinaryMatrices(gains=w.binm.gains)
    w.emim = EmissionMatrices()
    w.fluxm.P_Flux = sp.csc_matrix((n, n))
    w.fluxm.X_Flux = sp.csc_matrix((n, n))
    w.inj = np.zeros(n)
    return w


@pytest.mark.parametrize("p,u,batch,plan", [
    (8, 4, 8, None), (16, 8, 100, None), (8, 8, 300, None), (12, 6, 40, None),
    (16, 8, 100, (0, 128, 37)), (8, 8, 300, (0, 256, 37)), (8, 8, 300, (0, 128, 20)),
    (10, 8, 300, (1, 256, 37)), (16, 8, 260, (1, 256, 37)), (16, 8, 260, (1, 256, 13)),
    (10, 8, 300, (0, 64, 37))])
def test_batched_gain_term_matches_fp64(cuda, tmp_path, p, u, batch, plan):
    """One step with only the gain term: f1 - f0 = gain; covers BN = 64, 128, 256 on one SM and
    the SM-pair kernel (plans forced through the cache file, or the autotuner's choice), several
    N tiles, n2 padded to 64 (p*u = 32, 72, 80), more than one M tile, K splits aligned to the
    input-2 blocks and not (13 splits of 20 K tiles, one crossing the block boundary). On SM
    pairs: rows past M in the second m tile (M = 160), and a second column tile with 44 or 4
    running columns. The gain's error grows with the K range of a split (each split sums its
    range in one FP32 tensor-memory accumulator): a forced 5-split plan (3,328 K values per
    accumulator) reached 2.003e-5 here, the autotuner's plans fill the device with 36-37 splits."""
    w = _gain_only(synth.batched_two_species(p, 1e-2, 1e2, u, batch, seed=p * 100 + u))
    for g in w.binm.gains:  # make the gain dominate the step
        g.G = np.asarray(g.G) * 50.0
    with forced_plan(tmp_path, w, batch, plan):
        m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, batch)
    if plan is not None:
        got = m.gemm_plan(0)
        assert (got["pair"], got["bn"]) == (bool(plan[0]), plan[1])
    for i in range(batch):
        m.admit(i, w.f0[i], 1.0, 1)
    m.run(1)
    ns = w.ps.species_sizes[0]
    Ge = np.asarray(w.binm.gains[0].G)
    Gg = np.asarray(w.binm.gains[1].G)
    for i in list(range(min(batch, 6))) + [batch - 1]:
        f0 = w.f0[i]
        gain = np.concatenate([oracle.gain_rows(Ge, 0, ns, f0[:ns], f0[ns:]),
                               oracle.gain_rows(Gg, 0, ns, f0[:ns], f0[ns:])])
        got = m.get_f(i) - f0
        assert rel_linf(got, gain) <= TOL_GAIN, i
    m.close()


def test_batched_run_matches_oracle(cuda):
    """All operators, per-instance dt, 60 steps."""
    w = synth.batched_two_species(8, 1e-2, 1e2, 4, 12, seed=5)
    rng = np.random.default_rng(1)
    w.inj = rng.uniform(0, 1e-4, w.ps.n_state)
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 12)
    for i in range(12):
        m.admit(i, w.f0[i], w.dt[i], 60)
    m.run(60)
    ops = oracle.blocked_from_workload(w)
    for i in range(12):
        f = w.f0[i].copy()
        for _ in range(60):
            f, _, _ = ops.step(f, w.dt[i], 0)
        assert rel_linf(m.get_f(i), f) <= TOL_RUN, i
        info = m.info(i)
        assert info["steps_done"] == 60 and info["steps_left"] == 0 and info["finite"]
    m.close()


def test_slot_alone_equals_slot_in_mix(cuda):
    """A solve gives the same result alone in the batch and among other running solves."""
    w = synth.batched_two_species(8, 1e-2, 1e2, 4, 16, seed=6)
    a = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 16)
    b = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 16)
    a.admit(3, w.f0[3], w.dt[3], 40)
    for i in range(16):
        b.admit(i, w.f0[i], w.dt[i], 40 + 7 * i)
    a.run(40)
    b.run(40)
    np.testing.assert_array_equal(a.get_f(3), b.get_f(3))
    a.close()
    b.close()


def test_stop_and_readmit(cuda):
    w = synth.batched_two_species(8, 1e-2, 1e2, 4, 4, seed=7)
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 4)
    m.admit(0, w.f0[0], w.dt[0], 10)
    m.admit(1, w.f0[1], w.dt[1], 25)
    m.run(20)
    f10 = m.get_f(0)
    m.run(10)
    np.testing.assert_array_equal(m.get_f(0), f10)  # finished slots do not step
    assert m.info(0)["steps_done"] == 10 and m.info(1)["steps_done"] == 25
    # re-admit slot 0 mid-run: it restarts from its new initial state
    m.admit(0, w.f0[2], w.dt[2], 5)
    m.run(5)
    ops = oracle.blocked_from_workload(w)
    f = w.f0[2].copy()
    for _ in range(5):
        f, _, _ = ops.step(f, w.dt[2], 0)
    assert rel_linf(m.get_f(0), f) <= TOL_RUN
    m.close()


def test_config2_sampled_instances(cuda):
    """Config 2 (256 instances, N_s = 256, shared G 2 x 256 x 65,536): 24 steps, 3 instances
    checked against the FP64 oracle."""
    w = synth.config2(seed=2, gain_on_device=True)
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 256)
    for i in range(256):
        m.admit(i, w.f0[i], w.dt[i], 24)
    m.run(24)
    gains = [type(g)(g.out_sp, g.in1_sp, g.in2_sp, g.G.double().cpu().numpy()) for g in w.binm.gains]
    ops = oracle.BlockedOperands(w.ps.species_sizes, 1, gains, w.binm.losses, w.emim.blocks, w.fluxm.F_Flux,
                                 1.0 / np.asarray(w.fluxm.Ap_Flux), w.fluxm.Vol, w.inj)
    for i in (0, 101, 255):
        f = w.f0[i].copy()
        for _ in range(24):
            f, _, _ = ops.step(f, w.dt[i], 0)
        assert rel_linf(m.get_f(i), f) <= TOL_RUN, i
    m.close()


def test_three_species_three_interactions_matches_oracle(cuda):
    """The config-3 recipe (e-, e+, gamma; Compton-like and pair gain/loss; synchrotron-like
    emission) on a small grid: three gain groups with stacked rows, 40 steps vs FP64 oracle."""
    w = synth.three_species(8, 1e-3, 1e3, 6, 8, seed=11)
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 8)
    for i in range(8):
        m.admit(i, w.f0[i], w.dt[i], 40)
    m.run(40)
    ops = oracle.blocked_from_workload(w)
    for i in (0, 3, 7):
        f = w.f0[i].copy()
        for _ in range(40):
            f, _, _ = ops.step(f, w.dt[i], 0)
        assert rel_linf(m.get_f(i), f) <= TOL_RUN, i
    m.close()


def test_config3_full_size_moments(cuda):
    """Config 3 at full size (64 instances, 576 states per species, 4.6 GB of BF16 hi+lo gain per
    step): 50 steps stay finite; FP64 device moments equal the FP64 sums of the returned f."""
    from dtb.structs import energy_weights
    w = synth.config3(seed=3, batch=64, gain_on_device=True)
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 64)
    for i in range(64):
        m.admit(i, w.f0[i], w.dt[i], 50)
    wts = energy_weights(w.ps)
    num0, en0 = m.moments(wts)
    m.run(50)
    num1, en1 = m.moments(wts)
    for i in (0, 63):
        info = m.info(i)
        assert info["finite"] and info["steps_done"] == 50
        f = m.get_f(i)
        ns = w.ps.species_sizes[0]
        for s in range(3):
            assert num1[i, s] == pytest.approx(f[s * ns:(s + 1) * ns].sum(), rel=1e-12)
            assert en1[i, s] == pytest.approx((f * wts)[s * ns:(s + 1) * ns].sum(), rel=1e-12)
    assert np.all(np.isfinite(num1)) and np.all(num1 > 0)
    m.close()


def test_config3_full_size_matches_plain_fp64(cuda):
    """Config 3 at full size against the plain FP64 GPU path (which the tests hold to 1e-12 of
    the FP64 oracle) on the same operators promoted to FP64 (9.2 GB): 200 batched steps, three
    instances with their own dt within relative L-inf 1e-5, and their FP64 number moments
    within 1e-5 of the FP64 path's."""
    import torch
    from dtb.structs import energy_weights
    from dtb.stepping import ForwardEulerStruct
    n_steps = 200
    w = synth.config3(seed=3, batch=64, gain_on_device=True)
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 64)
    for i in range(64):
        m.admit(i, w.f0[i], w.dt[i], n_steps)
    m.run(n_steps)
    wts = energy_weights(w.ps)
    num, _ = m.moments(wts)
    g64 = [type(g)(g.out_sp, g.in1_sp, g.in2_sp, g.G.double()) for g in w.binm.gains]
    plain = ForwardEulerStruct(w.ps, w.f0[0], w.inj, BinaryMatrices(gains=g64, losses=w.binm.losses), w.emim,
                               w.fluxm, Precision=np.float64)
    del g64
    torch.cuda.empty_cache()
    for i in (0, 31, 63):
        plain.f = w.f0[i]
        plain.run(np.full(n_steps, float(w.dt[i])))
        assert rel_linf(m.get_f(i), plain.f) <= TOL_RUN, i
        pn, _ = plain.moments(wts)
        assert np.all(np.abs(num[i] - np.asarray(pn)[0]) / np.abs(np.asarray(pn)[0]) <= 1e-5), i
    plain.close()
    m.close()


def test_whole_batch_state_io(cuda):
    """set_f_all / get_f_all move the slot-major FP64 batch through the device transpose: the
    round trip keeps the FP32 hi+lo pair's precision, equals the per-slot reads, and a run
    after set_f_all steps from the uploaded state (37 slots: the capacity pads to 40)."""
    B = 37
    w = synth.batched_two_species(8, 1e-2, 1e2, 4, B, seed=9)
    n = w.ps.n_state
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
    for i in range(B):
        m.admit(i, w.f0[i], w.dt[i], 10)
    rng = np.random.default_rng(3)
    F = rng.lognormal(-2.0, 3.0, size=(B, n))
    m.set_f_all(F)
    G = m.get_f_all()
    assert G.shape == (B, n)
    assert float(np.max(np.abs(G - F) / F)) <= 2.0 ** -45
    for i in (0, 17, B - 1):
        np.testing.assert_array_equal(m.get_f(i), G[i])
    m.set_f_all(w.f0)
    m.run(10)
    G = m.get_f_all()
    ops = oracle.blocked_from_workload(w)
    for i in (0, B - 1):
        f = w.f0[i].copy()
        for _ in range(10):
            f, _, _ = ops.step(f, w.dt[i], 0)
        assert rel_linf(G[i], f) <= TOL_RUN, i
        np.testing.assert_array_equal(m.get_f(i), G[i])
    m.close()


def test_run_io_equals_separate_io_calls(cuda):
    """dtb_batch_run_io (upload, steps, download under one wait) gives bit-identical states to
    set_f_all + run + get_f_all on a second context; the same array may be input and output,
    and a None input keeps the device state."""
    B = 37
    w = synth.batched_two_species(8, 1e-2, 1e2, 4, B, seed=23)
    a = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
    b = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
    for m in (a, b):
        for i in range(B):
            m.admit(i, w.f0[i], w.dt[i], 40)
    F = np.array(w.f0, dtype=np.float64)
    b.set_f_all(F)
    for nsteps in (1, 3, 20):
        b.run(nsteps)
        ref = b.get_f_all()
        F = a.run_io(F, nsteps, F)
        np.testing.assert_array_equal(F, ref)
    b.run(2)
    np.testing.assert_array_equal(a.run_io(None, 2), b.get_f_all())
    a.close()
    b.close()


def test_page_locked_and_pageable_host_arrays_agree(cuda):
    """Batch I/O through page-locked host arrays (an array that starts inside a larger pinned
    buffer) and through pageable arrays gives bit-identical states, through run_io and
    set_f_all / get_f_all."""
    import torch
    B = 37
    w = synth.batched_two_species(8, 1e-2, 1e2, 4, B, seed=24)
    n = w.ps.n_state
    a = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
    b = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
    for m in (a, b):
        for i in range(B):
            m.admit(i, w.f0[i], w.dt[i], 40)
    big = torch.zeros((B + 3) * n, dtype=torch.float64).pin_memory().numpy()
    P = big[n:n + B * n].reshape(B, n)
    P[:] = w.f0
    F = np.array(w.f0, dtype=np.float64)
    for nsteps in (1, 5):
        a.run_io(P, nsteps, P)
        F = b.run_io(F, nsteps, F)
        np.testing.assert_array_equal(P, F)
    Q = torch.empty((B, n), dtype=torch.float64).pin_memory().numpy()
    a.set_f_all(P)
    a.get_f_all(Q)
    np.testing.assert_array_equal(Q, P)
    a.close()
    b.close()


def test_run_io_round_trip_graph_follows_host_buffers(cuda):
    """One-step round trips through page-locked arrays replay a captured graph per state buffer
    with the caller's host addresses patched into its copies: alternating between two pinned
    buffers (and switching input and output) over 7 steps gives bit-identical states to
    set_f_all + run + get_f_all on a second context."""
    import torch
    B = 21
    w = synth.batched_two_species(8, 1e-2, 1e2, 4, B, seed=25)
    n = w.ps.n_state
    a = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
    b = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
    for m in (a, b):
        for i in range(B):
            m.admit(i, w.f0[i], w.dt[i], 40)
    X = torch.empty((B, n), dtype=torch.float64).pin_memory().numpy()
    Y = torch.empty((B, n), dtype=torch.float64).pin_memory().numpy()
    X[:] = w.f0
    b.set_f_all(np.array(w.f0, dtype=np.float64))
    src, dst = X, Y
    for _ in range(7):
        a.run_io(src, 1, dst)
        b.run(1)
        np.testing.assert_array_equal(dst, b.get_f_all())
        src, dst = dst, src
    a.close()
    b.close()


@pytest.mark.parametrize("p,u,plan", [(8, 4, None), (10, 8, (1, 256, 37)), (10, 8, (0, 256, 37)),
                                      (10, 8, (0, 128, 37))])
def test_gemm_columns_follow_the_last_running_slot(cuda, tmp_path, p, u, plan):
    """The gain GEMM computes only up to the last running slot (rounded to 16 columns, 32 on SM
    pairs): a slot alone at index 3 or 200 of 256, and the same slot with every slot running,
    give the same f; finished slots keep their state while a higher slot runs on. (10, 8) has
    two m tiles and runs, forced, on SM pairs and on one SM."""
    B = 256
    w = synth.batched_two_species(p, 1e-2, 1e2, u, B, seed=12)
    with forced_plan(tmp_path, w, B, plan):
        full = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
        for i in range(B):
            full.admit(i, w.f0[i], w.dt[i], 30)
        full.run(30)
        for slot in (3, 200):
            one = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
            assert one.gemm_plan(0) == full.gemm_plan(0)
            one.admit(slot, w.f0[slot], w.dt[slot], 30)
            one.admit(0, w.f0[0], w.dt[0], 5)
            one.run(30)
            np.testing.assert_array_equal(one.get_f(slot), full.get_f(slot))
            assert one.info(0)["steps_done"] == 5
            one.close()
        if plan is not None:
            assert (full.gemm_plan(0)["pair"], full.gemm_plan(0)["bn"]) == (bool(plan[0]), plan[1])
        full.close()


def test_sm_pair_gemm_agrees_with_one_sm_gemm(cuda, tmp_path):
    """The SM-pair gain GEMM (two m tiles per MMA) and the one-SM kernel, each forced through a
    plan cache file, form the same products in the same K order: 8 steps of every operator on
    300 slots agree to 1e-6 (relative L-infinity per slot), and both stay within the FP64
    oracle's tolerance."""
    B = 300
    w = synth.batched_two_species(10, 1e-2, 1e2, 8, B, seed=21)
    cache = tmp_path / "plans.txt"
    out = {}
    try:
        for pair in (1, 0):
            cache.write_text(f"{_plan_key(w, B)} {pair} 256 37 0\n")
            set_tune_cache(str(cache))
            m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
            plan = m.gemm_plan(0)
            assert plan["pair"] == bool(pair) and plan["bn"] == 256 and plan["tuned_us"] == 0.0
            for i in range(B):
                m.admit(i, w.f0[i], w.dt[i], 8)
            m.run(8)
            out[pair] = m.get_f_all()
            m.close()
    finally:
        set_tune_cache(None)
    a, b = out[1], out[0]
    for i in range(B):
        assert rel_linf(a[i], b[i]) <= 1e-6, i
    ops = oracle.blocked_from_workload(w)
    for i in (0, 257, B - 1):
        f = w.f0[i].copy()
        for _ in range(8):
            f, _, _ = ops.step(f, w.dt[i], 0)
        assert rel_linf(a[i], f) <= TOL_RUN, i


def test_autotuned_plan_is_measured_shared_and_recorded(cuda, tmp_path):
    """The autotuner times the candidate plans of a new shape once (the chosen plan carries its
    measured time), a second context of the same shape reuses it and steps bit-identically, the
    cache file gets one line for the shape, and DTB_FLAG_NO_AUTOTUNE takes the fixed rule."""
    B = 260
    w = synth.batched_two_species(16, 1e-2, 1e2, 8, B, seed=22)
    cache = tmp_path / "plans.txt"
    set_tune_cache(str(cache))
    try:
        a = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
        pa = a.gemm_plan(0)
        assert a.gemm_plan(1) is None
        assert pa["tuned_us"] > 0 and pa["bn"] in (64, 128, 256) and pa["n_splits"] >= 1
        b = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
        assert b.gemm_plan(0) == pa
        lines = [ln for ln in cache.read_text().splitlines() if ln.strip()]
        assert len(lines) == 1 and lines[0].startswith(_plan_key(w, B) + " ")
        fields = lines[0].split()
        assert (int(fields[1]) == 1) == pa["pair"] and int(fields[2]) == pa["bn"]
        for m in (a, b):
            for i in range(B):
                m.admit(i, w.f0[i], w.dt[i], 6)
            m.run(6)
        np.testing.assert_array_equal(a.get_f_all(), b.get_f_all())
        a.close()
        b.close()
        c = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B, autotune=False)
        pc = c.gemm_plan(0)
        assert pc["tuned_us"] == 0.0 and pc["bn"] == 256 and pc["pair"]  # M = 256: two m tiles
        c.close()
    finally:
        set_tune_cache(None)


def _multicell(n_space, seed, domain=None):
    w = synth.small(p_num=8, u_num=4, seed=seed, n_space=n_space, randomize_vectors=True)
    w.fluxm.X_Flux = synth.space_flux(w.ps, np.random.default_rng(seed + 1), 1.0)
    w.binm.Domain = domain
    return w


@pytest.mark.parametrize("n_space,domain", [(3, None), (4, [0, 2]), (2, [])])
def test_multicell_slots_match_oracle(cuda, n_space, domain):
    """Slots of several space cells (update_Big_Bin!'s loop over cells, SteppingMethods.jl:360-386):
    every (cell, slot) pair is a gain-GEMM column, each cell with its Vol and BinM.Domain, a
    space flux coupling the cells; 6 slots with their own f0 and dt, 30 steps, against the FP64
    oracle of the same multi-cell grid."""
    w = _multicell(n_space, 60 + n_space, domain)
    n = w.ps.n_state
    rng = np.random.default_rng(5)
    f0s = [w.f0 * rng.uniform(0.7, 1.3, n) for _ in range(6)]
    dts = rng.uniform(0.5, 1.0, 6)
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 6)
    for i in range(6):
        m.admit(i, f0s[i], dts[i], 30)
    m.run(30)
    ops = oracle.blocked_from_workload(w)
    for i in range(6):
        f = f0s[i].copy()
        for _ in range(30):
            f, _, _ = ops.step(f, dts[i], 0)
        assert rel_linf(m.get_f(i), f) <= TOL_RUN, i
    m.close()


def test_multicell_slots_on_sm_pairs(cuda, tmp_path):
    """Multi-cell columns through the SM-pair GEMM (forced): 2 cells x 100 slots = 200 columns
    of one 256-column tile (224 computed), two m tiles (M = 160); 10 steps against the FP64
    oracle of the same two-cell grid for three slots."""
    w = synth.small(p_num=10, u_num=8, seed=66, n_space=2, randomize_vectors=True)
    w.fluxm.X_Flux = synth.space_flux(w.ps, np.random.default_rng(67), 1.0)
    B = 100
    n = w.ps.n_state
    rng = np.random.default_rng(6)
    f0s = [w.f0 * rng.uniform(0.7, 1.3, n) for _ in range(B)]
    dts = rng.uniform(0.5, 1.0, B)
    with forced_plan(tmp_path, w, B, (1, 256, 37)):
        m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
    assert m.gemm_plan(0)["pair"]
    for i in range(B):
        m.admit(i, f0s[i], dts[i], 10)
    m.run(10)
    ops = oracle.blocked_from_workload(w)
    for i in (0, 57, B - 1):
        f = f0s[i].copy()
        for _ in range(10):
            f, _, _ = ops.step(f, dts[i], 0)
        assert rel_linf(m.get_f(i), f) <= TOL_RUN, i
    m.close()


def test_multicell_moments_and_bulk_io(cuda):
    """Per-(slot, cell, species) FP64 moments and whole-batch state I/O with cells."""
    from dtb.structs import energy_weights
    w = _multicell(3, 71)
    n = w.ps.n_state
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 5)
    rng = np.random.default_rng(2)
    F = np.stack([w.f0 * rng.uniform(0.5, 1.5, n) for _ in range(5)])
    for i in range(5):
        m.admit(i, F[i], 0.8, 10)
    m.run(10)
    G = m.get_f_all()
    assert G.shape == (5, n)
    wts = energy_weights(w.ps)
    num, en = m.moments(wts)
    sizes = w.ps.species_sizes
    nm = w.ps.n_momentum
    assert num.shape == (5, 3, len(sizes))
    for i in range(5):
        np.testing.assert_array_equal(m.get_f(i), G[i])
        for cell in range(3):
            for s in range(len(sizes)):
                lo = cell * nm + sum(sizes[:s])
                sl = slice(lo, lo + sizes[s])
                assert num[i, cell, s] == pytest.approx(G[i][sl].sum(), rel=1e-12)
                assert en[i, cell, s] == pytest.approx((G[i][sl] * wts[sum(sizes[:s]):sum(sizes[:s]) + sizes[s]]).sum(),
                                                       rel=1e-12)
    m.close()


def test_number_conservation_plain_and_batched(cuda):
    """Known answer: gain and loss built to conserve number per species (flux and emission off)
    keep sum(f) of each species over 50 steps: to FP64 rounding on the plain FP64 path, and to
    the BF16 hi+lo contraction's accuracy on the batched path, with FP64 device moments."""
    from dtb.stepping import ForwardEulerStruct
    from dtb.structs import FluxMatrices
    w = synth.small(p_num=8, u_num=4, seed=8, with_emission=False)
    ns = w.ps.species_sizes[0]
    n = w.ps.n_state
    Ge = np.asarray(w.binm.gains[0].G)
    Gg = np.asarray(w.binm.gains[1].G)
    w.binm.losses = [LossBlock(0, 1, Ge.sum(axis=0)), LossBlock(1, 0, Gg.sum(axis=0).T)]
    w.fluxm = FluxMatrices(Ap_Flux=np.ones(n), Am_Flux=-np.ones(n), X_Flux=sp.csc_matrix((n, n)),
                           P_Flux=sp.csc_matrix((n, n)), Vol=np.ones(1))
    w.inj = np.zeros(n)
    n0 = [w.f0[:ns].sum(), w.f0[ns:].sum()]
    m = ForwardEulerStruct(w.ps, w.f0, w.inj, w.binm, w.emim, w.fluxm, Precision=np.float64)
    for _ in range(50):
        m(0.0, 1e9, 1.0, 0)
    f = m.f
    assert f.min() > 0
    assert abs(f[:ns].sum() - n0[0]) / n0[0] < 1e-12
    assert abs(f[ns:].sum() - n0[1]) / n0[1] < 1e-12
    m.close()
    b = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 4)
    for i in range(4):
        b.admit(i, w.f0 * (1.0 + 0.1 * i), 1.0, 50)
    b.run(50)
    num, _ = b.moments(np.ones(w.ps.n_momentum))
    for i in range(4):
        for s_ in range(2):
            assert abs(num[i, s_] - n0[s_] * (1.0 + 0.1 * i)) / (n0[s_] * (1.0 + 0.1 * i)) < 1e-5
    b.close()


def test_batched_cr_and_finite_flags_match_oracle(cuda):
    """Per-slot diagnostics: the largest Cr = -min(df ./ f) over a slot's steps
    (SteppingMethods.jl:48-94) and the finite flag, against the FP64 oracle's per-step Cr."""
    w = synth.batched_two_species(8, 1e-2, 1e2, 4, 5, seed=14)
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 5)
    for i in range(5):
        m.admit(i, w.f0[i], w.dt[i], 20)
    m.run(20)
    ops = oracle.blocked_from_workload(w)
    for i in range(5):
        f = w.f0[i].copy()
        crs = []
        for _ in range(20):
            f, d, _ = ops.step(f, w.dt[i], 1)
            crs.append(d[0])
        info = m.info(i)
        assert info["finite"]
        assert info["cr_max"] == pytest.approx(max(crs), rel=1e-4), i
    m.close()


def _moments_oracle(ps, f):
    from dtb.structs import energy_weights
    wts = energy_weights(ps)
    off = ps.momentum_species_offset
    sizes = ps.species_sizes
    return (np.array([f[off[s]:off[s] + sizes[s]].sum() for s in range(len(sizes))]),
            np.array([(f[off[s]:off[s] + sizes[s]] * wts[off[s]:off[s] + sizes[s]]).sum() for s in range(len(sizes))]))


@pytest.mark.parametrize("n_steps", [5000, 10000])
def test_long_run_matches_oracle_with_drift(cuda, n_steps):
    """Mixed precision over a configuration's full run length (5,000 steps as config 3, 10,000
    as config 2) on a reduced grid (2 species x 32 states, 16 instances, every operator, per-
    instance dt, injection): every instance within relative L-inf 1e-5 of the FP64 oracle run;
    the FP64 device moments of the mixed run within relative 1e-5 of the oracle's number and
    energy per species at the end, i.e. the mixed path's number and energy drift is the oracle's
    own to 1e-5."""
    from dtb.structs import energy_weights
    w = synth.batched_two_species(8, 1e-2, 1e2, 4, 16, seed=31)
    rng = np.random.default_rng(2)
    w.inj = rng.uniform(0, 1e-4, w.ps.n_state)
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 16)
    for i in range(16):
        m.admit(i, w.f0[i], w.dt[i], n_steps)
    wts = energy_weights(w.ps)
    num0, en0 = m.moments(wts)
    m.run(n_steps)
    num1, en1 = m.moments(wts)
    ops = oracle.blocked_from_workload(w)
    for i in range(16):
        f = w.f0[i].copy()
        for _ in range(n_steps):
            f, _, _ = ops.step(f, w.dt[i], 0)
        assert rel_linf(m.get_f(i), f) <= TOL_RUN, i
        on, oe = _moments_oracle(w.ps, f)
        assert np.all(np.abs(num1[i] - on) / np.abs(on) <= 1e-5), i
        assert np.all(np.abs(en1[i] - oe) / np.abs(oe) <= 1e-5), i
    m.close()


def test_long_run_number_conservation(cuda):
    """Known answer over 5,000 steps: gain and loss built to conserve number per species (flux
    and emission off); the mixed path's FP64 device number moments stay within 1e-5 of the
    initial number (the FP64 oracle conserves it to rounding)."""
    from dtb.structs import FluxMatrices
    w = synth.small(p_num=8, u_num=4, seed=8, with_emission=False)
    ns = w.ps.species_sizes[0]
    n = w.ps.n_state
    Ge = np.asarray(w.binm.gains[0].G)
    Gg = np.asarray(w.binm.gains[1].G)
    w.binm.losses = [LossBlock(0, 1, Ge.sum(axis=0)), LossBlock(1, 0, Gg.sum(axis=0).T)]
    w.fluxm = FluxMatrices(Ap_Flux=np.ones(n), Am_Flux=-np.ones(n), X_Flux=sp.csc_matrix((n, n)),
                           P_Flux=sp.csc_matrix((n, n)), Vol=np.ones(1))
    w.inj = np.zeros(n)
    n0 = np.array([w.f0[:ns].sum(), w.f0[ns:].sum()])
    b = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 4)
    for i in range(4):
        b.admit(i, w.f0 * (1.0 + 0.1 * i), 0.5 + 0.1 * i, 5000)
    b.run(5000)
    num, _ = b.moments(np.ones(w.ps.n_momentum))
    for i in range(4):
        ref = n0 * (1.0 + 0.1 * i)
        assert np.all(np.abs(num[i] - ref) / ref < 1e-5), (i, num[i], ref)
    ops = oracle.blocked_from_workload(w)
    f = w.f0.copy()
    for _ in range(5000):
        f, _, _ = ops.step(f, 0.5, 0)
    assert abs(f[:ns].sum() - n0[0]) / n0[0] < 1e-12 and abs(f[ns:].sum() - n0[1]) / n0[1] < 1e-12
    b.close()


def test_nan_seeded_slot_is_flagged_and_leaves_the_others_alone(cuda):
    """Host-side fault injection on the batched numeric path: one slot's f0 carries a NaN. That
    slot's finite flag drops and its state clamps to zeros (x * (x >= thr), Julia's strong
    zero); every other slot is bit-identical to the same batch without the NaN."""
    B = 8
    w = synth.batched_two_species(8, 1e-2, 1e2, 4, B, seed=27)
    a = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
    b = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
    for i in range(B):
        f = w.f0[i].copy()
        if i == 3:
            f[7] = np.nan
        a.admit(i, f, w.dt[i], 5)
        b.admit(i, w.f0[i], w.dt[i], 5)
    a.run(5)
    b.run(5)
    assert not a.info(3)["finite"] and np.all(a.get_f(3) == 0)
    for i in range(B):
        if i != 3:
            assert a.info(i)["finite"]
            np.testing.assert_array_equal(a.get_f(i), b.get_f(i))
    a.close()
    b.close()
