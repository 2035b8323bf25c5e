"""Edge cases through the C ABI: species of different sizes, zero-length runs, batches with no
running slot, slots admitted for zero steps.

Tolerances as elsewhere: relative L-inf 1e-12 (plain FP64) and 2e-5 (plain FP32) against the FP64
oracle, 1e-5 for the batched mixed-precision path.
"""
import numpy as np
import pytest

import oracle
from dtb import synth
from dtb.batch import BatchedEuler, set_tune_cache
from dtb.stepping import ForwardEulerStruct

pytestmark = pytest.mark.gpu

TOL64, TOL32, TOL_MIXED = 1e-12, 2e-5, 1e-5


def rel_linf(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(np.asarray(b))))


def _oracle_run(w, f0, dt, n):
    ops = oracle.blocked_from_workload(w)
    f = np.array(f0, dtype=np.float64)
    for _ in range(n):
        f, _, _ = ops.step(f, dt, 0)
    return f


@pytest.mark.parametrize("precision,tol", [(np.float64, TOL64), (np.float32, TOL32)])
@pytest.mark.parametrize("grid", [(10, 8, 12, 4), (5, 3, 7, 2)])
def test_plain_uneven_species_match_oracle(cuda, precision, tol, grid):
    """Electrons and photons on grids of different sizes (80 and 48 states; 15 and 14): gain blocks
    n_out x n_e x n_g, loss blocks of both sides and emission, 40 steps (two graphs of 16 and 8
    single steps)."""
    w = synth.uneven_two_species(*grid, seed=21)
    m = ForwardEulerStruct(w.ps, w.f0, w.inj, w.binm, w.emim, w.fluxm, Precision=precision, graph_steps=16)
    m.run(np.full(40, 0.9))
    assert rel_linf(m.f, _oracle_run(w, w.f0, 0.9, 40)) <= tol
    m.close()


def test_reference_layout_upload_uneven_species(cuda):
    """The reference's dense M_Bin (N^2 x N) and M_Emi of an uneven grid (15 + 14 states),
    decomposed by the library into blocks, step like the blocked upload (1e-13) and like the
    oracle (1e-12)."""
    from dtb.structs import BinaryMatrices, EmissionMatrices, blocked_to_ref, emission_to_dense
    w = synth.uneven_two_species(5, 3, 7, 2, seed=25)
    a = ForwardEulerStruct(w.ps, w.f0, w.inj, w.binm, w.emim, w.fluxm)
    b = ForwardEulerStruct(w.ps, w.f0, w.inj, BinaryMatrices(M_Bin=blocked_to_ref(w.ps, w.binm)),
                           EmissionMatrices(M_Emi=emission_to_dense(w.ps, w.emim)), w.fluxm)
    a.run(np.full(24, 0.9))
    b.run(np.full(24, 0.9))
    assert rel_linf(b.f, a.f) <= 1e-13
    assert rel_linf(b.f, _oracle_run(w, w.f0, 0.9, 24)) <= TOL64
    a.close()
    b.close()


@pytest.mark.parametrize("case", ["no_binary", "empty_domain"])
def test_plain_without_gain_kernel_runs_in_graphs(cuda, case):
    """Steps with no gain kernel (no binary term, or a binary domain with no cell): each row
    kernel follows the previous one in plain stream order. 45 steps through dtb_run (a loose
    step, two graphs of 16, 12 loose steps) against the FP64 oracle."""
    from dtb.structs import BinaryMatrices
    w = synth.small(p_num=8, u_num=4, seed=31, n_space=2, randomize_vectors=True)
    if case == "no_binary":
        w.binm = BinaryMatrices()
    else:
        w.binm.Domain = []
    m = ForwardEulerStruct(w.ps, w.f0, w.inj, w.binm, w.emim, w.fluxm, graph_steps=16)
    m.run(np.full(45, 0.9))
    assert rel_linf(m.f, _oracle_run(w, w.f0, 0.9, 45)) <= TOL64
    m.close()


def _diag_tuple(d):
    return (d.cr, d.cr_bin, d.cr_emi, d.cr_flux, d.sum_df, d.sum_f, d.finite)


@pytest.mark.parametrize("graph_steps", [4, 16, 0])
@pytest.mark.parametrize("symplectic", [False, True])
def test_step_records_do_not_depend_on_launch_grouping(cuda, graph_steps, symplectic):
    """The per-step diagnostics (Cr, Cr_Bin, Cr_Emi, Cr_Flux, sum df, sum f, finite) of 37 steps
    run as graph replays and loose sequences equal, bit for bit, those of 37 single dtb_step
    calls, and (forward Euler) match the oracle's (rtol 1e-10); the states agree bit for bit.
    dtb_launch_count counts the kernels of every step (gain and rows; the symplectic method's
    two row passes) plus one diagnostics reduction per sequence."""
    import ctypes
    from dtb.stepping import ForwardSymplecticEulerStruct
    w = synth.small(p_num=10, u_num=4, seed=32, n_space=2, randomize_vectors=True)
    cls = ForwardEulerStruct
    if symplectic:
        w.fluxm.X_Flux = synth.space_flux(w.ps, np.random.default_rng(6), 1.0)
        cls = ForwardSymplecticEulerStruct
    n = 37
    a = cls(w.ps, w.f0, w.inj, w.binm, w.emim, w.fluxm, graph_steps=graph_steps)
    b = cls(w.ps, w.f0, w.inj, w.binm, w.emim, w.fluxm, graph_steps=graph_steps)
    c0, c1 = ctypes.c_int64(), ctypes.c_int64()
    a.L.dtb_launch_count(a.ctx, ctypes.byref(c0))
    sc = (0.9 * a.dt0) / a.dt0  # the dt / dt0 dtb_step forms from dt = 0.9 dt0
    hist = a.run(np.full(n, sc), Verbose=3, diag=True)
    a.L.dtb_launch_count(a.ctx, ctypes.byref(c1))
    gs = graph_steps or 64  # 0: the default, 64 steps per graph on this grid
    graphs, loose = n // gs, n % gs
    per_step = 3 if symplectic else 2
    assert c1.value - c0.value == per_step * n + graphs + (1 if loose else 0)
    ops = oracle.blocked_from_workload(w)
    f = np.array(w.f0, dtype=np.float64)
    for k in range(n):
        b(0.0, 1e9, 0.9 * b.dt0, 3)
        assert _diag_tuple(hist[k]) == _diag_tuple(b.last_diag), k
        if symplectic:
            assert hist[k].finite == 1 and hist[k].cr_bin == 0.0 and hist[k].sum_df == 0.0
            continue
        f, diag, _ = ops.step(f, sc, 3)
        for got, exp in zip(_diag_tuple(hist[k])[:4], diag[:4]):
            assert got == pytest.approx(exp, rel=1e-10), k
        assert bool(hist[k].finite) == bool(diag[4])
    np.testing.assert_array_equal(a.f, b.f)
    a.close()
    b.close()


def test_plain_zero_length_run_leaves_the_state(cuda):
    w = synth.small(p_num=6, u_num=2, seed=4)
    m = ForwardEulerStruct(w.ps, w.f0, w.inj, w.binm, w.emim, w.fluxm)
    f0 = m.f
    m.run(np.zeros(0))
    np.testing.assert_array_equal(m.f, f0)
    m.close()


@pytest.mark.parametrize("grid,B", [((10, 8, 12, 4), 12), ((20, 8, 12, 8), 40)])
def test_batched_uneven_species_match_oracle(cuda, grid, B):
    """Batched mixed precision on uneven species. 80 + 48 states: the 32-row epilogue tile of
    rows 64-95 straddles the species boundary (the direct-load path), one 128-row m tile.
    160 + 96 states: two m tiles (N1 = 160, n2 = 96 padded to 128). 30 steps, instances with their
    own dt, against the FP64 oracle."""
    w = synth.uneven_two_species(*grid, seed=22, batch=B)
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
    for i in range(B):
        m.admit(i, w.f0[i], w.dt[i], 30)
    m.run(30)
    for i in (0, B // 2, B - 1):
        assert rel_linf(m.get_f(i), _oracle_run(w, w.f0[i], w.dt[i], 30)) <= TOL_MIXED, i
    m.close()


def test_batched_uneven_species_on_sm_pairs(cuda, tmp_path):
    """The 160 + 96-state grid forced onto the SM-pair GEMM (M = 256: two m tiles) through the plan
    cache: within 1e-5 of the FP64 oracle after 20 steps."""
    import torch
    B = 64
    w = synth.uneven_two_species(20, 8, 12, 8, seed=23, batch=B)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    key = f"sm{sms}:M256:N1160:n296:cols{B}:cells1"
    cache = tmp_path / "plans.txt"
    cache.write_text(f"{key} 1 256 30 0\n")
    set_tune_cache(str(cache))
    try:
        m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
    finally:
        set_tune_cache(None)
    assert m.gemm_plan(0)["pair"]
    for i in range(B):
        m.admit(i, w.f0[i], w.dt[i], 20)
    m.run(20)
    for i in (0, 33, B - 1):
        assert rel_linf(m.get_f(i), _oracle_run(w, w.f0[i], w.dt[i], 20)) <= TOL_MIXED, i
    m.close()


def test_batched_idle_runs_and_zero_step_slots(cuda):
    """run(0) does nothing; a slot admitted for 0 steps never steps; once every slot has finished,
    further runs (the GEMM then has no live column) leave every state as it was; a finished slot
    re-admitted steps again and matches the oracle."""
    B = 8
    w = synth.batched_two_species(8, 1e-2, 1e2, 4, B, seed=24)
    m = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, B)
    for i in range(B):
        m.admit(i, w.f0[i], w.dt[i], 0 if i == 3 else 5)
    f3 = m.get_f(3)
    m.run(0)
    assert all(m.info(i)["steps_done"] == 0 for i in range(B))
    m.run(5)
    np.testing.assert_array_equal(m.get_f(3), f3)
    assert m.info(3)["steps_done"] == 0 and m.info(0)["steps_done"] == 5
    snap = m.get_f_all()
    m.run(20)  # nothing runs
    np.testing.assert_array_equal(m.get_f_all(), snap)
    m.admit(5, w.f0[5], w.dt[5], 7)
    m.run(7)
    assert rel_linf(m.get_f(5), _oracle_run(w, w.f0[5], w.dt[5], 7)) <= TOL_MIXED
    assert m.info(5)["steps_done"] == 7
    m.close()
