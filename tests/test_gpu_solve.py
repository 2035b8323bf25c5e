"""The pipelined Solve (dtb_solve / dtb_solve_ex): the whole schedule enqueued without a host
round trip per save interval, save points copied out behind the stepping, moments of every
saved state computed on the device.

Bar: the saved states are bit-identical to the reference-shaped stepwise loop (one functor call
per step, Solver.jl:25-43) on the same context; device moments equal the FP64 sums of the saved
states to 1e-12 relative (FP64 state) or 1e-6 (FP32 state, sums in FP64 of FP32 values).
"""
import numpy as np
import pytest

from dtb import synth
from dtb.stepping import ForwardEulerStruct, Solve, solve_schedule
from dtb.structs import energy_weights

pytestmark = pytest.mark.gpu


def _method(w, precision=np.float64, **kw):
    return ForwardEulerStruct(w.ps, w.f0, w.inj, w.binm, w.emim, w.fluxm, Precision=precision, **kw)


@pytest.mark.parametrize("precision", [np.float64, np.float32])
def test_many_irregular_saves_bitwise(cuda, precision):
    """40 save points at irregular times, so intervals end mid-graph and the truncated dt of the
    first save (0.25) is carried into the later intervals (Solver.jl:35). Save times are
    multiples of 0.25 so the carried dt stays 0.25 (an arbitrary grid would shrink it at every
    save until the schedule explodes, as the reference would)."""
    w = synth.small(p_num=8, u_num=4, seed=41, randomize_vectors=True)
    rng = np.random.default_rng(3)
    t_save = [0.0, 3.25] + list(3.25 + 0.25 * np.cumsum(rng.integers(1, 40, 39)))
    per, _ = solve_schedule(0.5, t_save, 1.0)
    assert per.sum() < 2000
    m = _method(w, precision, graph_steps=8)
    a = Solve(m, 0.5, t_save, Verbose=0, stepwise=True)
    b = Solve(m, 0.5, t_save, Verbose=0)
    assert len(b.f) == len(t_save)
    for x, y in zip(a.f, b.f):
        np.testing.assert_array_equal(x, y)
    m.close()


def test_schedule_longer_than_one_chunk(cuda):
    """70,000 steps: the dt staging wraps (65,536 steps per chunk) with save points on both
    sides of the boundary."""
    w = synth.small(p_num=4, u_num=2, seed=42, randomize_vectors=True)
    t_save = [0.0, 10000.0, 33000.0, 65530.0, 65540.0, 70000.0]
    assert solve_schedule(1.0, t_save, 1.0)[0].sum() == 70000
    m = _method(w)
    a = Solve(m, 1.0, t_save, Verbose=0, stepwise=True)
    b = Solve(m, 1.0, t_save, Verbose=0)
    assert b.n_steps == 70000
    for x, y in zip(a.f, b.f):
        np.testing.assert_array_equal(x, y)
    m.close()


@pytest.mark.parametrize("precision,rel", [(np.float64, 1e-12), (np.float32, 1e-6)])
def test_device_moments_of_every_save(cuda, precision, rel):
    """Moments at each of 12 save points on a 2-cell grid equal the sums of the saved states."""
    w = synth.small(p_num=6, u_num=3, seed=43, n_space=2, randomize_vectors=True)
    wts = energy_weights(w.ps)
    t_save = [0.0] + [3.0 * k + 0.5 for k in range(1, 12)]
    m = _method(w, precision)
    out = Solve(m, 0.5, t_save, Verbose=0, moment_weights=wts)
    ref = Solve(m, 0.5, t_save, Verbose=0)
    assert out.n_steps == 67
    sizes = w.ps.species_sizes
    n_mom = w.ps.n_momentum
    assert out.number.shape == (len(t_save), 2, len(sizes))
    for k, f in enumerate(out.f):
        np.testing.assert_array_equal(f, ref.f[k])
        for cell in range(2):
            off = cell * n_mom
            for s in range(len(sizes)):
                lo = off + sum(sizes[:s])
                sl = slice(lo, lo + sizes[s])
                ws = wts[lo - off:lo - off + sizes[s]]
                assert out.number[k, cell, s] == pytest.approx(f[sl].sum(), rel=rel, abs=1e-300)
                assert out.energy[k, cell, s] == pytest.approx((f[sl] * ws).sum(), rel=rel, abs=1e-300)
    m.close()


def test_verbose_lines_in_step_order(cuda, capfd):
    """Verbose = 2 prints one Cr line per step (SteppingMethods.jl:83-85), in step order, from
    the diagnostics read back behind the stepping."""
    w = synth.small(p_num=4, u_num=2, seed=44)
    m = _method(w, graph_steps=4)
    out = Solve(m, 1.0, [0.0, 7.0, 19.0, 30.0], Verbose=2)
    txt = capfd.readouterr().out
    ts = [float(part.split("t=")[1].split(",")[0]) for part in txt.replace("\r", "\n").splitlines() if "t=" in part]
    assert len(ts) == out.n_steps == 30
    assert ts == sorted(ts) and ts[0] == 0.0
    m.close()
