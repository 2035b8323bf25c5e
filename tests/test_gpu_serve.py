"""Serving loop (continuous batching over batched contexts of two grids) through the C ABI.

Each served result must equal the same request run alone (relative L-infinity <= 1e-12; the
per-instance arithmetic does not depend on the other slots) and match the FP64 oracle within
1e-5."""
import numpy as np
import pytest

import oracle
from dtb import _lib, synth
from dtb.batch import BatchedEuler
from dtb.serve import Server

pytestmark = pytest.mark.gpu


def rel_linf(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(np.asarray(b))))


def _grids():
    return [synth.batched_two_species(8, 1e-2, 1e2, 4, 6, seed=21),
            synth.batched_two_species(8, 1e-2, 1e2, 8, 6, seed=22)]


def test_served_results_equal_alone_and_oracle(cuda):
    ws = _grids()
    cap = 4
    srv = Server(max_chunk_steps=16)
    ctxs = [BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, cap) for w in ws]
    gids = [srv.add_grid(b) for b in ctxs]
    srv.start()
    rng = np.random.default_rng(3)
    reqs = []
    for k in range(14):  # more requests than slots: later ones join as earlier ones finish
        g = k % 2
        i = int(rng.integers(0, 6))
        steps = int(rng.integers(10, 90))
        rid = srv.submit(gids[g], ws[g].f0[i], float(ws[g].dt[i]), steps)
        reqs.append((rid, g, i, steps))
    results = {rid: srv.wait(rid, timeout_s=120) for rid, *_ in reqs}
    stats = srv.stats()
    srv.close()
    assert stats["completed"] == 14 and stats["instance_steps"] == sum(r[3] for r in reqs)
    for rid, g, i, steps in reqs[:6]:
        f_srv, info = results[rid]
        assert info["t_submit"] <= info["t_admit"] <= info["t_done"] and info["finite"]
        alone = BatchedEuler(ws[g].ps, ws[g].inj, ws[g].binm, ws[g].emim, ws[g].fluxm, cap)
        alone.admit(0, ws[g].f0[i], float(ws[g].dt[i]), steps)
        alone.run(steps)
        assert rel_linf(f_srv, alone.get_f(0)) <= 1e-12
        alone.close()
        ops = oracle.blocked_from_workload(ws[g])
        f = ws[g].f0[i].copy()
        for _ in range(steps):
            f, _, _ = ops.step(f, float(ws[g].dt[i]), 0)
        assert rel_linf(f_srv, f) <= 1e-5
    for b in ctxs:
        b.close()


def test_grid_over_hbm_budget_is_refused(cuda):
    w = _grids()[0]
    b = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 4)
    srv = Server(hbm_budget_bytes=1024)
    with pytest.raises(_lib.DtbError) as e:
        srv.add_grid(b)
    assert e.value.code == _lib.DTB_ENOMEM
    srv.close()
    b.close()


def test_wait_times_out_and_unknown_ids(cuda):
    w = _grids()[0]
    b = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 4)
    srv = Server()
    gid = srv.add_grid(b)
    with pytest.raises(_lib.DtbError) as e:
        srv.wait(12345)
    assert e.value.code == _lib.DTB_ENOTFOUND
    srv.start()
    rid = srv.submit(gid, w.f0[0], float(w.dt[0]), 200000)
    with pytest.raises(_lib.DtbError) as e:
        srv.wait(rid, timeout_s=0.2)
    assert e.value.code == _lib.DTB_ETIMEOUT
    srv.close()
    b.close()


def test_cancelled_requests_free_their_slots(cuda):
    """Host-side fault injection: a running request and a queued one are cancelled. The queued
    one leaves the queue at once, the running one frees its slot at the next chunk boundary;
    waiting on either reports DTB_ESTATE, and later requests run in the freed slot and match the
    same request run alone."""
    w = _grids()[0]
    b = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 1)
    srv = Server(max_chunk_steps=16)
    gid = srv.add_grid(b)
    srv.start()
    long_id = srv.submit(gid, w.f0[0], float(w.dt[0]), 10_000_000)
    queued_id = srv.submit(gid, w.f0[1], float(w.dt[1]), 50)
    srv.cancel(queued_id)
    with pytest.raises(_lib.DtbError) as e:
        srv.wait(queued_id, timeout_s=30)
    assert e.value.code == _lib.DTB_ESTATE
    srv.cancel(long_id)
    with pytest.raises(_lib.DtbError) as e:
        srv.wait(long_id, timeout_s=30)
    assert e.value.code == _lib.DTB_ESTATE
    rid = srv.submit(gid, w.f0[2], float(w.dt[2]), 40)
    f_srv, info = srv.wait(rid, timeout_s=60)
    st = srv.stats()
    srv.close()
    assert info["finite"] and st["completed"] == 1 and st["instance_steps"] == 40
    alone = BatchedEuler(w.ps, w.inj, w.binm, w.emim, w.fluxm, 1)
    alone.admit(0, w.f0[2], float(w.dt[2]), 40)
    alone.run(40)
    assert rel_linf(f_srv, alone.get_f(0)) <= 1e-12
    alone.close()
    b.close()
