"""DTB_PROFILE: every context appends one JSON summary line at dtb_destroy (its shape, the steps
it launched, its device bytes, and for a batched context its gain-GEMM plans), and every server
one at dtb_serve_destroy (requests served, instance-steps/s, p50/p99 time to solution)."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys
sys.path.insert(0, sys.argv[1])
import numpy as np
from dtb import synth
from dtb.batch import BatchedEuler
from dtb.stepping import ForwardEulerStruct
w = synth.small(p_num=8, u_num=4, seed=3)
m = ForwardEulerStruct(w.ps, w.f0, w.inj, w.binm, w.emim, w.fluxm, Precision=np.float64)
m.run(np.ones(20))
m.close()
wb = synth.batched_two_species(8, 1e-2, 1e2, 4, 8, seed=4)
b = BatchedEuler(wb.ps, wb.inj, wb.binm, wb.emim, wb.fluxm, 8)
for i in range(8):
    b.admit(i, wb.f0[i], float(wb.dt[i]), 30)
b.run(30)
b.close()
from dtb.serve import Server
g = BatchedEuler(wb.ps, wb.inj, wb.binm, wb.emim, wb.fluxm, 2)
srv = Server()
gid = srv.add_grid(g)
srv.start()
for rid in [srv.submit(gid, wb.f0[i], float(wb.dt[i]), 20 + 10 * i) for i in range(3)]:
    srv.wait(rid, timeout_s=60, with_f=False)
srv.close()
g.close()
"""


def test_profile_summary_lines(cuda, tmp_path):
    out = tmp_path / "prof.jsonl"
    env = dict(os.environ, DTB_PROFILE=str(out))
    subprocess.run([sys.executable, "-c", SCRIPT, os.path.join(ROOT, "diplodocustransport.jl_b200")], env=env,
                   check=True, timeout=300)
    lines = [json.loads(x) for x in out.read_text().splitlines() if x.strip()]
    assert len(lines) == 4
    plain, batched, server, grid = lines
    assert plain["precision"] == 0 and plain["n_state"] == 64 and plain["steps_run"] == 20
    assert plain["device_bytes"] > 0
    assert batched["precision"] == 2 and batched["batch"] == 8 and batched["steps_run"] == 30
    assert batched["batched_steps"] == 30 and len(batched["gemm_plans"]) == 1
    assert server["server"] == 1 and server["completed"] == 3 and server["instance_steps"] == 20 + 30 + 40
    assert 0 < server["tts_p50_s"] <= server["tts_p99_s"]
    assert grid["precision"] == 2 and grid["batch"] == 2
