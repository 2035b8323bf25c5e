"""Host-side checks that need no GPU: the C ABI loads and exports every declared symbol,
the library's Solve schedule equals the oracle's, and the synthetic workloads keep their
recorded properties."""
import ctypes
import json
import os
import re

import numpy as np
import pytest

import oracle
from dtb import _lib, synth
from dtb.stepping import solve_schedule

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "golden_small.json")))


def _declared_symbols():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names |= set(re.findall(r"^\s*(?:int32_t|const char\*|void)\s+(dtb_\w+)\s*\(", txt, re.M))
    return names


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    names = _declared_symbols()
    assert len(names) >= 25
    for n in sorted(names):
        assert hasattr(L, n), n
    # every declared symbol has a Python binding with a signature
    assert names <= set(_lib.SIGNATURES), sorted(names - set(_lib.SIGNATURES))
    assert L.dtb_abi_version() == 1


def test_library_exports_match_nm():
    """The shared object's dynamic symbol table holds exactly the dtb_ names the headers declare."""
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\sT\s(dtb_\w+)$", out, re.M))
    assert exported == _declared_symbols()


def test_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    L = _lib.load()
    dims = _lib.Dims(n_species=1, n_space=1)
    dims.species_size[0] = 4
    opts = _lib.Opts(precision=0, device=0, index_base=0, dt0=1.0, batch=1)
    ctx = ctypes.c_void_p()
    rc = L.dtb_create(ctypes.byref(dims), ctypes.byref(opts), ctypes.byref(ctx))
    assert rc == _lib.DTB_ENODEV
    assert b"device" in L.dtb_last_error()


def test_bad_arguments_are_rejected():
    L = _lib.load()
    dims = _lib.Dims(n_species=0, n_space=1)
    opts = _lib.Opts(precision=0, device=0, index_base=0, dt0=1.0, batch=1)
    ctx = ctypes.c_void_p()
    assert L.dtb_create(ctypes.byref(dims), ctypes.byref(opts), ctypes.byref(ctx)) == _lib.DTB_EINVAL
    dims.n_species = 1
    dims.species_size[0] = 4
    opts.precision = 7
    assert L.dtb_create(ctypes.byref(dims), ctypes.byref(opts), ctypes.byref(ctx)) == _lib.DTB_EINVAL
    assert L.dtb_create(None, None, None) == _lib.DTB_EINVAL
    opts.precision = _lib.DTB_F64
    for bad in (-1, 1025, 2 ** 31 - 1):  # refused on the host, before any device is touched
        opts.graph_steps = bad
        assert L.dtb_create(ctypes.byref(dims), ctypes.byref(opts), ctypes.byref(ctx)) == _lib.DTB_EINVAL
        assert b"graph_steps" in L.dtb_last_error()
    # entry points on a null context refuse before touching a device
    n = ctypes.c_int64()
    assert L.dtb_launch_count(None, ctypes.byref(n)) == _lib.DTB_EINVAL
    f = np.zeros(4)
    assert L.dtb_step_io(None, _lib.dptr(f), _lib.dptr(f), 0.0, 1.0, 0.5, 0, None, None, None) == _lib.DTB_EINVAL


@pytest.mark.parametrize("dt,t_save", [(0.4, [0.0, 1.0, 2.5, 2.6]), (0.3, [0.0, 1.0, 2.0, 3.0]),
                                       (0.3, list(np.linspace(0, 7, 11))), (1.0, [0.0, 1000.0]), (0.25, [0.0, 1.0, 2.5, 3.0]),
                                       (0.07, [0.0, 0.5, 0.51, 2.0])])
@pytest.mark.parametrize("prec,dt0", [(_lib.DTB_F64, 1.0), (_lib.DTB_F64, 0.3), (_lib.DTB_F32, 0.1)])
def test_solve_schedule_matches_oracle(dt, t_save, prec, dt0):
    d0 = float(np.float32(dt0)) if prec == _lib.DTB_F32 else dt0
    try:
        ref = oracle.solve_schedule(dt, t_save, d0, max_steps=2_000_000)
    except ValueError:  # carried dt collapsed: both sides must refuse
        with pytest.raises(_lib.DtbError):
            solve_schedule(dt, t_save, dt0, prec)
        return
    per, scales = solve_schedule(dt, t_save, dt0, prec)
    assert list(per) == [len(s[1]) for s in ref]
    assert list(scales) == [x for s in ref for x in s[1]]  # bit-exact


def test_solve_schedule_carried_dt_explosion_is_reported():
    """dt = 0.1 over [0, 1]: 0.1 * 10 falls 1.1e-16 short of 1, the last step is truncated to
    1.1e-16 and Solve keeps that dt (Solver.jl:35), so the next interval would need ~1e16 steps.
    The library refuses instead of spinning; the oracle does the same."""
    with pytest.raises(_lib.DtbError) as e:
        solve_schedule(0.1, [0.0, 1.0, 2.0], 1.0)
    assert e.value.code == _lib.DTB_EINVAL and b"Solver.jl:35" in _lib.load().dtb_last_error()
    with pytest.raises(ValueError):
        oracle.solve_schedule(0.1, [0.0, 1.0, 2.0], 1.0)


def test_solve_schedule_golden():
    k = GOLD["kat_sched"]
    per, scales = solve_schedule(k["dt_initial"], k["t_save"], k["dt0"])
    assert list(per) == k["counts"]
    assert list(scales) == [x for s in k["scales"] for x in s]
    k = GOLD["kat_sched32"]
    per, scales = solve_schedule(k["dt_initial"], k["t_save"], k["dt0"], _lib.DTB_F32)
    assert list(scales) == k["scales"][0]


def test_synthetic_flux_is_conserving_and_scaled():
    w = synth.small(p_num=8, u_num=4, seed=2)
    F = w.fluxm.F_Flux.toarray()
    np.testing.assert_allclose(F.sum(axis=0), 0.0, atol=1e-14)  # number conserving columns
    assert np.all(np.diag(F) >= 0)
    rho = np.max(np.abs(np.linalg.eigvals(F)))
    assert rho * w.dt == pytest.approx(synth.CFL_TARGET, rel=1e-9)
    assert max(np.count_nonzero(F, axis=1)) <= 5


def test_synthetic_config0_shapes():
    w = synth.config0(0)
    assert w.ps.species_sizes == [128, 128]
    assert [g.G.shape for g in w.binm.gains] == [(128, 128, 128)] * 2
    assert [l.L.shape for l in w.binm.losses] == [(128, 128)] * 2
    assert w.emim.blocks[0].E.shape == (128, 128)
    assert w.f0[:128].sum() == pytest.approx(1.0) and w.f0[128:].sum() == pytest.approx(1.0)
    g = np.asarray(w.binm.gains[0].G) / w.meta["kappa_gain"]
    assert g.min() >= 1e-6 and g.max() <= 1.0


def test_server_host_errors_without_a_device():
    """Server errors that need no GPU: starting without grids, unknown grids and requests."""
    import ctypes
    L = _lib.load()
    srv = ctypes.c_void_p()
    opts = _lib.ServeOpts(hbm_budget_bytes=0, max_chunk_steps=0, flags=0, chunk_ms=0.0)
    assert L.dtb_serve_create(ctypes.byref(opts), ctypes.byref(srv)) == _lib.DTB_OK
    assert L.dtb_serve_start(srv) == _lib.DTB_ESTATE
    f = np.zeros(4)
    rid = ctypes.c_int64()
    assert L.dtb_serve_submit(srv, 0, _lib.dptr(f), 1.0, 10, ctypes.byref(rid)) == _lib.DTB_ENOTFOUND
    st = _lib.RequestStats()
    assert L.dtb_serve_wait(srv, 7, 0.01, None, ctypes.byref(st)) == _lib.DTB_ENOTFOUND
    assert L.dtb_serve_destroy(srv) == _lib.DTB_OK


def test_entry_scripts_compile_and_bench_parses_its_arguments():
    """bench.py and __graft_entry__.py are valid Python, and bench.py answers --help without a
    device (its argument parser is reachable before any CUDA call)."""
    import py_compile
    import subprocess
    import sys
    for name in ("bench.py", "__graft_entry__.py"):
        py_compile.compile(os.path.join(ROOT, name), doraise=True)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0, out.stderr
    assert "--config" in out.stdout and "--impl" in out.stdout


@pytest.mark.parametrize("path", [("diplodocustransport.jl_b200", "julia", "DTB200Backend.jl"),
                                  ("INTEGRATION.md",)])
def test_julia_binding_calls_only_declared_exported_symbols(path):
    """Every C function the Julia backend and the integration guide call
    (ccall((:dtb_..., libdtb), ...)) is declared in include/dtb.h, exported by the library, and
    given as many argument types as the declaration has parameters (no Julia toolchain here to
    run the binding itself)."""
    jl = open(os.path.join(ROOT, *path)).read()
    header = open(os.path.join(ROOT, "include", "dtb.h")).read()
    lib = _lib.load()
    calls = re.findall(r"ccall\(\(:(dtb_\w+),\s*libdtb\),\s*\w+(?:\{\w+\})?,\s*\(([^()]*(?:\([^()]*\))?[^()]*)\)", jl)
    names = {n for n, _ in calls}
    assert len(calls) == jl.count("ccall((:dtb_")
    assert {"dtb_create", "dtb_step"} <= names
    for name, argtypes in calls:
        m = re.search(r"\b" + name + r"\s*\(([^;]*)\)\s*;", header)
        assert m, name
        params = m.group(1).strip()
        n_decl = 0 if params in ("", "void") else params.count(",") + 1
        n_jl = len([a for a in argtypes.split(",") if a.strip()])
        assert n_jl == n_decl, (name, n_jl, n_decl)
        assert hasattr(lib, name), name


def test_reference_arm_prints_one_contract_line():
    """bench.py --impl reference runs the FP64 oracle port on the host cores (no device) and
    prints exactly one JSON line with the keys of the measurement contract, the same config
    object as the GPU arm, and e2e copies of zero bytes."""
    import json
    import subprocess
    import sys
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "3"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 3
    assert d["unit"] == "instance-steps/s" and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("batching (config 2)") and d["config"]["batch"] == 256


def test_tune_cache_is_host_only(tmp_path):
    """dtb_set_tune_cache needs no device: it loads a cache file (recorded lines and a file that
    does not exist yet alike) and forgets the plans with NULL."""
    L = _lib.load()
    cache = tmp_path / "plans.txt"
    cache.write_text("sm148:M512:N1256:n2256:cols256:cells1 1 256 37 37.267\n")
    assert L.dtb_set_tune_cache(str(cache).encode()) == _lib.DTB_OK
    assert L.dtb_set_tune_cache(str(tmp_path / "new.txt").encode()) == _lib.DTB_OK
    assert L.dtb_set_tune_cache(None) == _lib.DTB_OK
    assert not (tmp_path / "new.txt").exists()  # written only when a plan is measured


def test_gain_contract_entries_refuse_misaligned_pointers_on_the_host():
    """Both kernel-level entries check alignment before any CUDA call (no device needed): G must
    be 16-byte aligned (bulk copies), out 8-byte aligned, f1 and f2 aligned to their element."""
    import ctypes
    from dtb import _lib
    L = _lib.load()
    P = ctypes.c_void_p
    ok, g_bad, o_bad = P(0x10000), P(0x10008), P(0x10004)
    for fn in (L.dtb_gain_contract, L.dtb_gain_contract_noalloc):
        assert fn(_lib.DTB_DTYPE_F32, g_bad, 8, 8, 8, ok, ok, ok, None) == _lib.DTB_EINVAL
        assert b"16-byte aligned" in L.dtb_last_error()
        assert fn(_lib.DTB_DTYPE_F32, ok, 8, 8, 8, ok, ok, o_bad, None) == _lib.DTB_EINVAL
        assert fn(_lib.DTB_DTYPE_F64, ok, 8, 8, 8, o_bad, ok, ok, None) == _lib.DTB_EINVAL


def test_last_ptr_follows_the_array_object():
    """The round-trip bindings reuse the ctypes pointer of the array passed last; another array
    object (or None) is converted afresh."""
    p = _lib.LastPtr()
    a, b = np.zeros(8), np.ones(8)
    pa = p(a)
    assert ctypes.addressof(pa.contents) == a.ctypes.data
    assert p(a) is pa
    pb = p(b)
    assert pb is not pa and ctypes.addressof(pb.contents) == b.ctypes.data
    assert p(None) is None
    assert ctypes.addressof(p(a).contents) == a.ctypes.data
